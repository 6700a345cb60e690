// Class-update kernels of the plain chains (int8 / float32 spins, packed words) and the sequential reference.
//
// One class launch updates every site of one (colour, sublattice) class of every replica
// (Spin_Colour_Kernel/generator.py:150-319). A thread owns one (replica, class site); class sites of a row are
// x0 + P j with P the x-period of the colouring, so no thread is spent on sites of other colours. Float32
// arithmetic uses explicit round-to-nearest intrinsics in the reference's operation order (no FMA
// contraction), so only the transcendental functions (cos, sin, exp) differ from the reference's CPU path.
//
// Ising never evaluates exp on the device: the energy change of an Ising flip is one of finitely many values,
// fixed by the integer group sums G_g, the extra-bond neighbours and the own spin. The host builds, for every
// replica, a float32 table of exp(-beta dE) (Metropolis) or exp(beta dE) (Barker) over that key space with the
// same float32 arithmetic and exp as the reference's CPU path, so Ising decisions are bit-exact.
#include <stdio.h>

#include "site.cuh"

namespace sck {

// --------------------------------------------------------------------------------------------- dispatchers
template <int N, typename ST>
__device__ __forceinline__ void plain_site(const Common& c, const SubDev& sub, int alpha, int rep, int x, int y,
                                           int z, int32_t key) {
  const size_t base = (size_t)rep * N * c.g.nsite;
  if constexpr (N == 1) {
    ising_site<ST>(c, sub, alpha, rep, x, y, z, key, (const ST*)c.src + base, (ST*)c.dst + base);
  } else {
    vec_site<N>(c, sub, alpha, rep, x, y, z, key, (const float*)c.src + base, (float*)c.dst + base);
  }
}

// Grid (ceil(rows * bx / 256), replicas): thread t of a replica owns class site t = row * bx + j.
template <int N, typename ST>
__global__ void __launch_bounds__(256) plain_class_kernel(const __grid_constant__ ClassParams p) {
  const uint32_t per_rep = (uint32_t)p.c.rows * (uint32_t)p.c.bx;
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= per_rep) return;
  int x, y, z;
  if (!class_site(p.c, p.colour, p.alpha, t, x, y, z)) return;
  const int32_t key = sweep_key(p.c.state);
  for (int rep = blockIdx.y; rep < p.c.B; rep += gridDim.y) plain_site<N, ST>(p.c, p.sub, p.alpha, rep, x, y, z, key);
}

// Packed storage: a warp owns one (word, class site); lane j is replica 32 w + j. Each lane runs the int8 update
// of its replica (same Philox counter), and the new word is assembled with a ballot.
// Grid (ceil(rows * bx / 8), words), 8 warps per block.
__global__ void __launch_bounds__(256) packed_class_kernel(const __grid_constant__ ClassParams p) {
  const Common& c = p.c;
  const Geometry& g = c.g;
  const int lane = threadIdx.x & 31;
  const uint32_t per_word = (uint32_t)c.rows * (uint32_t)c.bx;
  const uint32_t t = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (t >= per_word) return;
  int x, y, z;
  if (!class_site(c, p.colour, p.alpha, t, x, y, z)) return;
  const int own = p.alpha * g.plane + (z * g.L2 + y) * g.L1 + x;
  if (g.has_mask && c.mask[own] == 0) return;
  const int32_t key = sweep_key(c.state);
  const uint32_t* src = (const uint32_t*)c.src;
  uint32_t* dst = (uint32_t*)c.dst;
  for (int w = blockIdx.y; w < c.W; w += gridDim.y) {
    const size_t wb = (size_t)w * g.nsite;
    const int s = (src[wb + own] >> lane) & 1u ? 1 : -1;
    int k = s > 0 ? 1 : 0;
    int bi = 0;
#pragma unroll
    for (int gi = 0; gi < SCK_MAX_GROUPS; ++gi) {
      if (gi < p.sub.n_groups) {
        int G = 0;
        for (; bi < p.sub.group_end[gi]; ++bi) {
          const BondDev bd = p.sub.bonds[bi];
          const int q = neighbour_index(g, bd, x, y, z);
          int tv = 0;
          if (q >= 0 && (!g.has_mask || c.mask[q] != 0)) tv = (src[wb + q] >> lane) & 1u ? 1 : -1;
          G += tv;
          if (bd.extra >= 0) k += (tv + 1) * p.sub.extra_stride[bd.extra];
        }
        k += (G + p.sub.group_z[gi]) * p.sub.key_stride[gi];
      }
    }
    const int rep = w * 32 + lane;
    const float e = ((const float*)c.table)[(size_t)rep * c.lut_rep_stride + p.alpha * c.keys + k];
    const Philox4 r = philox4x32_10(counter32(rep, g.nsite, own), 0u, key_lo(key), key_hi(key));
    const float u0 = to_uniform(r.x0);
    const bool acc = g.acceptance == SCK_BARKER ? __fmul_rn(u0, __fadd_rn(1.0f, e)) < 1.0f : u0 < e;
    const bool bit = acc ? (s < 0) : (s > 0);
    const uint32_t word = __ballot_sync(0xFFFFFFFFu, bit);
    if (lane == 0) dst[wb + own] = word;
  }
}

// ---------------------------------------------------------------------------------------- resident sweeps
// A replica small enough for shared memory stays there for all n sweeps of one call: one block per replica
// loads its spins once, runs every class of every sweep with a block barrier between classes (a class reads
// only other classes, so the barrier is the whole dependency), and writes the spins back once. Sweep k of the
// call uses the key of state[1] + k, as n separate sweeps would.
struct ResidentParams {
  Common c;
  SubDev sub[SCK_MAX_BASIS];
  int n_classes;
  int classes[128][2];
  int n_sweeps;
};

template <int N, typename ST>
__global__ void __launch_bounds__(1024) resident_kernel(const __grid_constant__ ResidentParams p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  ST* S = reinterpret_cast<ST*>(smem_raw);
  const int rep = blockIdx.x;
  const int n = N * p.c.g.nsite;
  ST* home = (ST*)p.c.dst + (size_t)rep * n;
  for (int i = threadIdx.x; i < n; i += blockDim.x) S[i] = home[i];
  __syncthreads();
  const uint32_t per = (uint32_t)p.c.rows * (uint32_t)p.c.bx;
  for (int sw = 0; sw < p.n_sweeps; ++sw) {
    const int32_t key = sweep_key_at(p.c.state, sw);
    for (int ci = 0; ci < p.n_classes; ++ci) {
      const int colour = p.classes[ci][0], alpha = p.classes[ci][1];
      for (uint32_t t = threadIdx.x; t < per; t += blockDim.x) {
        int x, y, z;
        if (!class_site(p.c, colour, alpha, t, x, y, z)) continue;
        if constexpr (N == 1)
          ising_site<ST>(p.c, p.sub[alpha], alpha, rep, x, y, z, key, S, S);
        else
          vec_site<N>(p.c, p.sub[alpha], alpha, rep, x, y, z, key, (const float*)S, (float*)S);
      }
      __syncthreads();
    }
  }
  for (int i = threadIdx.x; i < n; i += blockDim.x) home[i] = S[i];
}

template <int N, typename ST>
static int launch_resident_t(const ResidentParams& p, int threads, size_t smem, cudaStream_t s) {
  cudaError_t e = cudaFuncSetAttribute(resident_kernel<N, ST>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return cuda_status(e, "resident kernel shared memory");
  resident_kernel<N, ST><<<p.c.B, threads, smem, s>>>(p);
  return cuda_status(cudaGetLastError(), "resident launch");
}

size_t resident_bytes(const sck_plan* plan) {
  return (size_t)plan->geom.n * plan->geom.nsite * (plan->mode == SCK_MODE_INT8 ? 1 : 4);
}

int launch_resident(const sck_plan* plan, const Common& c, int n_sweeps, cudaStream_t s) {
  ResidentParams p;
  p.c = c;
  for (int a = 0; a < SCK_MAX_BASIS; ++a) p.sub[a] = plan->sub[a];
  p.n_classes = plan->desc.n_classes;
  for (int i = 0; i < p.n_classes; ++i) {
    p.classes[i][0] = plan->desc.classes[i][0];
    p.classes[i][1] = plan->desc.classes[i][1];
  }
  p.n_sweeps = n_sweeps;
  const uint32_t per = (uint32_t)c.rows * (uint32_t)c.bx;
  int threads = (int)((per + 31) / 32 * 32);
  threads = threads < 128 ? 128 : (threads > 1024 ? 1024 : threads);
  const size_t smem = (resident_bytes(plan) + 15) / 16 * 16;
  if (plan->mode == SCK_MODE_INT8) return launch_resident_t<1, int8_t>(p, threads, smem, s);
  switch (c.g.n) {
    case 1: return launch_resident_t<1, float>(p, threads, smem, s);
    case 2: return launch_resident_t<2, float>(p, threads, smem, s);
    default: return launch_resident_t<3, float>(p, threads, smem, s);
  }
}

// ---------------------------------------------------------------------------------------- sequential chain
// One thread per replica walks the classes in sweep order and, inside a class, the sites in raster order
// (z, y, x): the definition of the chain that the parallel class launches must reproduce (sampler.py:281-293).
template <int N, typename ST>
__global__ void plain_sequential_kernel(const __grid_constant__ SeqParams p) {
  const int rep = blockIdx.x * blockDim.x + threadIdx.x;
  if (rep >= p.c.B) return;
  const int32_t key = sweep_key(p.c.state);
  const Geometry& g = p.c.g;
  for (int ci = 0; ci < p.n_classes; ++ci) {
    const int colour = p.classes[ci][0], alpha = p.classes[ci][1];
    for (int z = 0; z < g.L3; ++z)
      for (int y = 0; y < g.L2; ++y)
        for (int x = 0; x < g.L1; ++x)
          if (colour_of(p.c.col, alpha, x, y, z) == colour) plain_site<N, ST>(p.c, p.sub[alpha], alpha, rep, x, y, z, key);
  }
}

// Packed sequential chain: one warp per word, same site order.
__global__ void packed_sequential_kernel(const __grid_constant__ SeqParams p) {
  const Common& c = p.c;
  const Geometry& g = c.g;
  const int w = blockIdx.x;
  const int lane = threadIdx.x;
  if (w >= c.W) return;
  const int32_t key = sweep_key(c.state);
  uint32_t* sp = (uint32_t*)c.dst;
  const size_t wb = (size_t)w * g.nsite;
  for (int ci = 0; ci < p.n_classes; ++ci) {
    const int colour = p.classes[ci][0], alpha = p.classes[ci][1];
    const SubDev& sub = p.sub[alpha];
    for (int z = 0; z < g.L3; ++z)
      for (int y = 0; y < g.L2; ++y)
        for (int x = 0; x < g.L1; ++x) {
          if (colour_of(c.col, alpha, x, y, z) != colour) continue;
          const int own = alpha * g.plane + (z * g.L2 + y) * g.L1 + x;
          if (g.has_mask && c.mask[own] == 0) continue;
          const int s = (sp[wb + own] >> lane) & 1u ? 1 : -1;
          int k = s > 0 ? 1 : 0;
          int bi = 0;
          for (int gi = 0; gi < sub.n_groups; ++gi) {
            int G = 0;
            for (; bi < sub.group_end[gi]; ++bi) {
              const BondDev bd = sub.bonds[bi];
              const int q = neighbour_index(g, bd, x, y, z);
              int t = 0;
              if (q >= 0 && (!g.has_mask || c.mask[q] != 0)) t = (sp[wb + q] >> lane) & 1u ? 1 : -1;
              G += t;
              if (bd.extra >= 0) k += (t + 1) * sub.extra_stride[bd.extra];
            }
            k += (G + sub.group_z[gi]) * sub.key_stride[gi];
          }
          const int rep = w * 32 + lane;
          const float e = ((const float*)c.table)[(size_t)rep * c.lut_rep_stride + alpha * c.keys + k];
          const Philox4 r = philox4x32_10(counter32(rep, g.nsite, own), 0u, key_lo(key), key_hi(key));
          const float u0 = to_uniform(r.x0);
          const bool acc = g.acceptance == SCK_BARKER ? __fmul_rn(u0, __fadd_rn(1.0f, e)) < 1.0f : u0 < e;
          const uint32_t word = __ballot_sync(0xFFFFFFFFu, acc ? (s < 0) : (s > 0));
          if (lane == 0) sp[wb + own] = word;
          __syncwarp();
        }
  }
}

// ---------------------------------------------------------------------------------------------- conversions
// Grid (ceil(nsite / 256), words).
__global__ void pack_kernel(const int8_t* __restrict__ spins, int32_t* __restrict__ words, int B, int W, int nsite) {
  const int site = blockIdx.x * blockDim.x + threadIdx.x;
  if (site >= nsite) return;
  for (int w = blockIdx.y; w < W; w += gridDim.y) {
    uint32_t word = 0;
    for (int j = 0; j < 32; ++j) {
      const int rep = w * 32 + j;
      if (rep < B && spins[(size_t)rep * nsite + site] > 0) word |= 1u << j;
    }
    words[(size_t)w * nsite + site] = (int32_t)word;
  }
}

// Grid (ceil(nsite / 256), replicas).
__global__ void unpack_kernel(const int32_t* __restrict__ words, const int8_t* __restrict__ mask,
                              int8_t* __restrict__ spins, int B, int nsite) {
  const int site = blockIdx.x * blockDim.x + threadIdx.x;
  if (site >= nsite) return;
  const bool present = mask == nullptr || mask[site] != 0;
  for (int rep = blockIdx.y; rep < B; rep += gridDim.y) {
    const uint32_t word = (uint32_t)words[(size_t)(rep >> 5) * nsite + site];
    const int8_t v = (word >> (rep & 31)) & 1u ? 1 : -1;
    spins[(size_t)rep * nsite + site] = present ? v : 0;
  }
}

__global__ void advance_kernel(int64_t* state, int n) { state[1] += n; }

// -------------------------------------------------------------------------------------------------- launch
static dim3 grid2(uint32_t per_unit, int per_block, int units) {
  return dim3((per_unit + per_block - 1) / per_block, (unsigned)(units < 65535 ? units : 65535));
}

void set_rows(Common& c, int P, int bx) {
  c.P = P;
  c.bx = bx;
  c.fd_bx = make_fastdiv((uint32_t)bx);
}

int launch_class(const sck_plan* plan, const Common& c, int colour, int alpha, cudaStream_t s) {
  ClassParams p;
  p.c = c;
  p.sub = plan->sub[alpha];
  p.colour = colour;
  p.alpha = alpha;
  if (colour < 0) set_rows(p.c, 1, c.g.L1);
  const uint32_t per = (uint32_t)p.c.rows * (uint32_t)p.c.bx;
  if (plan->mode == SCK_MODE_PACKED) {
    packed_class_kernel<<<grid2(per, 8, c.W), 256, 0, s>>>(p);
  } else {
    const dim3 grid = grid2(per, 256, c.B);
    switch (c.g.n) {
      case 1:
        if (plan->mode == SCK_MODE_INT8)
          plain_class_kernel<1, int8_t><<<grid, 256, 0, s>>>(p);
        else
          plain_class_kernel<1, float><<<grid, 256, 0, s>>>(p);
        break;
      case 2:
        plain_class_kernel<2, float><<<grid, 256, 0, s>>>(p);
        break;
      default:
        plain_class_kernel<3, float><<<grid, 256, 0, s>>>(p);
        break;
    }
  }
  return cuda_status(cudaGetLastError(), "class launch");
}

int launch_sequential(const sck_plan* plan, const Common& c, cudaStream_t s) {
  SeqParams p;
  p.c = c;
  for (int a = 0; a < SCK_MAX_BASIS; ++a) p.sub[a] = plan->sub[a];
  p.n_classes = plan->desc.n_classes;
  for (int i = 0; i < p.n_classes; ++i) {
    p.classes[i][0] = plan->desc.classes[i][0];
    p.classes[i][1] = plan->desc.classes[i][1];
  }
  if (plan->mode == SCK_MODE_PACKED) {
    packed_sequential_kernel<<<c.W, 32, 0, s>>>(p);
  } else {
    const int grid = (c.B + 63) / 64;
    switch (c.g.n) {
      case 1:
        if (plan->mode == SCK_MODE_INT8)
          plain_sequential_kernel<1, int8_t><<<grid, 64, 0, s>>>(p);
        else
          plain_sequential_kernel<1, float><<<grid, 64, 0, s>>>(p);
        break;
      case 2:
        plain_sequential_kernel<2, float><<<grid, 64, 0, s>>>(p);
        break;
      default:
        plain_sequential_kernel<3, float><<<grid, 64, 0, s>>>(p);
        break;
    }
  }
  return cuda_status(cudaGetLastError(), "sequential launch");
}

int launch_pack(const sck_plan* plan, const int8_t* spins, int32_t* words, cudaStream_t s) {
  pack_kernel<<<grid2(plan->geom.nsite, 256, plan->W), 256, 0, s>>>(spins, words, plan->batch, plan->W,
                                                                    plan->geom.nsite);
  return cuda_status(cudaGetLastError(), "pack");
}

int launch_unpack(const sck_plan* plan, const int32_t* words, const int8_t* mask, int8_t* spins, cudaStream_t s) {
  unpack_kernel<<<grid2(plan->geom.nsite, 256, plan->batch), 256, 0, s>>>(words, mask, spins, plan->batch,
                                                                         plan->geom.nsite);
  return cuda_status(cudaGetLastError(), "unpack");
}

int launch_advance(int64_t* state, int n, cudaStream_t s) {
  advance_kernel<<<1, 1, 0, s>>>(state, n);
  return cuda_status(cudaGetLastError(), "advance");
}

}  // namespace sck
