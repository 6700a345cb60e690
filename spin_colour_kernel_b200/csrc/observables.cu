// FP64 observables (Spin_Colour_Kernel/sampler.py:296-345): energy per replica and per-sublattice
// magnetization, read directly from int8, float32 or packed-word storage.
//
// Grid (blocks_per_rep, B). A thread walks sites of one replica; per site it forms the bond field
// v_i = sum_b (J_b I + E_b) s_j in FP64, the site energy -1/2 s.v - h.s + k1 ((sx sy)^2 + (sx sz)^2 + (sy sz)^2)
// + k2 (sx sy sz)^2 and its contribution to M[alpha][k]. Warp shuffles, then shared memory, reduce a block to one
// partial per value; a second kernel sums the partials of a replica in block order, so results do not depend
// on scheduling.
#include <string>

#include "internal.h"
#include "spec.cuh"

namespace sck {

template <int N, int STORE>
__device__ __forceinline__ void load_spin(const ObsParams& p, int rep, int site, double (&s)[N]) {
  const Geometry& g = p.g;
  if constexpr (STORE == 2) {
    const uint32_t w = ((const uint32_t*)p.spins)[(size_t)(rep >> 5) * g.nsite + site];
    const bool present = p.mask == nullptr || p.mask[site] != 0;
    s[0] = present ? (((w >> (rep & 31)) & 1u) ? 1.0 : -1.0) : 0.0;
  } else if constexpr (STORE == 0) {
    s[0] = (double)((const int8_t*)p.spins)[(size_t)rep * g.nsite + site];
  } else {
#pragma unroll
    for (int k = 0; k < N; ++k) s[k] = (double)((const float*)p.spins)[((size_t)rep * N + k) * g.nsite + site];
  }
}

template <int N, int STORE>
__global__ void __launch_bounds__(256) observables_kernel(const __grid_constant__ ObsParams p) {
  const Geometry& g = p.g;
  const int rep = blockIdx.y;
  constexpr int NV = 1 + SCK_MAX_BASIS * N;
  double acc[NV];
#pragma unroll
  for (int i = 0; i < NV; ++i) acc[i] = 0.0;
  for (int site = blockIdx.x * blockDim.x + threadIdx.x; site < g.nsite; site += p.blocks_per_rep * blockDim.x) {
    if (p.mask != nullptr && p.mask[site] == 0) continue;
    const int alpha = (int)fdiv((uint32_t)site, p.fd_plane);
    const int rem = site - alpha * g.plane;
    const int row = (int)fdiv((uint32_t)rem, p.fd_L1);
    const int x = rem - row * g.L1;
    const int z = (int)fdiv((uint32_t)row, p.fd_L2);
    const int y = row - z * g.L2;
    double s[N];
    load_spin<N, STORE>(p, rep, site, s);
    double v[N];
#pragma unroll
    for (int k = 0; k < N; ++k) v[k] = 0.0;
    const SubDev& sub = p.sub[alpha];
    const SubObs& ob = p.obs[alpha];
    for (int bi = 0; bi < sub.n_bonds; ++bi) {
      const BondDev bd = sub.bonds[bi];
      const int q = neighbour_index(g, bd, x, y, z);
      if (q < 0) continue;
      double t[N];
      load_spin<N, STORE>(p, rep, q, t);
      const double J = ob.J[bi];
#pragma unroll
      for (int k = 0; k < N; ++k) v[k] += J * t[k];
      if (bd.extra >= 0) {
#pragma unroll
        for (int k = 0; k < N; ++k)
#pragma unroll
          for (int l = 0; l < N; ++l) v[k] += ob.E[bd.extra][3 * k + l] * t[l];
      }
    }
    double e = 0.0;
#pragma unroll
    for (int k = 0; k < N; ++k) e += -0.5 * s[k] * v[k] - p.h64[k] * s[k];
    if constexpr (N == 3) {
      if (g.has_cubic) {
        const double k1 = (double)p.k1[site];
        const double xy = s[0] * s[1], xz = s[0] * s[2], yz = s[1] * s[2], xyz = s[0] * s[1] * s[2];
        e += k1 * (xy * xy + xz * xz + yz * yz) + p.k2 * xyz * xyz;
      }
    }
    acc[0] += e;
#pragma unroll
    for (int a = 0; a < SCK_MAX_BASIS; ++a)
      if (a == alpha) {
#pragma unroll
        for (int k = 0; k < N; ++k) acc[1 + a * N + k] += s[k];
      }
  }
  __shared__ double red[NV][8];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int i = 0; i < NV; ++i) {
    double x = acc[i];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) x += __shfl_down_sync(0xFFFFFFFFu, x, off);
    if (lane == 0) red[i][warp] = x;
  }
  __syncthreads();
  if (threadIdx.x < NV) {
    double x = 0.0;
    for (int wi = 0; wi < (int)(blockDim.x >> 5); ++wi) x += red[threadIdx.x][wi];
    p.partial[((size_t)rep * p.blocks_per_rep + blockIdx.x) * OBS_VALUES + threadIdx.x] = x;
  }
}

// Systems with a compile-time bond table (lattices.h): every neighbour offset is a constant and each bond is
// visited once, from the end for which it points "forward" (to a higher sublattice, or within a sublattice to a
// positive offset in z, then y, then x); its reverse sits in the partner's table with the same coupling, so
// E = -sum_bonds J s_i . s_j - h . sum s + anisotropy equals -1/2 sum_i s_i . v_i of the generic kernel up to
// FP64 rounding, at half the neighbour reads. Still FP64 throughout.
__device__ __forceinline__ bool step_axis(int& v, int d, int L, int per) {
  v += d;
  if (v < 0) {
    if (!per) return false;
    v += L;
  } else if (v >= L) {
    if (!per) return false;
    v -= L;
  }
  return true;
}

template <class Lat, int N, int STORE>
__global__ void __launch_bounds__(256) observables_spec_kernel(const __grid_constant__ ObsParams p) {
  static_assert(bonds_paired<Lat>(), "every bond needs its reverse in the partner's table");
  const Geometry& g = p.g;
  const int rep = blockIdx.y;
  constexpr int NV = 1 + SCK_MAX_BASIS * N;
  double acc[NV];
#pragma unroll
  for (int i = 0; i < NV; ++i) acc[i] = 0.0;
  // four sites per iteration: their loads and FP64 chains overlap
#pragma unroll 4
  for (int site = blockIdx.x * blockDim.x + threadIdx.x; site < g.nsite; site += p.blocks_per_rep * blockDim.x) {
    if (p.mask != nullptr && p.mask[site] == 0) continue;
    const int alpha = (int)fdiv((uint32_t)site, p.fd_plane);
    const int rem = site - alpha * g.plane;
    const int row = (int)fdiv((uint32_t)rem, p.fd_L1);
    const int x = rem - row * g.L1;
    const int z = (int)fdiv((uint32_t)row, p.fd_L2);
    const int y = row - z * g.L2;
    double s[N];
    load_spin<N, STORE>(p, rep, site, s);
    double e = 0.0;
    static_for<0, Lat::b>([&](auto ac) {
      constexpr int a = decltype(ac)::value;
      if (a != alpha) return;
      const SubObs& ob = p.obs[a];
      static_for<0, Lat::n_bonds(a)>([&](auto ic) {
        constexpr int i = decltype(ic)::value;
        if constexpr (forward_bond<Lat, a>(i)) {
          constexpr BondC bd = Lat::bond(a, i);
          int x2 = x, y2 = y, z2 = z;
          if (!step_axis(x2, bd.dx, g.L1, g.per[0]) || !step_axis(y2, bd.dy, g.L2, g.per[1])) return;
          if (Lat::dim == 3 && !step_axis(z2, bd.dz, g.L3, g.per[2])) return;
          const int q = bd.a2 * g.plane + (z2 * g.L2 + y2) * g.L1 + x2;
          double t[N];
          load_spin<N, STORE>(p, rep, q, t);
          double dot = 0.0;
#pragma unroll
          for (int k = 0; k < N; ++k) dot += s[k] * t[k];
          e -= ob.J[i] * dot;
        }
      });
    });
#pragma unroll
    for (int k = 0; k < N; ++k) e -= p.h64[k] * s[k];
    if constexpr (N == 3) {
      if (g.has_cubic) {
        const double k1 = (double)p.k1[site];
        const double xy = s[0] * s[1], xz = s[0] * s[2], yz = s[1] * s[2], xyz = s[0] * s[1] * s[2];
        e += k1 * (xy * xy + xz * xz + yz * yz) + p.k2 * xyz * xyz;
      }
    }
    acc[0] += e;
#pragma unroll
    for (int a = 0; a < SCK_MAX_BASIS; ++a)
      if (a == alpha) {
#pragma unroll
        for (int k = 0; k < N; ++k) acc[1 + a * N + k] += s[k];
      }
  }
  __shared__ double red[NV][8];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int i = 0; i < NV; ++i) {
    double v = acc[i];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xFFFFFFFFu, v, off);
    if (lane == 0) red[i][warp] = v;
  }
  __syncthreads();
  if (threadIdx.x < NV) {
    double v = 0.0;
    for (int wi = 0; wi < (int)(blockDim.x >> 5); ++wi) v += red[threadIdx.x][wi];
    p.partial[((size_t)rep * p.blocks_per_rep + blockIdx.x) * OBS_VALUES + threadIdx.x] = v;
  }
}

template <class Lat>
static void launch_obs_spec(const ObsParams& p, dim3 grid, cudaStream_t s) {
  if (p.storage == 0) observables_spec_kernel<Lat, 1, 0><<<grid, 256, 0, s>>>(p);
  else if (p.g.n == 1) observables_spec_kernel<Lat, 1, 1><<<grid, 256, 0, s>>>(p);
  else if (p.g.n == 2) observables_spec_kernel<Lat, 2, 1><<<grid, 256, 0, s>>>(p);
  else observables_spec_kernel<Lat, 3, 1><<<grid, 256, 0, s>>>(p);
}

// Tiled variant for float32 storage on periodic boxes with a lattice table and a row length of 16, 32, 64 or
// 128. The spins of one replica are read in bands of OBS_TY rows: a block of threads marches along z keeping
// three planes of its band (plus one halo row on each side and one halo site at each end of a row) in shared
// memory, converted to FP64 once when they arrive. Every forward bond then reads FP64 neighbours from shared
// memory at compile-time offsets from one address per plane, so each spin component is converted
// ~(OBS_TY + 2) / OBS_TY times instead of once per bond that reaches it, and no per-bond index arithmetic is
// left: the conversions and the index arithmetic, not the FP64 arithmetic or the HBM reads, bound the per-site
// kernel above. Same bond-once energy and the same fixed-order partial sums.
constexpr int OBS_TY = 4;                     // rows per band
constexpr int OBS_THREADS = 256;              // threads per block
constexpr int OBS_PAD = 2;                    // doubles before x = 0 in a shared row: x = -1 sits at OBS_PAD - 1
constexpr size_t OBS_TILE_SMEM_MAX = 110 * 1024;

template <int L1T>
struct ObsRow {
  static constexpr int RS = L1T + 2 * OBS_PAD;   // doubles per shared row
  static constexpr int R2 = OBS_TY + 2;          // band rows plus halo rows
};

static size_t obs_tile_smem(const sck_plan* plan) {
  const Geometry& g = plan->geom;
  return (size_t)3 * g.b * g.n * (OBS_TY + 2) * (g.L1 + 2 * OBS_PAD) * sizeof(double);
}

// geometry that the tiled kernel serves (its lattice table may still be switched off by tuning)
static bool obs_tile_geometry(const sck_plan* plan) {
  const Geometry& g = plan->geom;
  if (plan->mode != SCK_MODE_F32 || find_spec(plan) == 0) return false;
  if (g.L1 != 16 && g.L1 != 32 && g.L1 != 64 && g.L1 != 128) return false;
  if (!g.per[0] || !g.per[1] || g.L2 % OBS_TY != 0 || g.L2 < 3) return false;
  if (g.dim == 3 && (!g.per[2] || g.L3 < 3)) return false;
  return obs_tile_smem(plan) <= OBS_TILE_SMEM_MAX;
}

// FP64 shared-memory load at a compile-time byte offset from a register address
template <int OFF>
__device__ __forceinline__ double ldsd(uint32_t addr) {
  double v;
  asm volatile("ld.shared.f64 %0, [%1+%2];\n" : "=d"(v) : "r"(addr), "n"(OFF));
  return v;
}

template <class Lat, int N, int L1T>
__global__ void __launch_bounds__(OBS_THREADS) observables_tile_kernel(const __grid_constant__ ObsParams p) {
  extern __shared__ __align__(16) double ring[];   // [3 planes][b][N][R2 rows][RS]
  using RW = ObsRow<L1T>;
  constexpr int RS = RW::RS, R2 = RW::R2;
  constexpr int COMP = R2 * RS;                    // doubles of one component of one sublattice
  constexpr int SLOT = Lat::b * N * COMP;
  constexpr int Q = L1T / 4;                       // float4 loads per row
  constexpr int ITEMS = Lat::b * N * R2 * Q;       // float4 loads per plane
  constexpr int LOADS = (ITEMS + OBS_THREADS - 1) / OBS_THREADS;       // per thread
  const Geometry& g = p.g;
  const int rep = blockIdx.y, y0 = blockIdx.x * OBS_TY;
  const float* src = (const float*)p.spins + (size_t)rep * N * g.nsite;
  // The next plane's loads are issued into registers before the current plane is computed and written to
  // shared memory (as FP64) after it, so HBM latency overlaps the FP64 work.
  float4 pf[LOADS];
  auto fetch = [&](int zu) {   // unwrapped plane index -1 .. L3
    const int zz = zu < 0 ? zu + g.L3 : (zu >= g.L3 ? zu - g.L3 : zu);
#pragma unroll
    for (int j = 0; j < LOADS; ++j) {
      const int i = threadIdx.x + OBS_THREADS * j;
      if (ITEMS % OBS_THREADS == 0 || i < ITEMS) {
        const int row = i / Q, q = i % Q;
        const int r = row % R2, ak = row / R2, k = ak % N, a = ak / N;
        int y = y0 - 1 + r;
        y = y < 0 ? y + g.L2 : (y >= g.L2 ? y - g.L2 : y);
        pf[j] = *(const float4*)(src + (size_t)k * g.nsite + (size_t)a * g.plane +
                                 ((size_t)zz * g.L2 + y) * L1T + 4 * q);
      }
    }
  };
  auto deposit = [&](int zu) {
    double* dst = ring + ((zu + 3) % 3) * SLOT;
#pragma unroll
    for (int j = 0; j < LOADS; ++j) {
      const int i = threadIdx.x + OBS_THREADS * j;
      if (ITEMS % OBS_THREADS == 0 || i < ITEMS) {
        const int row = i / Q, q = i % Q;
        double* d = dst + row * RS + OBS_PAD + 4 * q;
        const float4 v = pf[j];
        d[0] = v.x;
        d[1] = v.y;
        d[2] = v.z;
        d[3] = v.w;
        if (q == 0) d[L1T] = v.x;            // x = L1 is x = 0
        if (q == Q - 1) d[-L1T + 3] = v.w;   // x = -1 is x = L1 - 1
      }
    }
  };
  fetch(-1);
  deposit(-1);
  fetch(0);
  deposit(0);
  fetch(1);
  deposit(1);
  __syncthreads();
  constexpr int NV = 1 + SCK_MAX_BASIS * N;
  double acc[NV];
#pragma unroll
  for (int i = 0; i < NV; ++i) acc[i] = 0.0;
  const uint32_t sbase = (uint32_t)__cvta_generic_to_shared(ring);
  constexpr uint32_t SLOT_BYTES = 8u * SLOT;
  uint32_t pl[3] = {sbase + 2 * SLOT_BYTES, sbase, sbase + SLOT_BYTES};   // planes zu - 1, zu, zu + 1 at zu = 0
  constexpr int XY = OBS_TY * L1T;                 // (x, row) positions of a band; each covers every sublattice
  const bool masked = p.mask != nullptr;
  for (int zu = 0; zu < g.L3; ++zu) {
    const bool more = zu + 1 < g.L3;
    if (more) fetch(zu + 2);
    for (int i = threadIdx.x; i < XY; i += OBS_THREADS) {
      const int x = i % L1T, ty = i / L1T;
      const int rsite = (zu * g.L2 + y0 + ty) * L1T + x;
      const uint32_t so = 8u * (uint32_t)((ty + 1) * RS + OBS_PAD + x);
      static_for<0, Lat::b>([&](auto ac) {
        constexpr int a = decltype(ac)::value;
        const int site = a * g.plane + rsite;
        if (masked && p.mask[site] == 0) return;
        double s[N];
        static_for<0, N>([&](auto kc) {
          constexpr int k = decltype(kc)::value;
          s[k] = ldsd<8 * (a * N + k) * COMP>(pl[1] + so);
        });
        const SubObs& ob = p.obs[a];
        double e = 0.0;
        static_for<0, Lat::n_bonds(a)>([&](auto ic) {
          constexpr int bi = decltype(ic)::value;
          if constexpr (forward_bond<Lat, a>(bi)) {
            constexpr BondC bd = Lat::bond(a, bi);
            constexpr int off = 8 * (bd.a2 * N * COMP + bd.dy * RS + bd.dx);
            const uint32_t q = pl[bd.dz + 1] + so;
            double dot = s[0] * ldsd<off>(q);
            static_for<1, N>([&](auto kc) {
              constexpr int k = decltype(kc)::value;
              dot = fma(s[k], ldsd<off + 8 * k * COMP>(q), dot);
            });
            e = fma(-ob.J[bi], dot, e);
          }
        });
#pragma unroll
        for (int k = 0; k < N; ++k) e = fma(-p.h64[k], s[k], e);
        if constexpr (N == 3) {
          if (g.has_cubic) {
            const double k1 = (double)p.k1[site];
            const double xy = s[0] * s[1], xz = s[0] * s[2], yz = s[1] * s[2], xyz = xy * s[2];
            e += k1 * (xy * xy + xz * xz + yz * yz) + p.k2 * xyz * xyz;
          }
        }
        acc[0] += e;
#pragma unroll
        for (int k = 0; k < N; ++k) acc[1 + a * N + k] += s[k];
      });
    }
    __syncthreads();                              // every thread is done with plane zu - 1
    const uint32_t rot = pl[0];                   // the ring turns
    pl[0] = pl[1];
    pl[1] = pl[2];
    pl[2] = rot;
    if (more) {
      deposit(zu + 2);                            // into plane zu - 1's slot
      __syncthreads();
    }
  }
  __shared__ double red[NV][OBS_THREADS / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int i = 0; i < NV; ++i) {
    double v = acc[i];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xFFFFFFFFu, v, off);
    if (lane == 0) red[i][warp] = v;
  }
  __syncthreads();
  if (threadIdx.x < NV) {
    double v = 0.0;
    for (int wi = 0; wi < (int)(blockDim.x >> 5); ++wi) v += red[threadIdx.x][wi];
    p.partial[((size_t)rep * p.blocks_per_rep + blockIdx.x) * OBS_VALUES + threadIdx.x] = v;
  }
}

template <class Lat, int N, int L1T>
static int launch_obs_tile_t(const sck_plan* plan, const ObsParams& p, cudaStream_t s) {
  const size_t smem = obs_tile_smem(plan);
  const dim3 grid(plan->geom.L2 / OBS_TY, p.B);
  const int rc = cuda_status(cudaFuncSetAttribute(observables_tile_kernel<Lat, N, L1T>,
                                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                             "obs tile");
  if (rc == SCK_OK) observables_tile_kernel<Lat, N, L1T><<<grid, OBS_THREADS, smem, s>>>(p);
  return rc;
}

template <class Lat, int N>
static int launch_obs_tile_n(const sck_plan* plan, const ObsParams& p, cudaStream_t s) {
  switch (plan->geom.L1) {
    case 16: return launch_obs_tile_t<Lat, N, 16>(plan, p, s);
    case 32: return launch_obs_tile_t<Lat, N, 32>(plan, p, s);
    case 64: return launch_obs_tile_t<Lat, N, 64>(plan, p, s);
    default: return launch_obs_tile_t<Lat, N, 128>(plan, p, s);
  }
}

template <class Lat>
static int launch_obs_tile(const sck_plan* plan, const ObsParams& p, cudaStream_t s) {
  switch (plan->geom.n) {
    case 1: return launch_obs_tile_n<Lat, 1>(plan, p, s);
    case 2: return launch_obs_tile_n<Lat, 2>(plan, p, s);
    default: return launch_obs_tile_n<Lat, 3>(plan, p, s);
  }
}

// Sum the partials of every replica in block order; E[r] and M[r][alpha][k] (B x b x n).
__global__ void observables_finish(const double* __restrict__ partial, int B, int blocks_per_rep, int b, int n,
                                   double* __restrict__ E, double* __restrict__ M) {
  const int rep = blockIdx.x * blockDim.y + threadIdx.y;
  const int v = threadIdx.x;
  if (rep >= B || v >= 1 + b * n) return;
  double x = 0.0;
  for (int i = 0; i < blocks_per_rep; ++i) x += partial[((size_t)rep * blocks_per_rep + i) * OBS_VALUES + v];
  if (v == 0) {
    if (E != nullptr) E[rep] = x;
  } else if (M != nullptr) {
    M[(size_t)rep * b * n + (v - 1)] = x;
  }
}

// Enough blocks in flight to cover the GPU, never more than the sites of one replica need.
static int obs_blocks_generic(const sck_plan* plan, int batch) {
  const int per_rep = (plan->geom.nsite + 255) / 256;
  const int want = (148 * 8 + batch - 1) / batch;
  return want < per_rep ? (want < 1 ? 1 : want) : per_rep;
}

// Whether an observables call of this storage takes the tiled path (its lattice table on, float32 storage, a
// geometry the tiled kernel serves).
static bool obs_tiled(const sck_plan* plan, int storage) {
  return plan->spec != 0 && storage == SCK_MODE_F32 && obs_tile_geometry(plan);
}

// Blocks per replica, hence partial-sum slots per replica, of one observables call: the one count that both the
// launch and the size checks of its callers use, so the slots written and the slots summed always agree.
static bool obs_words_ok(const sck_plan* plan, int storage);

// Blocks per word of 32 replicas of the word-parallel kernel: about 8 blocks per SM over all words.
static int obs_blocks_words(const sck_plan* plan, int batch) {
  const int per_rep = (plan->geom.nsite + 255) / 256;
  const int words = (batch + 31) / 32;
  const int want = (148 * 8 + words - 1) / words;
  return want < per_rep ? (want < 1 ? 1 : want) : per_rep;
}

int obs_launch_blocks(const sck_plan* plan, int storage, int batch) {
  if (storage == SCK_MODE_QUAD) return quad_obs_blocks(plan);
  if (obs_words_ok(plan, storage)) return obs_blocks_words(plan, batch);
  return obs_tiled(plan, storage) ? plan->geom.L2 / OBS_TY : obs_blocks_generic(plan, batch);
}

// Partial sums per replica a caller's workspace must hold: the largest count any storage and tuning of this plan
// can launch, so that a workspace stays valid whatever the plan's tuning selects later.
int obs_blocks_per_rep(const sck_plan* plan, int batch) {
  int most = obs_blocks_generic(plan, batch);
  const int tile = obs_tile_geometry(plan) ? plan->geom.L2 / OBS_TY : 0;
  if (tile > most) most = tile;
  if (plan->mode == SCK_MODE_QUAD && quad_obs_blocks(plan) > most) most = quad_obs_blocks(plan);
  if (obs_words_ok(plan, SCK_MODE_PACKED) && obs_blocks_words(plan, batch) > most) most = obs_blocks_words(plan, batch);
  return most;
}

// One observation of a measure step folded into FP64 accumulators, per replica r (one thread each): with
// d = E - E_ref and m = (sum over sublattices of M) / n_active,
//   acc[0][r] += d, acc[1][r] += d^2, acc[2][r] += |m|, acc[3][r] += |m|^2, accv[r][k] += m_k,
// the quantities the reference's ladder runner accumulates per observation (simulate.py:338-353), rounded
// operation by operation in the same order (no contraction into fused multiply-adds).
__global__ void observables_fold(const double* __restrict__ E, const double* __restrict__ M, int B, int b, int n,
                                 double n_active, const double* __restrict__ E_ref, double* __restrict__ acc,
                                 double* __restrict__ accv) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= B) return;
  const double d = __dsub_rn(E[r], E_ref[r]);
  double sq = 0.0;
  for (int k = 0; k < n; ++k) {
    double m = 0.0;
    for (int a = 0; a < b; ++a) m = __dadd_rn(m, M[((size_t)r * b + a) * n + k]);
    m = __ddiv_rn(m, n_active);
    sq = __dadd_rn(sq, __dmul_rn(m, m));
    accv[(size_t)r * n + k] = __dadd_rn(accv[(size_t)r * n + k], m);
  }
  const double am = __dsqrt_rn(sq);
  acc[r] = __dadd_rn(acc[r], d);
  acc[B + r] = __dadd_rn(acc[B + r], __dmul_rn(d, d));
  acc[2 * B + r] = __dadd_rn(acc[2 * B + r], am);
  acc[3 * B + r] = __dadd_rn(acc[3 * B + r], __dmul_rn(am, am));
}

int launch_observables_fold(const sck_plan* plan, int batch, const double* E, const double* M, double n_active,
                            const double* E_ref, double* acc, double* accv, cudaStream_t s) {
  observables_fold<<<(batch + 127) / 128, 128, 0, s>>>(E, M, batch, plan->geom.b, plan->geom.n, n_active, E_ref,
                                                       acc, accv);
  return cuda_status(cudaGetLastError(), "observables fold");
}

// Berg-Luscher topological charge of one z-layer of sublattice 0 (the nanodisk's middle layer,
// anneal.py:69-80): every plaquette (y, x)-(y+1, x+1) whose four corners are active is cut into the spherical
// triangles (s00, s10, s11) and (s00, s11, s01), each of solid angle
//   Omega(a, b, c) = 2 atan2(a . (b x c), 1 + a . b + b . c + c . a),
// and Q = sum Omega / 4 pi, in FP64 from the float32 spins. One block per replica, partial sums in a fixed order.
__device__ __forceinline__ double solid_angle(const double (&a)[3], const double (&b)[3], const double (&c)[3]) {
  const double x0 = __dsub_rn(__dmul_rn(b[1], c[2]), __dmul_rn(b[2], c[1]));
  const double x1 = __dsub_rn(__dmul_rn(b[2], c[0]), __dmul_rn(b[0], c[2]));
  const double x2 = __dsub_rn(__dmul_rn(b[0], c[1]), __dmul_rn(b[1], c[0]));
  const double num = __dadd_rn(__dadd_rn(__dmul_rn(a[0], x0), __dmul_rn(a[1], x1)), __dmul_rn(a[2], x2));
  auto dot = [](const double (&u)[3], const double (&v)[3]) {
    return __dadd_rn(__dadd_rn(__dmul_rn(u[0], v[0]), __dmul_rn(u[1], v[1])), __dmul_rn(u[2], v[2]));
  };
  const double den = __dadd_rn(__dadd_rn(__dadd_rn(1.0, dot(a, b)), dot(b, c)), dot(c, a));
  return 2.0 * atan2(num, den);
}

__global__ void __launch_bounds__(256) topological_charge_kernel(const float* __restrict__ spins,
                                                                 const int8_t* __restrict__ mask, Geometry g, int z,
                                                                 double* __restrict__ Q) {
  const int rep = blockIdx.x;
  const int nx = g.L1 - 1, ny = g.L2 - 1;
  const float* base = spins + (size_t)rep * 3 * g.nsite + (size_t)z * g.L2 * g.L1;   // sublattice 0, layer z
  const int8_t* mz = mask != nullptr ? mask + (size_t)z * g.L2 * g.L1 : nullptr;
  double acc = 0.0;
  for (int i = threadIdx.x; i < nx * ny; i += blockDim.x) {
    const int y = i / nx, x = i - y * nx;
    const int o00 = y * g.L1 + x, o10 = o00 + 1, o01 = o00 + g.L1, o11 = o01 + 1;
    if (mz != nullptr && !(mz[o00] && mz[o10] && mz[o01] && mz[o11])) continue;
    double s00[3], s10[3], s01[3], s11[3];
    for (int k = 0; k < 3; ++k) {
      const float* c = base + (size_t)k * g.nsite;
      s00[k] = c[o00];
      s10[k] = c[o10];
      s01[k] = c[o01];
      s11[k] = c[o11];
    }
    acc += solid_angle(s00, s10, s11) + solid_angle(s00, s11, s01);
  }
  __shared__ double part[256];
  part[threadIdx.x] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double sum = 0.0;
    for (int i = 0; i < (int)blockDim.x; ++i) sum += part[i];
    Q[rep] = sum / (4.0 * 3.14159265358979323846);
  }
}

int launch_topological_charge(const sck_plan* plan, const float* spins, const int8_t* mask, int batch, int z,
                              double* Q, cudaStream_t s) {
  topological_charge_kernel<<<batch, 256, 0, s>>>(spins, plan->geom.has_mask ? mask : nullptr, plan->geom, z, Q);
  return cuda_status(cudaGetLastError(), "topological charge");
}

// Packed words of a single-sublattice Ising system with isotropic bonds (at most 8): one thread per (word, site)
// updates 32 replicas at once. Per present bond b, x_b = s XOR s_j marks the anti-aligned replicas; a warp turns
// each per-thread lane mask into per-replica counts over its 32 sites (a 32 x 32 bit transpose across the warp,
// then a popcount: lane l ends with bit l of every thread's mask), so lane l accumulates, in integers (exact in any order), A_b = anti-aligned pairs of bond b, U = up spins, and
// the lane-independent P_b = present pairs and S = present sites. Then replica 32 w + l of the block:
//   E = sum_b -J_b (P_b - 2 A_b) / 2 - h (2 U - S),   M = 2 U - S,
// the same site energy -1/2 s v - h s as observables_kernel, written to the same partial slots.
constexpr int kWordObsBonds = 8;

// Number of threads of the warp whose mask has bit `lane` set, for every lane at once: the warp's 32 masks as a
// 32 x 32 bit matrix (row = thread, column = bit) transposed by exchanging off-diagonal blocks of 16, 8, 4, 2 and
// 1 across lane ^ s, then the popcount of the lane's column.
__device__ __forceinline__ unsigned warp_lane_counts(uint32_t x, int lane) {
  const uint32_t lo[5] = {0x0000FFFFu, 0x00FF00FFu, 0x0F0F0F0Fu, 0x33333333u, 0x55555555u};
#pragma unroll
  for (int i = 0, sh = 16; i < 5; ++i, sh >>= 1) {
    const uint32_t y = __shfl_xor_sync(0xFFFFFFFFu, x, sh);
    x = (lane & sh) ? ((x & ~lo[i]) | ((y & ~lo[i]) >> sh)) : ((x & lo[i]) | ((y & lo[i]) << sh));
  }
  return (unsigned)__popc(x);
}

__global__ void __launch_bounds__(256) observables_words_kernel(const __grid_constant__ ObsParams p) {
  const Geometry& g = p.g;
  const int w = blockIdx.y;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const SubDev& sub = p.sub[0];
  const int nb = sub.n_bonds;
  unsigned A[kWordObsBonds], P[kWordObsBonds], U = 0u, S = 0u;
#pragma unroll
  for (int b = 0; b < kWordObsBonds; ++b) A[b] = P[b] = 0u;
  const uint32_t* words = (const uint32_t*)p.spins + (size_t)w * g.nsite;
  const int stride = p.blocks_per_rep * blockDim.x;
  // every thread of a warp runs the same iterations (the ballots and shuffles need the whole warp)
  for (int base = blockIdx.x * blockDim.x + warp * 32; base < g.nsite; base += stride) {
    const int site = base + lane;
    bool present = site < g.nsite && (p.mask == nullptr || p.mask[site] != 0);
    uint32_t s0 = 0u;
    int x = 0, y = 0, z = 0;
    if (present) {
      const int row = (int)fdiv((uint32_t)site, p.fd_L1);
      x = site - row * g.L1;
      z = (int)fdiv((uint32_t)row, p.fd_L2);
      y = row - z * g.L2;
      s0 = words[site];
    }
    const unsigned sites_here = __popc(__ballot_sync(0xFFFFFFFFu, present));
    S += sites_here;
    U += warp_lane_counts(present ? s0 : 0u, lane);
#pragma unroll
    for (int b = 0; b < kWordObsBonds; ++b) {
      if (b >= nb) break;
      bool pb = false;
      uint32_t xb = 0u;
      if (present) {
        const int q = neighbour_index(g, sub.bonds[b], x, y, z);
        if (q >= 0 && (p.mask == nullptr || p.mask[q] != 0)) {
          pb = true;
          xb = s0 ^ words[q];
        }
      }
      P[b] += __popc(__ballot_sync(0xFFFFFFFFu, pb));
      A[b] += warp_lane_counts(xb, lane);
    }
  }
  // block sums per lane (integers), then FP64 per replica
  __shared__ unsigned red[8][2 * kWordObsBonds + 2][32];
#pragma unroll
  for (int b = 0; b < kWordObsBonds; ++b) {
    red[warp][b][lane] = A[b];
    red[warp][kWordObsBonds + b][lane] = P[b];
  }
  red[warp][2 * kWordObsBonds][lane] = U;
  red[warp][2 * kWordObsBonds + 1][lane] = S;
  __syncthreads();
  if (threadIdx.x < 32) {
    unsigned long long a[kWordObsBonds], pp[kWordObsBonds], u = 0, sn = 0;
#pragma unroll
    for (int b = 0; b < kWordObsBonds; ++b) a[b] = pp[b] = 0;
    for (int wi = 0; wi < (int)(blockDim.x >> 5); ++wi) {
#pragma unroll
      for (int b = 0; b < kWordObsBonds; ++b) {
        a[b] += red[wi][b][lane];
        pp[b] += red[wi][kWordObsBonds + b][lane];
      }
      u += red[wi][2 * kWordObsBonds][lane];
      sn += red[wi][2 * kWordObsBonds + 1][lane];
    }
    double e = 0.0;
#pragma unroll
    for (int b = 0; b < kWordObsBonds; ++b)
      if (b < nb) e += -0.5 * p.obs[0].J[b] * ((double)pp[b] - 2.0 * (double)a[b]);
    const double m = 2.0 * (double)u - (double)sn;
    e -= p.h64[0] * m;
    const int rep = 32 * w + lane;
    if (rep < p.B) {
      double* out = p.partial + ((size_t)rep * p.blocks_per_rep + blockIdx.x) * OBS_VALUES;
      out[0] = e;
      out[1] = m;
    }
  }
}

// The word kernel's conditions: packed words, one sublattice, n = 1, at most kWordObsBonds isotropic bonds.
static bool obs_words_ok(const sck_plan* plan, int storage) {
  if (storage != SCK_MODE_PACKED || plan->geom.b != 1 || plan->geom.n != 1) return false;
  const SubDev& sub = plan->sub[0];
  if (sub.n_bonds > kWordObsBonds) return false;
  for (int i = 0; i < sub.n_bonds; ++i)
    if (sub.bonds[i].extra >= 0) return false;
  return true;
}

int launch_observables(const sck_plan* plan, const void* spins, int storage, int batch, const int8_t* mask,
                       const float* k1, double* E, double* M, void* workspace, cudaStream_t s) {
  if (storage == SCK_MODE_QUAD) return launch_quad_observables(plan, spins, batch, k1, E, M, workspace, s);
  ObsParams p;
  p.g = plan->geom;
  p.B = batch;
  p.storage = storage == SCK_MODE_INT8 ? 0 : (storage == SCK_MODE_F32 ? 1 : 2);
  for (int a = 0; a < SCK_MAX_BASIS; ++a) {
    p.sub[a] = plan->sub[a];
    p.obs[a] = plan->obs[a];
  }
  for (int k = 0; k < 3; ++k) p.h64[k] = plan->desc.h64[k];
  p.k2 = plan->desc.k2_64;
  // float32 storage of a tiled-geometry system with its lattice table on: bands of OBS_TY rows
  const bool tile = obs_tiled(plan, storage);
  p.blocks_per_rep = obs_launch_blocks(plan, storage, batch);
  p.fd_plane = make_fastdiv((uint32_t)plan->geom.plane);
  p.fd_L1 = make_fastdiv((uint32_t)plan->geom.L1);
  p.fd_L2 = make_fastdiv((uint32_t)plan->geom.L2);
  if (batch > 65535) return cuda_status(cudaErrorInvalidConfiguration, "observables: batch above 65535");
  p.spins = spins;
  p.mask = plan->geom.has_mask ? mask : nullptr;
  p.k1 = k1;
  p.partial = (double*)workspace;
  dim3 grid(p.blocks_per_rep, p.B);
  const int n = plan->geom.n;
  // the lattice table fixes the bonds of int8 and float32 storage (packed storage reads the generic way)
  const bool spec = plan->spec != 0 && p.storage != 2;
  if (tile) {
    int rc = SCK_OK;
    switch (plan->spec) {
      case Lat_square_1::id: rc = launch_obs_tile<Lat_square_1>(plan, p, s); break;
      case Lat_triangular_1::id: rc = launch_obs_tile<Lat_triangular_1>(plan, p, s); break;
      case Lat_sc_1::id: rc = launch_obs_tile<Lat_sc_1>(plan, p, s); break;
      case Lat_bcc_1::id: rc = launch_obs_tile<Lat_bcc_1>(plan, p, s); break;
      case Lat_bcc_1_2::id: rc = launch_obs_tile<Lat_bcc_1_2>(plan, p, s); break;
      default: rc = launch_obs_tile<Lat_fcc_1>(plan, p, s); break;
    }
    if (rc != SCK_OK) return rc;
  } else if (spec) {
    switch (plan->spec) {
      case Lat_square_1::id: launch_obs_spec<Lat_square_1>(p, grid, s); break;
      case Lat_triangular_1::id: launch_obs_spec<Lat_triangular_1>(p, grid, s); break;
      case Lat_sc_1::id: launch_obs_spec<Lat_sc_1>(p, grid, s); break;
      case Lat_bcc_1::id: launch_obs_spec<Lat_bcc_1>(p, grid, s); break;
      case Lat_bcc_1_2::id: launch_obs_spec<Lat_bcc_1_2>(p, grid, s); break;
      default: launch_obs_spec<Lat_fcc_1>(p, grid, s); break;
    }
  } else if (p.storage == 2 && obs_words_ok(plan, storage)) {
    observables_words_kernel<<<dim3(p.blocks_per_rep, (p.B + 31) / 32), 256, 0, s>>>(p);
  } else if (p.storage == 2) observables_kernel<1, 2><<<grid, 256, 0, s>>>(p);
  else if (p.storage == 0) observables_kernel<1, 0><<<grid, 256, 0, s>>>(p);
  else if (n == 1) observables_kernel<1, 1><<<grid, 256, 0, s>>>(p);
  else if (n == 2) observables_kernel<2, 1><<<grid, 256, 0, s>>>(p);
  else observables_kernel<3, 1><<<grid, 256, 0, s>>>(p);
  int rc = cuda_status(cudaGetLastError(), "observables");
  if (rc != SCK_OK) return rc;
  return launch_observables_finish(p.partial, p.B, p.blocks_per_rep, plan->geom.b, n, E, M, s);
}

int launch_observables_finish(const double* partial, int B, int blocks_per_rep, int b, int n, double* E, double* M,
                              cudaStream_t s) {
  dim3 fb(OBS_VALUES, 8);
  observables_finish<<<(B + 7) / 8, fb, 0, s>>>(partial, B, blocks_per_rep, b, n, E, M);
  return cuda_status(cudaGetLastError(), "observables finish");
}

}  // namespace sck

// ------------------------------------------------------------------------------------ allocation-free entry
// Some callers cannot allocate device memory: a host that hands every device byte to its own pool or caching
// allocator (a cudaMalloc behind its back breaks its accounting or its budget), a latency-critical loop that
// cannot pay the device-wide synchronisation cudaMalloc / cudaFree may imply, or an FFI binding with no way to
// own a device buffer. For them the per-block partial sums of the observables live in this fixed array, which
// every GPU that loads the library keeps for the life of the process.
namespace sck {

constexpr size_t kScratchDoubles = (size_t)1 << 18;   // 2 MiB of FP64 partial sums
static __device__ __align__(256) double g_observables_scratch[kScratchDoubles];


// Device address of the scratch array in the current context. In host code the array's name is only a host-side
// handle, so the address must come from the runtime; it is looked up on every call (cheap, allocates nothing),
// so a context that was reset or replaced never receives a stale address. The first lookup on a device may load
// the library's module into the context, which is why the first call on a device belongs before any capture.
static int scratch_address(double** out) {
  void* p = nullptr;
  const int rc = cuda_status(cudaGetSymbolAddress(&p, g_observables_scratch), "no-alloc observables: scratch address");
  if (rc != SCK_OK) return rc;
  *out = (double*)p;
  return SCK_OK;
}

}  // namespace sck

extern "C" int sck_observables_noalloc(const sck_plan* plan, const sck_buffers* buf, const void* spins,
                                       int32_t storage, int32_t batch, double* E, double* M, void* stream) {
  using namespace sck;
  if (plan == nullptr || buf == nullptr || spins == nullptr) {
    set_error("null plan, buffers or spins");
    return SCK_ERR_INVALID;
  }
  const int rc0 = check_observables_request(plan, storage, batch);
  if (rc0 != SCK_OK) return rc0;
  if ((plan->geom.has_mask && buf->mask == nullptr) || (plan->geom.has_cubic && buf->k1 == nullptr)) {
    set_error("the system needs its mask / k1 buffers");
    return SCK_ERR_INVALID;
  }
  const size_t need = (size_t)batch * obs_launch_blocks(plan, storage, batch) * OBS_VALUES;
  if (need > kScratchDoubles) {
    set_error("no-alloc observables: " + std::to_string(need * sizeof(double)) + " bytes of partial sums exceed the " +
              std::to_string(kScratchDoubles * sizeof(double)) + "-byte scratch; use sck_observables with a workspace");
    return SCK_ERR_INVALID;
  }
  double* scratch = nullptr;
  const int rc = scratch_address(&scratch);
  if (rc != SCK_OK) return rc;
  return launch_observables(plan, spins, storage, batch, buf->mask, buf->k1, E, M, scratch, (cudaStream_t)stream);
}
