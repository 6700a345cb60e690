// Bitwise multi-spin-coded Ising (Spin_Colour_Kernel/bitwise.py): 32 replicas per int32 word, updated with
// bit operations only.
//
// Per (word, site): x = s XOR s_j marks the anti-aligned replicas of each present neighbour j; a ripple adder
// accumulates x into NP bit planes, so lane j of plane p holds bit p of replica j's anti-aligned count k. The
// lanes whose count is k form eq_k = AND_p (bit p of k ? c_p : ~c_p). The flip mask is assembled from the host
// acceptance table indexed [word, s, z_eff, k]:
//   shared mode      acc = OR_k (u < p[w, s, z_eff, k]) ? eq_k : 0, one uniform u per (word, site, sweep);
//   independent mode acc = lanes whose own 32-bit integer U is below P = floor(p 2^32), compared bit-sliced
//                    from the most significant bit: at level l a random word R_l holds bit 31 - l of every
//                    lane's U and pb the same bit of every lane's P; acc |= und & ~R_l & pb and
//                    und &= ~(R_l ^ pb); lanes with P = 2^32 accept outright, P = 0 never.
// The count templates ZM bound the coordination, so eq_k and the table entries stay in registers.
#include "internal.h"

namespace sck {

constexpr int bitlen(int v) { return v <= 0 ? 0 : 1 + bitlen(v >> 1); }

// Neighbour site indices of (x, y, z) along the sublattice's bonds, in bond order (-1: absent, outside an open box
// or masked); returns z_eff. Computed once per site and shared by every word the thread updates.
template <int ZM>
__device__ __forceinline__ int neighbour_sites(const Common& c, const SubDev& sub, int x, int y, int z,
                                               int (&nq)[ZM]) {
  const Geometry& g = c.g;
  int ze = 0;
#pragma unroll
  for (int bi = 0; bi < ZM; ++bi) {
    int q = -1;
    if (bi < sub.n_bonds) {
      q = neighbour_index(g, sub.bonds[bi], x, y, z);
      if (q >= 0 && g.has_mask && c.mask[q] == 0) q = -1;
    }
    nq[bi] = q;
    ze += q >= 0 ? 1 : 0;
  }
  return ze;
}

// Count planes c[0..NP) of one (word, site) from its neighbour sites: a ripple adder over the present bonds.
template <int NP, int ZM>
__device__ __forceinline__ void count_planes(const int (&nq)[ZM], uint32_t s0, const uint32_t* sp, size_t wb,
                                             uint32_t (&cp)[NP]) {
#pragma unroll
  for (int p = 0; p < NP; ++p) cp[p] = 0u;
#pragma unroll
  for (int bi = 0; bi < ZM; ++bi) {
    if (nq[bi] < 0) continue;
    uint32_t cy = s0 ^ sp[wb + nq[bi]];
#pragma unroll
    for (int p = 0; p < NP; ++p) {
      const uint32_t carry = cp[p] & cy;
      cp[p] ^= cy;
      cy = carry;
    }
  }
}

template <int NP>
__device__ __forceinline__ uint32_t lanes_with_count(const uint32_t (&cp)[NP], int k) {
  uint32_t eq = 0xFFFFFFFFu;
#pragma unroll
  for (int p = 0; p < NP; ++p) eq &= ((k >> p) & 1) ? cp[p] : ~cp[p];
  return eq;
}

// Shared draws: one thread per (group of four words, site); output q of one Philox call serves word 4 grp + q.
template <int ZM>
__device__ __forceinline__ void shared_site(const Common& c, const SubDev& sub, int alpha, int grp, int x, int y,
                                            int z, int32_t key, const uint32_t* src, uint32_t* dst) {
  constexpr int NP = bitlen(ZM);
  const Geometry& g = c.g;
  const int own = alpha * g.plane + (z * g.L2 + y) * g.L1 + x;
  if (g.has_mask && c.mask[own] == 0) return;
  const Philox4 r = philox4x32_10((uint32_t)((unsigned long long)grp * g.nsite + own), 0u, key_lo(key), key_hi(key));
  const float us[4] = {to_uniform(r.x0), to_uniform(r.x1), to_uniform(r.x2), to_uniform(r.x3)};
  const float* table = (const float*)c.table;
  int nq[ZM];
  const int ze = neighbour_sites<ZM>(c, sub, x, y, z, nq);
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int w = grp * 4 + q;
    if (w >= c.W) break;
    const size_t wb = (size_t)w * g.nsite;
    const uint32_t s0 = src[wb + own];
    uint32_t cp[NP];
    count_planes<NP, ZM>(nq, s0, src, wb, cp);
    const float* tb = table + (size_t)w * c.NT + ze * c.Z1;
    const float u = us[q];
    uint32_t acc = 0u;
#pragma unroll
    for (int k = 0; k <= ZM; ++k) {
      if (k <= ze) {
        const uint32_t eq = lanes_with_count<NP>(cp, k);
        if (c.field) {
          const float pm = tb[k], pp = tb[c.Z1 * c.Z1 + k];
          acc |= (u < pp ? (eq & s0) : 0u) | (u < pm ? (eq & ~s0) : 0u);
        } else {
          acc |= u < tb[k] ? eq : 0u;
        }
      }
    }
    dst[wb + own] = s0 ^ acc;
  }
}

constexpr long long TWO32 = 1LL << 32;

// Independent draws: one thread per (word, site).
template <int ZM>
__device__ __forceinline__ void independent_site(const Common& c, const SubDev& sub, int alpha, int w, int x, int y,
                                                 int z, int32_t key, const uint32_t* src, uint32_t* dst) {
  constexpr int NP = bitlen(ZM);
  const Geometry& g = c.g;
  const int own = alpha * g.plane + (z * g.L2 + y) * g.L1 + x;
  if (g.has_mask && c.mask[own] == 0) return;
  const size_t wb = (size_t)w * g.nsite;
  const uint32_t s0 = src[wb + own];
  uint32_t cp[NP];
  int nq[ZM];
  const int ze = neighbour_sites<ZM>(c, sub, x, y, z, nq);
  count_planes<NP, ZM>(nq, s0, src, wb, cp);
  const long long* tb = (const long long*)c.table + (size_t)w * c.NT + ze * c.Z1;
  uint32_t em[ZM + 1], ep[ZM + 1], Pm[ZM + 1], Pp[ZM + 1];
  uint32_t acc = 0u, und = 0u;
#pragma unroll
  for (int k = 0; k <= ZM; ++k) {
    em[k] = ep[k] = Pm[k] = Pp[k] = 0u;
    if (k <= ze) {
      const uint32_t eq = lanes_with_count<NP>(cp, k);
      const uint32_t lanes_m = c.field ? (eq & ~s0) : eq;
      const long long P_m = tb[k];
      if (P_m >= TWO32) acc |= lanes_m;
      else if (P_m > 0) { und |= lanes_m; em[k] = lanes_m; Pm[k] = (uint32_t)P_m; }
      if (c.field) {
        const uint32_t lanes_p = eq & s0;
        const long long P_p = tb[c.Z1 * c.Z1 + k];
        if (P_p >= TWO32) acc |= lanes_p;
        else if (P_p > 0) { und |= lanes_p; ep[k] = lanes_p; Pp[k] = (uint32_t)P_p; }
      }
    }
  }
  const uint32_t ctr = (uint32_t)((unsigned long long)w * g.nsite + own);
  for (int grp = 0; grp < 8; ++grp) {
    if (grp >= 2 && und == 0u) break;
    const long long kg64 = ((long long)key + (long long)(grp + 1) * 104729LL) % 2147483629LL;
    const int32_t kg = (int32_t)kg64;
    const Philox4 r = philox4x32_10(ctr, 0u, key_lo(kg), key_hi(kg));
    const uint32_t rw4[4] = {r.x0, r.x1, r.x2, r.x3};
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int sh = 31 - (4 * grp + q);
      uint32_t pb = 0u;
#pragma unroll
      for (int k = 0; k <= ZM; ++k)
        pb |= (em[k] & (0u - ((Pm[k] >> sh) & 1u))) | (ep[k] & (0u - ((Pp[k] >> sh) & 1u)));
      const uint32_t rw = rw4[q];
      acc |= und & ~rw & pb;
      und &= ~(rw ^ pb);
    }
  }
  dst[wb + own] = s0 ^ acc;
}

// Blocks of 256 threads per SM the class kernel is compiled for.
#ifndef SCK_BITWISE_MIN_BLOCKS
#define SCK_BITWISE_MIN_BLOCKS 4
#endif

// Grid (ceil(rows * bx / 256), units): units are groups of four words (shared) or words (independent).
template <int ZM, bool INDEP>
__global__ void __launch_bounds__(256, SCK_BITWISE_MIN_BLOCKS) bitwise_class_kernel(const __grid_constant__ ClassParams p) {
  const Common& c = p.c;
  const uint32_t per = (uint32_t)c.rows * (uint32_t)c.bx;
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= per) return;
  int x, y, z;
  if (!class_site(c, p.colour, p.alpha, t, x, y, z)) return;
  const int units = INDEP ? c.W : (c.W + 3) / 4;
  const int32_t key = sweep_key(c.state);
  for (int u = blockIdx.y; u < units; u += gridDim.y) {
    if (INDEP)
      independent_site<ZM>(c, p.sub, p.alpha, u, x, y, z, key, (const uint32_t*)c.src, (uint32_t*)c.dst);
    else
      shared_site<ZM>(c, p.sub, p.alpha, u, x, y, z, key, (const uint32_t*)c.src, (uint32_t*)c.dst);
  }
}

template <int ZM, bool INDEP>
__global__ void bitwise_sequential_kernel(const __grid_constant__ SeqParams p) {
  const Common& c = p.c;
  const int units = INDEP ? c.W : (c.W + 3) / 4;
  const int u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= units) return;
  const int32_t key = sweep_key(c.state);
  const Geometry& g = c.g;
  for (int ci = 0; ci < p.n_classes; ++ci) {
    const int colour = p.classes[ci][0], alpha = p.classes[ci][1];
    for (int z = 0; z < g.L3; ++z)
      for (int y = 0; y < g.L2; ++y)
        for (int x = 0; x < g.L1; ++x) {
          if (colour_of(c.col, alpha, x, y, z) != colour) continue;
          if (INDEP)
            independent_site<ZM>(c, p.sub[alpha], alpha, u, x, y, z, key, (const uint32_t*)c.dst, (uint32_t*)c.dst);
          else
            shared_site<ZM>(c, p.sub[alpha], alpha, u, x, y, z, key, (const uint32_t*)c.dst, (uint32_t*)c.dst);
        }
  }
}

template <bool INDEP>
static void class_dispatch(int Z, const ClassParams& p, dim3 grid, cudaStream_t s) {
  if (Z <= 4) bitwise_class_kernel<4, INDEP><<<grid, 256, 0, s>>>(p);
  else if (Z <= 6) bitwise_class_kernel<6, INDEP><<<grid, 256, 0, s>>>(p);
  else if (Z <= 8) bitwise_class_kernel<8, INDEP><<<grid, 256, 0, s>>>(p);
  else if (Z <= 12) bitwise_class_kernel<12, INDEP><<<grid, 256, 0, s>>>(p);
  else if (Z <= 16) bitwise_class_kernel<16, INDEP><<<grid, 256, 0, s>>>(p);
  else if (Z <= 32) bitwise_class_kernel<32, INDEP><<<grid, 256, 0, s>>>(p);
  else bitwise_class_kernel<64, INDEP><<<grid, 256, 0, s>>>(p);
}

template <bool INDEP>
static void seq_dispatch(int Z, const SeqParams& p, int grid, int block, cudaStream_t s) {
  if (Z <= 4) bitwise_sequential_kernel<4, INDEP><<<grid, block, 0, s>>>(p);
  else if (Z <= 6) bitwise_sequential_kernel<6, INDEP><<<grid, block, 0, s>>>(p);
  else if (Z <= 8) bitwise_sequential_kernel<8, INDEP><<<grid, block, 0, s>>>(p);
  else if (Z <= 12) bitwise_sequential_kernel<12, INDEP><<<grid, block, 0, s>>>(p);
  else if (Z <= 16) bitwise_sequential_kernel<16, INDEP><<<grid, block, 0, s>>>(p);
  else if (Z <= 32) bitwise_sequential_kernel<32, INDEP><<<grid, block, 0, s>>>(p);
  else bitwise_sequential_kernel<64, INDEP><<<grid, block, 0, s>>>(p);
}

int launch_bitwise_class(const sck_plan* plan, const Common& c, int colour, int alpha, cudaStream_t s) {
  ClassParams p;
  p.c = c;
  p.sub = plan->sub[alpha];
  p.colour = colour;
  p.alpha = alpha;
  if (colour < 0) set_rows(p.c, 1, c.g.L1);
  const bool indep = plan->mode == SCK_MODE_BITWISE_INDEP;
  const int units = indep ? c.W : (c.W + 3) / 4;
  const uint32_t per = (uint32_t)p.c.rows * (uint32_t)p.c.bx;
  const dim3 grid((per + 255) / 256, (unsigned)(units < 65535 ? units : 65535));
  if (indep)
    class_dispatch<true>(plan->Z, p, grid, s);
  else
    class_dispatch<false>(plan->Z, p, grid, s);
  return cuda_status(cudaGetLastError(), "bitwise class launch");
}

int launch_bitwise_sequential(const sck_plan* plan, const Common& c, cudaStream_t s) {
  SeqParams p;
  p.c = c;
  for (int a = 0; a < SCK_MAX_BASIS; ++a) p.sub[a] = plan->sub[a];
  p.n_classes = plan->desc.n_classes;
  for (int i = 0; i < p.n_classes; ++i) {
    p.classes[i][0] = plan->desc.classes[i][0];
    p.classes[i][1] = plan->desc.classes[i][1];
  }
  const bool indep = plan->mode == SCK_MODE_BITWISE_INDEP;
  const int units = indep ? c.W : (c.W + 3) / 4;
  const int block = 32;
  const int grid = (units + block - 1) / block;
  if (indep)
    seq_dispatch<true>(plan->Z, p, grid, block, s);
  else
    seq_dispatch<false>(plan->Z, p, grid, block, s);
  return cuda_status(cudaGetLastError(), "bitwise sequential launch");
}

}  // namespace sck
