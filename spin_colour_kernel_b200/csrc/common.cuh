// Device-side definitions shared by every kernel of libsckb200: geometry, colouring, the per-sublattice bond
// descriptor passed in kernel-parameter (constant-bank) space, Philox4x32-10 and the uniform conversion.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/sck.h"

namespace sck {

// ------------------------------------------------------------------------------------------------ geometry
struct Geometry {
  int n, b, dim;
  int L1, L2, L3;
  int per[3];
  int plane;   // L3 * L2 * L1: one (component, sublattice) plane
  int nsite;   // b * plane
  int has_mask, has_cubic, acceptance;
};

struct Colouring {
  int r;
  int m[SCK_MAX_FACTORS];
  int K[SCK_MAX_FACTORS][3];
  int o[SCK_MAX_BASIS][SCK_MAX_FACTORS];
};

// One bond in 8 bytes: neighbour sublattice, cell offset, extra-matrix slot (-1 none).
struct BondDev {
  int8_t a2, dx, dy, dz, extra, pad0, pad1, pad2;
};

// The bonds of one sublattice in accumulation order (groups contiguous), with the float32 couplings of the
// sweep and the mixed-radix strides of the Ising acceptance-table key.
struct SubDev {
  int n_bonds, n_groups, n_extra;
  int group_end[SCK_MAX_GROUPS];
  float J[SCK_MAX_GROUPS];
  int apply[SCK_MAX_GROUPS];
  int key_stride[SCK_MAX_GROUPS];    // Ising key: (G_g + z_g) * stride (0 when the group is not applied)
  int group_z[SCK_MAX_GROUPS];       // members of the group = largest |G_g|
  int extra_stride[SCK_MAX_EXTRA];   // Ising key: (n_slot + 1) * stride (0 when E == 0)
  float E[SCK_MAX_EXTRA][9];
  int Enz[SCK_MAX_EXTRA];            // bit 3k+l set when E[k][l] != 0
  BondDev bonds[SCK_MAX_BONDS];
};

// FP64 couplings of one sublattice for the observables (same bond order as SubDev).
struct SubObs {
  int n_bonds;
  double J[SCK_MAX_BONDS];
  double E[SCK_MAX_EXTRA][9];
};

// ------------------------------------------------------------------------------------------- fast division
// Division by a runtime-invariant divisor d >= 1 through one 32x32->64 multiply and a shift (Granlund and
// Montgomery, PLDI'94): with l = ceil(log2 d), m = ceil(2^(31+l) / d) fits in 32 bits and
// floor(n m / 2^(31+l)) = floor(n / d) for every 0 <= n < 2^31 (the rounding error n (m d - 2^(31+l)) /
// (d 2^(31+l)) stays below 2^-l <= 1/d).
struct FastDiv {
  uint32_t m, s;
};

inline FastDiv make_fastdiv(uint32_t d) {
  uint32_t l = 0;
  while ((1ull << l) < d) ++l;
  const unsigned long long m = ((1ull << (31 + l)) + d - 1) / d;
  return FastDiv{(uint32_t)m, 31 + l};
}

__host__ __device__ __forceinline__ uint32_t fdiv(uint32_t n, FastDiv f) {
  return (uint32_t)(((unsigned long long)n * f.m) >> f.s);
}

// ------------------------------------------------------------------------------------------------- helpers
__host__ __device__ inline int colour_of(const Colouring& c, int a, int x, int y, int z) {
  int idx = 0;
  for (int r = 0; r < c.r; ++r) {
    int g = (c.K[r][0] * x + c.K[r][1] * y + c.K[r][2] * z + c.o[a][r]) % c.m[r];
    idx = idx * c.m[r] + g;
  }
  return idx;
}

// Neighbour coordinate along one axis: periodic wrap, or -1 outside an open box. Offsets are bounded by the
// descriptor check (|d| <= 64); the remainder is taken only when a tiny box needs more than one wrap.
__device__ __forceinline__ int wrap_axis(int x, int d, int L, int periodic) {
  int q = x + d;
  if (periodic) {
    if (q < 0) q += L;
    else if (q >= L) q -= L;
    if ((unsigned)q >= (unsigned)L) q = ((q % L) + L) % L;
    return q;
  }
  return (q >= 0 && q < L) ? q : -1;
}

// Site index of the neighbour of (x, y, z) along bond bd, or -1 when it lies outside an open box.
__device__ __forceinline__ int neighbour_index(const Geometry& g, const BondDev& bd, int x, int y, int z) {
  int qx = wrap_axis(x, bd.dx, g.L1, g.per[0]);
  int qy = wrap_axis(y, bd.dy, g.L2, g.per[1]);
  int qz = wrap_axis(z, bd.dz, g.L3, g.per[2]);
  if ((qx | qy | qz) < 0) return -1;
  return bd.a2 * g.plane + (qz * g.L2 + qy) * g.L1 + qx;
}

// ---------------------------------------------------------------------------------------------- randomness
// Per-sweep Philox key: (base_seed * 1000003 + sweep * 7919 + 12345) mod 2147483629 with int64 wrap-around
// products and a C remainder, then truncated to int32 (generator.py:205).
__device__ __forceinline__ int32_t sweep_key(const int64_t* state) {
  uint64_t v = (uint64_t)state[0] * 1000003ull + (uint64_t)state[1] * 7919ull + 12345ull;
  int64_t sv = (int64_t)v;
  return (int32_t)(sv % 2147483629ll);
}

// The key of sweep state[1] + offset (kernels that run several sweeps of one call).
__device__ __forceinline__ int32_t sweep_key_at(const int64_t* state, int offset) {
  const uint64_t v = (uint64_t)state[0] * 1000003ull + (uint64_t)(state[1] + offset) * 7919ull + 12345ull;
  return (int32_t)((int64_t)v % 2147483629ll);
}

// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11) with counter (c0, c1, 0, 0) and key (k0, k1): the
// generator of Triton's randint4x. Each round multiplies c0 and c2 by the round constants, keeps the low
// halves and mixes the high halves with the other words and the key; the key steps by the Weyl constants.
struct Philox4 {
  uint32_t x0, x1, x2, x3;
};

__device__ __forceinline__ Philox4 philox4x32_10(uint32_t c0, uint32_t c1, uint32_t k0, uint32_t k1) {
  uint32_t c2 = 0u, c3 = 0u;
#pragma unroll
  for (int i = 0; i < 10; ++i) {
    const uint32_t lo_a = 0xD2511F53u * c0, hi_a = __umulhi(0xD2511F53u, c0);
    const uint32_t lo_b = 0xCD9E8D57u * c2, hi_b = __umulhi(0xCD9E8D57u, c2);
    c0 = hi_b ^ c1 ^ k0;
    c2 = hi_a ^ c3 ^ k1;
    c1 = lo_b;
    c3 = lo_a;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  return Philox4{c0, c1, c2, c3};
}

// Key words of an int32 seed extended to int64 (Triton: seed.to(uint64), low and high halves).
__device__ __forceinline__ uint32_t key_lo(int32_t seed) { return (uint32_t)seed; }
__device__ __forceinline__ uint32_t key_hi(int32_t seed) { return seed < 0 ? 0xFFFFFFFFu : 0u; }

// Triton's uint_to_uniform_float for 32-bit words: x as int32, x < 0 -> -x - 1, times float32 4.6566127342e-10
// (bit pattern 0x2FFFFFFF), all in round-to-nearest float32.
__device__ __forceinline__ float to_uniform(uint32_t bits) {
  int32_t i = (int32_t)bits;
  i = i < 0 ? ~i : i;
  return __fmul_rn(__int2float_rn(i), __int_as_float(0x2FFFFFFF));
}

}  // namespace sck
