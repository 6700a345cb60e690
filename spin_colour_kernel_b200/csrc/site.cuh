// Generic site updates shared by the class kernels (sweep.cu), the resident kernel and ragged batches
// (batch.cu): one (class site, replica) of any system, with the bond list read from a runtime descriptor.
#pragma once

#include "internal.h"

namespace sck {

__device__ __forceinline__ uint32_t counter32(long long rep, int nsite, int own) {
  return (uint32_t)((unsigned long long)rep * (unsigned long long)nsite + (unsigned long long)own);
}

// ---------------------------------------------------------------------------------------------- Ising (LUT)
// Spin values enter the key through their sign, so a malformed value can never index outside the table.
template <typename T>
__device__ __forceinline__ int spin_sign(T v) { return (v > T(0)) - (v < T(0)); }

// src / dst point at replica `rep`'s block (global memory, or shared memory in the resident kernel); rep only
// selects the random stream and the table row.
template <typename ST>
__device__ __forceinline__ void ising_site(const Common& c, const SubDev& sub, int alpha, int rep, int x, int y,
                                           int z, int32_t key, const ST* src, ST* dst) {
  const Geometry& g = c.g;
  const int own = alpha * g.plane + (z * g.L2 + y) * g.L1 + x;
  if (g.has_mask && c.mask[own] == 0) return;
  const int s = spin_sign(src[own]);
  int k = s > 0 ? 1 : 0;
  int bi = 0;
#pragma unroll
  for (int gi = 0; gi < SCK_MAX_GROUPS; ++gi) {
    if (gi < sub.n_groups) {
      int G = 0;
      for (; bi < sub.group_end[gi]; ++bi) {
        const BondDev bd = sub.bonds[bi];
        const int q = neighbour_index(g, bd, x, y, z);
        const int t = q >= 0 ? spin_sign(src[q]) : 0;
        G += t;
        if (bd.extra >= 0) k += (t + 1) * sub.extra_stride[bd.extra];
      }
      k += (G + sub.group_z[gi]) * sub.key_stride[gi];
    }
  }
  const float e = ((const float*)c.table)[(size_t)rep * c.lut_rep_stride + alpha * c.keys + k];
  const Philox4 r = philox4x32_10(counter32(rep, g.nsite, own), 0u, key_lo(key), key_hi(key));
  const float u0 = to_uniform(r.x0);
  const bool acc = g.acceptance == SCK_BARKER ? __fmul_rn(u0, __fadd_rn(1.0f, e)) < 1.0f : u0 < e;
  if (acc)
    dst[own] = (ST)(-s);
  else if ((const void*)src != (const void*)dst)
    dst[own] = (ST)s;
}

// ------------------------------------------------------------------------------------------- vector models
template <int N>
__device__ __forceinline__ void vec_site(const Common& c, const SubDev& sub, int alpha, int rep, int x, int y,
                                         int z, int32_t key, const float* src, float* dst) {
  const Geometry& g = c.g;
  const int own = alpha * g.plane + (z * g.L2 + y) * g.L1 + x;
  if (g.has_mask && c.mask[own] == 0) return;
  const int NS = g.nsite;
  float s[N], v[N];
#pragma unroll
  for (int k = 0; k < N; ++k) {
    s[k] = src[k * NS + own];
    v[k] = 0.0f;
  }
  float ex[SCK_MAX_EXTRA][N];
  int bi = 0;
#pragma unroll
  for (int gi = 0; gi < SCK_MAX_GROUPS; ++gi) {
    if (gi < sub.n_groups) {
      float gs[N];
#pragma unroll
      for (int k = 0; k < N; ++k) gs[k] = 0.0f;
      for (; bi < sub.group_end[gi]; ++bi) {
        const BondDev bd = sub.bonds[bi];
        const int q = neighbour_index(g, bd, x, y, z);
#pragma unroll
        for (int k = 0; k < N; ++k) {
          const float t = q >= 0 ? src[k * NS + q] : 0.0f;
          gs[k] = __fadd_rn(gs[k], t);
          if (bd.extra >= 0) ex[bd.extra][k] = t;
        }
      }
      if (sub.apply[gi]) {
#pragma unroll
        for (int k = 0; k < N; ++k) v[k] = __fadd_rn(v[k], __fmul_rn(sub.J[gi], gs[k]));
      }
    }
  }
  for (int e = 0; e < sub.n_extra; ++e) {
#pragma unroll
    for (int k = 0; k < N; ++k) {
      float tot = 0.0f;
      bool any = false;
#pragma unroll
      for (int l = 0; l < N; ++l) {
        if ((sub.Enz[e] >> (3 * k + l)) & 1) {
          const float term = __fmul_rn(sub.E[e][3 * k + l], ex[e][l]);
          tot = any ? __fadd_rn(tot, term) : term;
          any = true;
        }
      }
      if (any) v[k] = __fadd_rn(v[k], tot);
    }
  }
#pragma unroll
  for (int k = 0; k < N; ++k)
    if (c.hnz[k]) v[k] = __fadd_rn(v[k], c.h[k]);

  const Philox4 r = philox4x32_10(counter32(rep, g.nsite, own), 0u, key_lo(key), key_hi(key));
  const float u0 = to_uniform(r.x0);
  const float TWO_PI = 6.2831855f;
  float t[N];
  if (N == 2) {
    float sn, cs;
    sincosf(__fmul_rn(TWO_PI, to_uniform(r.x1)), &sn, &cs);
    t[0] = cs;
    t[1 % N] = sn;
  } else if (N == 3) {
    const float cz = __fsub_rn(__fmul_rn(2.0f, to_uniform(r.x1)), 1.0f);
    float sn, cs;
    sincosf(__fmul_rn(TWO_PI, to_uniform(r.x2)), &sn, &cs);
    const float rr = sqrtf(fmaxf(__fsub_rn(1.0f, __fmul_rn(cz, cz)), 0.0f));
    t[0] = __fmul_rn(rr, cs);
    t[1 % N] = __fmul_rn(rr, sn);
    t[2 % N] = cz;
  } else {
    t[0] = -s[0];
  }
  float d = __fmul_rn(__fsub_rn(t[0], s[0]), v[0]);
#pragma unroll
  for (int k = 1; k < N; ++k) d = __fadd_rn(d, __fmul_rn(__fsub_rn(t[k], s[k]), v[k]));
  float dE = -d;
  if (N == 3 && g.has_cubic) {
    const float k1 = c.k1[own];
    auto aniso = [&](const float* p) {
      const float q01 = __fmul_rn(p[0], p[1 % N]), q02 = __fmul_rn(p[0], p[2 % N]);
      const float q12 = __fmul_rn(p[1 % N], p[2 % N]);
      const float tri = __fmul_rn(q01, p[2 % N]);
      const float quad = __fadd_rn(__fadd_rn(__fmul_rn(q01, q01), __fmul_rn(q02, q02)), __fmul_rn(q12, q12));
      return __fadd_rn(__fmul_rn(k1, quad), __fmul_rn(__fmul_rn(c.k2, tri), tri));
    };
    dE = __fadd_rn(dE, __fsub_rn(aniso(t), aniso(s)));
  }
  const float beta = c.beta[rep];
  bool acc;
  if (g.acceptance == SCK_BARKER)
    acc = __fmul_rn(u0, __fadd_rn(1.0f, expf(__fmul_rn(beta, dE)))) < 1.0f;
  else
    acc = u0 < expf(__fmul_rn(-beta, dE));
  if (acc || (const void*)src != (const void*)dst) {
#pragma unroll
    for (int k = 0; k < N; ++k) dst[k * NS + own] = acc ? t[k] : s[k];
  }
}

}  // namespace sck
