// Site updates of the specialised lattice kernels (compile-time bond tables of lattices.h), shared by the class
// and pipeline kernels of fast_sweep.cu and the ragged-batch kernel of batch.cu.
#pragma once

#include "spec.cuh"

namespace sck {

// Wrapped coordinates of one site for compile-time offsets -R..R on each axis. PER: every axis of the box is
// periodic (2D systems never offset along z) and each extent is at least R, so one conditional add or subtract
// wraps an offset and no validity is tracked; otherwise open axes mark neighbours outside the box invalid.
template <int R, bool PER>
struct Around {
  int xo[2 * R + 1], yo[2 * R + 1], zo[2 * R + 1];
  bool xv[2 * R + 1], yv[2 * R + 1], zv[2 * R + 1];

  __device__ __forceinline__ static int wrap1(int x, int d, int L) {
    int q = x + d;
    q += q < 0 ? L : 0;
    q -= q >= L ? L : 0;
    return q;
  }

  __device__ __forceinline__ Around(const Geometry& g, int x, int y, int z) {
#pragma unroll
    for (int d = -R; d <= R; ++d) {
      int qx, qy, qz;
      if constexpr (PER) {
        qx = wrap1(x, d, g.L1);
        qy = wrap1(y, d, g.L2);
        qz = g.dim == 3 ? wrap1(z, d, g.L3) : z;
      } else {
        qx = wrap_axis(x, d, g.L1, g.per[0]);
        qy = wrap_axis(y, d, g.L2, g.per[1]);
        qz = wrap_axis(z, d, g.L3, g.per[2]);
      }
      xv[d + R] = qx >= 0;
      yv[d + R] = qy >= 0;
      zv[d + R] = qz >= 0;
      xo[d + R] = qx < 0 ? 0 : qx;
      yo[d + R] = (qy < 0 ? 0 : qy) * g.L1;
      zo[d + R] = (qz < 0 ? 0 : qz) * g.L2 * g.L1;
    }
  }
  __device__ __forceinline__ int index(const Geometry& g, const BondC b) const {
    return b.a2 * g.plane + zo[b.dz + R] + yo[b.dy + R] + xo[b.dx + R];
  }
  __device__ __forceinline__ bool valid(const BondC b) const {
    if constexpr (PER) return true;
    return xv[b.dx + R] && yv[b.dy + R] && zv[b.dz + R];
  }
};

// ---------------------------------------------------------------------------------------------------- Ising
template <class Lat, int A, typename ST, bool PER>
__device__ __forceinline__ void ising_spec_site(const Common& c, int rep, int x, int y, int z, int32_t key) {
  const Geometry& g = c.g;
  const int own = A * g.plane + (z * g.L2 + y) * g.L1 + x;
  if (g.has_mask && c.mask[own] == 0) return;
  const ST* src = (const ST*)c.src + (size_t)rep * g.nsite;
  ST* dst = (ST*)c.dst + (size_t)rep * g.nsite;
  const int s = sgn(src[own]);
  const Around<Lat::reach, PER> nb(g, x, y, z);
  int k = s > 0 ? 1 : 0;
  int stride = 2;
  static_for<0, Lat::groups>([&](auto gc) {
    using R = GroupRange<Lat, A, decltype(gc)::value>;
    int G = 0;
    static_for<R::begin, R::end>([&](auto ic) {
      constexpr BondC bd = Lat::bond(A, decltype(ic)::value);
      G += nb.valid(bd) ? sgn(src[nb.index(g, bd)]) : 0;
    });
    k += (G + (R::end - R::begin)) * stride;
    stride *= 2 * (R::end - R::begin) + 1;
  });
  const float e = ((const float*)c.table)[(size_t)rep * c.lut_rep_stride + A * c.keys + k];
  const Philox4 r = philox4x32_10(counter_of(rep, g.nsite, own), 0u, key_lo(key), key_hi(key));
  const float u0 = to_uniform(r.x0);
  const bool acc = g.acceptance == SCK_BARKER ? __fmul_rn(u0, __fadd_rn(1.0f, e)) < 1.0f : u0 < e;
  if (acc) dst[own] = (ST)(-s);
}

// --------------------------------------------------------------------------------------------- vector models
// Two replicas (lanes .x and .y) of one class site. `two` = false runs lane y as a copy of lane x and stores
// lane x only (an odd replica count).
// NSL > 0: the replica has 2^NSL sites, so component offsets are compile-time and every neighbour load of a
// replica is one address plus an immediate offset (each replica of the pair gets its own base); NSL = 0: one
// base for the pair, runtime offsets.
template <class Lat, int A, int N, bool PER, int NSL>
__device__ __forceinline__ void vec_spec_pair(const Common& c, const float (&J)[SCK_MAX_GROUPS], int rep0, bool two,
                                              int x, int y, int z, int32_t key) {
  const Geometry& g = c.g;
  const int own = A * g.plane + (z * g.L2 + y) * g.L1 + x;
  if (g.has_mask && c.mask[own] == 0) return;
  // component k of replica rep0 + j sits at k * NS + j * RS
  const float* base = (const float*)c.src + (size_t)rep0 * N * g.nsite;
  float* obase = (float*)c.dst + (size_t)rep0 * N * g.nsite;
  const size_t NS = NSL ? ((size_t)1 << NSL) : (size_t)g.nsite, RS = two ? (size_t)N * NS : 0;
  const float* base1 = base + RS;
  const int rep1 = two ? rep0 + 1 : rep0;
  const Around<Lat::reach, PER> nb(g, x, y, z);
  float2 s[N], v[N];
  {
    const float* po = base + own;
#pragma unroll
    for (int k = 0; k < N; ++k) {
      s[k] = make_float2(po[k * NS], po[k * NS + RS]);
      v[k] = f2(0.0f);
    }
  }
  static_for<0, Lat::groups>([&](auto gc) {
    constexpr int gi = decltype(gc)::value;
    using R = GroupRange<Lat, A, gi>;
    float2 gs[N];
#pragma unroll
    for (int k = 0; k < N; ++k) gs[k] = f2(0.0f);
    static_for<R::begin, R::end>([&](auto ic) {
      constexpr BondC bd = Lat::bond(A, decltype(ic)::value);
      const int qi = nb.index(g, bd);
      const float* pq = base + qi;
      const float* pq1 = base1 + qi;
      const bool ok = nb.valid(bd);
#pragma unroll
      for (int k = 0; k < N; ++k) {
        float2 t;
        if constexpr (NSL > 0)
          t = ok ? make_float2(pq[k * NS], pq1[k * NS]) : f2(0.0f);
        else
          t = ok ? make_float2(pq[k * NS], pq[k * NS + RS]) : f2(0.0f);
        gs[k] = __fadd2_rn(gs[k], t);
      }
    });
#pragma unroll
    for (int k = 0; k < N; ++k) v[k] = __fadd2_rn(v[k], __fmul2_rn(f2(J[gi]), gs[k]));
  });
#pragma unroll
  for (int k = 0; k < N; ++k)
    if (c.hnz[k]) v[k] = __fadd2_rn(v[k], f2(c.h[k]));
  float2 t[N];
  bool acc0, acc1;
  finish_pair<N>(c, own, rep0, rep1, two, key, s, v, t, acc0, acc1);
  float* po = obase + own;
  if (acc0) {
#pragma unroll
    for (int k = 0; k < N; ++k) po[k * NS] = t[k].x;
  }
  if (two && acc1) {
#pragma unroll
    for (int k = 0; k < N; ++k) po[k * NS + RS] = t[k].y;
  }
}

}  // namespace sck
