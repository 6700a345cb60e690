// Shared pieces of the specialised class kernels (fast_sweep.cu, segment.cu): task lists of the L2 group
// pipeline, compile-time loops over the lattice tables, and the second half of a vector-model update (proposal,
// energy change, anisotropy, acceptance) for two attempts in packed float32x2 arithmetic.
#pragma once

#include <type_traits>

#include "internal.h"
#include "lattices.h"

namespace sck {

struct Task {
  int colour, alpha, rep_begin, rep_end, sweep_offset;
};

constexpr int kMaxTasks = 8;

struct SpecParams {
  Common c;
  float J[SCK_MAX_BASIS][SCK_MAX_GROUPS];
  int n_tasks;
  int units_per_task;     // grid.y slots per task (replicas, or replica pairs for vector models)
  FastDiv fd_segs;        // segment kernels: 4-site segments per row
  Task tasks[kMaxTasks];
};

// The streamed group pipeline (fast_sweep.cu:stream_kernel).
struct StreamParams {
  Common c;
  float J[SCK_MAX_BASIS][SCK_MAX_GROUPS];
  int C;                  // classes per sweep, in sweep order
  int cls[8][2];          // (colour, alpha) of each class
  int group, ngroups;     // replicas per group, groups
  int units;              // sweeps of this launch x groups
  int sweep_base;         // sweeps run by earlier launches of the same call
  int chunks;             // tickets per slot (replica or replica pair) and class
  int T;                  // tickets per class task: slots per group x chunks
  unsigned* ticket;       // next ticket
  unsigned* done;         // finished tickets per (group, class), summed over the launch's sweeps
};

__device__ __forceinline__ uint32_t counter_of(int rep, int nsite, int own) {
  return (uint32_t)((unsigned long long)rep * (unsigned long long)nsite + (unsigned long long)own);
}

template <typename T>
__device__ __forceinline__ int sgn(T v) { return (v > T(0)) - (v < T(0)); }

// Compile-time loop: f(std::integral_constant<int, I>) for I in [B, E).
template <int I, int E, class F>
__device__ __forceinline__ void static_for(F&& f) {
  if constexpr (I < E) {
    f(std::integral_constant<int, I>{});
    static_for<I + 1, E>(f);
  }
}

template <class Lat, int A, int G>
struct GroupRange {
  static constexpr int begin = G == 0 ? 0 : Lat::group_end(A, G - 1);
  static constexpr int end = Lat::group_end(A, G);
};

// A bond of a compile-time table points "forward" when it goes to a higher sublattice, or within a sublattice
// to a positive offset in z, then y, then x; summing forward bonds only visits every bond of the lattice once.
template <class Lat, int A>
__host__ __device__ constexpr bool forward_bond(int i) {
  const BondC b = Lat::bond(A, i);
  if (b.a2 != A) return b.a2 > A;
  if (b.dz != 0) return b.dz > 0;
  if (b.dy != 0) return b.dy > 0;
  return b.dx > 0;
}

template <class Lat>
__host__ __device__ constexpr bool bonds_paired() {
  for (int a = 0; a < Lat::b; ++a)
    for (int i = 0; i < Lat::n_bonds(a); ++i) {
      const BondC b = Lat::bond(a, i);
      bool found = false;
      for (int j = 0; j < Lat::n_bonds(b.a2); ++j) {
        const BondC r = Lat::bond(b.a2, j);
        if (r.a2 == a && r.dx == -b.dx && r.dy == -b.dy && r.dz == -b.dz) {
          int gi = 0, gj = 0;
          while (Lat::group_end(a, gi) <= i) ++gi;
          while (Lat::group_end(b.a2, gj) <= j) ++gj;
          found = found || gi == gj;
        }
      }
      if (!found) return false;
    }
  return true;
}

__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }

// sin and cos of phi in [0, 2 pi] through the SFU on the reduced range [-pi, pi].
__device__ __forceinline__ void sincos_2pi(float phi, float& sn, float& cs) {
  const float red = phi - 3.14159265358979f;
  sn = -__sinf(red);
  cs = -__cosf(red);
}

// Proposal, energy change with cubic anisotropy, and Metropolis / Barker decision of two attempts (lane .x, lane
// .y) with Philox counters cnt0 / cnt1, anisotropy coefficients k1 (used only when `cubic`) and inverse
// temperatures beta, given their spins s and local fields v (field included). Returns the proposals in t and the
// decisions in acc0 / acc1. Same operation order as the reference's kernel (generator.py:275-305); packed
// float32x2 operations round each lane to nearest. With two == false lane .y repeats lane .x's draws and its
// result is ignored. The lattice kernels (finish_core below) and the interleaved kernels (quad.cu) both call it,
// so the two storage layouts compute identical numbers.
// With MEAS (a measure step), also fm: the products s.wm and t.wm with the measure field wm (the fields of the
// neighbours updated earlier in the sweep and the external field), and the anisotropy energies of s and t (0
// without cubic anisotropy), so that the energy share of the site's final spin needs no second evaluation.
struct FinishMeasure {
  float2 es, et, as, at;
};

template <int N, bool MEAS = false>
__device__ __forceinline__ void finish_values(int acceptance, bool cubic, float2 k1, float k2c, uint32_t cnt0,
                                              uint32_t cnt1, bool two, float2 beta, int32_t key, const float2 (&s)[N],
                                              const float2 (&v)[N], float2 (&t)[N], bool& acc0, bool& acc1,
                                              const float2 (*wm)[N] = nullptr, FinishMeasure* fm = nullptr) {
  const Philox4 ra = philox4x32_10(cnt0, 0u, key_lo(key), key_hi(key));
  const Philox4 rb = two ? philox4x32_10(cnt1, 0u, key_lo(key), key_hi(key)) : ra;
  const float2 u0 = make_float2(to_uniform(ra.x0), to_uniform(rb.x0));
  const float TWO_PI = 6.2831855f;
  if constexpr (N == 2) {
    float sa, ca, sb, cb;
    sincos_2pi(__fmul_rn(TWO_PI, to_uniform(ra.x1)), sa, ca);
    sincos_2pi(__fmul_rn(TWO_PI, to_uniform(rb.x1)), sb, cb);
    t[0] = make_float2(ca, cb);
    t[1] = make_float2(sa, sb);
  } else {
    const float2 u1 = make_float2(to_uniform(ra.x1), to_uniform(rb.x1));
    const float2 cz = __fadd2_rn(__fmul2_rn(f2(2.0f), u1), f2(-1.0f));
    float sa, ca, sb, cb;
    sincos_2pi(__fmul_rn(TWO_PI, to_uniform(ra.x2)), sa, ca);
    sincos_2pi(__fmul_rn(TWO_PI, to_uniform(rb.x2)), sb, cb);
    const float2 w = __fadd2_rn(f2(1.0f), __fmul2_rn(f2(-1.0f), __fmul2_rn(cz, cz)));
    // sqrt(w) as w * rsqrt(w) on the SFU (a few ulp, like the SFU sine and cosine above; w = 0 gives 0)
    const float2 rr = make_float2(w.x > 0.0f ? w.x * rsqrtf(w.x) : 0.0f, w.y > 0.0f ? w.y * rsqrtf(w.y) : 0.0f);
    t[0] = __fmul2_rn(rr, make_float2(ca, cb));
    t[1] = __fmul2_rn(rr, make_float2(sa, sb));
    t[2] = cz;
  }
  // -1 * x is exact, so the reference's t + (-1) s and (-1) d are written as a subtraction and a negation
  auto neg = [](float2 a) { return make_float2(-a.x, -a.y); };
  if constexpr (MEAS) {
    float2 es = __fmul2_rn(s[0], (*wm)[0]), et = __fmul2_rn(t[0], (*wm)[0]);
#pragma unroll
    for (int k = 1; k < N; ++k) {
      es = __fadd2_rn(es, __fmul2_rn(s[k], (*wm)[k]));
      et = __fadd2_rn(et, __fmul2_rn(t[k], (*wm)[k]));
    }
    fm->es = es;
    fm->et = et;
    fm->as = fm->at = f2(0.0f);
  }
  float2 d = __fmul2_rn(__fadd2_rn(t[0], neg(s[0])), v[0]);
#pragma unroll
  for (int k = 1; k < N; ++k) d = __fadd2_rn(d, __fmul2_rn(__fadd2_rn(t[k], neg(s[k])), v[k]));
  float2 dE = neg(d);
  if constexpr (N == 3) {
    if (cubic) {
      const float2 k2 = f2(k2c);
      auto aniso = [&](const float2* p) {
        const float2 q01 = __fmul2_rn(p[0], p[1]), q02 = __fmul2_rn(p[0], p[2]), q12 = __fmul2_rn(p[1], p[2]);
        const float2 tri = __fmul2_rn(q01, p[2]);
        const float2 quad = __fadd2_rn(__fadd2_rn(__fmul2_rn(q01, q01), __fmul2_rn(q02, q02)), __fmul2_rn(q12, q12));
        return __fadd2_rn(__fmul2_rn(k1, quad), __fmul2_rn(__fmul2_rn(k2, tri), tri));
      };
      const float2 an_t = aniso(t), an_s = aniso(s);
      dE = __fadd2_rn(dE, __fadd2_rn(an_t, neg(an_s)));
      if constexpr (MEAS) {
        fm->as = an_s;
        fm->at = an_t;
      }
    }
  }
  if (acceptance == SCK_BARKER) {
    const float2 xb = __fmul2_rn(beta, dE);
    acc0 = __fmul_rn(u0.x, __fadd_rn(1.0f, __expf(xb.x))) < 1.0f;
    acc1 = __fmul_rn(u0.y, __fadd_rn(1.0f, __expf(xb.y))) < 1.0f;
  } else {
    const float2 xm = __fmul2_rn(neg(beta), dE);
    acc0 = u0.x < __expf(xm.x);
    acc1 = u0.y < __expf(xm.y);
  }
}

template <int N>
__device__ __forceinline__ void finish_core(const Common& c, uint32_t cnt0, uint32_t cnt1, bool two, int k1_0,
                                            int k1_1, float2 beta, int32_t key, const float2 (&s)[N],
                                            const float2 (&v)[N], float2 (&t)[N], bool& acc0, bool& acc1) {
  const bool cubic = N == 3 && c.g.has_cubic;
  const float2 k1 = cubic ? make_float2(c.k1[k1_0], c.k1[k1_1]) : f2(0.0f);
  finish_values<N>(c.g.acceptance, cubic, k1, c.k2, cnt0, cnt1, two, beta, key, s, v, t, acc0, acc1);
}

// Two replicas rep0 / rep1 of site `own`.
template <int N>
__device__ __forceinline__ void finish_pair(const Common& c, int own, int rep0, int rep1, bool two, int32_t key,
                                            const float2 (&s)[N], const float2 (&v)[N], float2 (&t)[N], bool& acc0,
                                            bool& acc1) {
  finish_core<N>(c, counter_of(rep0, c.g.nsite, own), counter_of(rep1, c.g.nsite, own), two, own, own,
                 make_float2(c.beta[rep0], c.beta[rep1]), key, s, v, t, acc0, acc1);
}

// 1 when the plan's compile-time lattice table applies with the branch-free periodic wrap (every axis periodic,
// extents at least the table's reach), else 0 (fast_sweep.cu).
int spec_periodic_box(const sck_plan* plan);

// Segment kernels (segment.cu): eligibility and the task launch.
bool seg_kernel_ok(const sck_plan* plan);
int launch_seg_tasks(const sck_plan* plan, SpecParams& p, int ys, cudaStream_t s);

// Tile kernels (tile.cu): eligibility and one class over all replicas.
bool tile_kernel_ok(const sck_plan* plan);
int launch_tile_class(const sck_plan* plan, const Common& c, int colour, int alpha, cudaStream_t s);

}  // namespace sck
