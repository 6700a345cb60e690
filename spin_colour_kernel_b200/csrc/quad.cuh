// Interleaved storage for vector models (SCK_MODE_QUAD): parameter blocks shared by the host code (quad.cu) and the
// per-lattice kernel translation units (quad_<lattice>.cu), and, under SCK_QUAD_KERNELS, the class, pipeline and
// FP64 observables kernels with their launchers. Each lattice's kernels are instantiated in a file of its own so
// that they compile in parallel; quad.cu reaches them through quad_grid / quad_pipe / quad_obs.
//
//
// Layout. Replicas are stored four at a time: one float4 holds one spin component of one site for replicas
// 4q .. 4q + 3 (lane j = replica 4q + j). Within a quad the float4 elements are ordered
//     element(a, z, y, k, x) = (((a L3 + z) L2 + y) N + k) L1 + (x mod P) (L1 / P) + x / P
// with P the x-period of the colouring (1 or 2): every row of the lattice keeps its N components side by side,
// and each component row is split by x residue, so the sites one class owns in a row (all of one residue) are
// L1 / P consecutive float4s. A thread updates one class site of four replicas: every spin it reads or writes is
// one 16-byte load or store, a warp's loads of one neighbour row are contiguous, and the two float32x2 halves of
// a float4 go through the same packed-pair arithmetic (finish_values) as the lattice kernels of fast_sweep.cu,
// so the chain is identical to theirs. Philox counters stay keyed on the reference's site index.
#pragma once

#include "spec.cuh"

namespace sck {

struct QuadParams {
  Geometry g;
  Colouring col;
  FastDiv fd_m[SCK_MAX_FACTORS];
  FastDiv fd_hp, fd_L2;
  int hp;                // L1 / P: class sites of a row
  float J[SCK_MAX_BASIS][SCK_MAX_GROUPS];
  float h[3];
  int hnz[3];
  float k2;
  float4* spins;
  const float* k1;
  const float* beta;     // 4 per quad
  const int64_t* state;
  int colour, alpha, sweep_offset, q0;
  // measure sweeps (MEASURE kernels): the class's index in the sweep, the coupling groups whose bonds all reach
  // classes updated earlier in the sweep, per-block FP64 partial sums [replica][class][block][1 + N]
  int measure_ci, n_classes, blocks_x, B;
  unsigned lower_groups;
  double* partial;
};


// ------------------------------------------------------------------------------------------ L2 pipeline
// Class-by-class launches read the whole state once per class (every class's neighbours span the other classes)
// and write it once per sweep. The pipeline runs the classes of a group of quads back to back so that, after
// the group's first read from HBM, its later classes find it in L2: one launch carries a whole call. Blocks take
// tickets from a counter in the order they start. Units u = sweep-major groups; class ci of unit u sits at
// position D u + ci (D, the skew, divides the class count C), so each position holds C / D tasks and about
// C / D + 1 groups are in flight: D trades overlap between groups against the L2 working set. Within a position,
// tasks run in increasing class order; a task is T tickets (quads of the group x site blocks of a class). Before
// touching spins a block waits until every ticket of the task it follows has finished: class ci - 1 of its unit,
// or class C - 1 of the same group's previous sweep. That task sits at an earlier position, so its tickets were
// taken earlier by blocks that are running or done, and the wait ends. The waits poll with an iteration limit;
// a block whose wait gives up skips its sites, counts itself done (so nothing waits forever) and raises the
// plan's give-up flag, which sck_sweep reports as SCK_ERR_TIMEOUT.
struct QuadPipeParams {
  QuadParams p;
  int C, D, group, ngroups, units, sweep_base, T, Q, blocks_x;
  int cpt, tq;              // site blocks of 256 threads per ticket, tickets per quad and class (T = group tq)
  int cls[8][2];
  unsigned* ticket;
  unsigned* done;           // finished tickets per (group, class), summed over the launch's sweeps
  unsigned wait_limit;      // polls of a completion counter before giving up
  int* giveup;              // host-mapped flag, set (system scope) when a wait gives up
  // measure step: the launch's last sweep also writes FP64 partial sums [replica][class][ticket][1 + N]
  double* partial;
  unsigned lower_groups[8];
  int B;
};


// --------------------------------------------------------------------------------------- FP64 observables
// Per replica: E = -sum_bonds J s_i . s_j - h . sum s + sum anisotropy and M[alpha][k], each bond visited once
// from its forward end (as observables_spec_kernel of observables.cu), all in FP64. Grid (blocks per quad,
// quads); a thread walks sites of one sublattice at a time, keeping the four lanes' sums in registers; block
// sums go to partial[rep][block][value] for observables_finish.
struct QuadObsParams {
  Geometry g;
  SubObs obs[SCK_MAX_BASIS];
  double h64[3];
  double k2;
  int hp, blocks_per_quad, B;
  const float4* spins;
  const float* k1;
  double* partial;
};


// Launch one class of the launch's quads (grid: site blocks x quads), the pipeline (blocks tickets), or the FP64
// observables (grid: blocks per quad x quads) for lattice table Lat; defined in quad_<lattice>.cu.
template <class Lat>
void quad_grid(const sck_plan* plan, const QuadParams& p, dim3 grid, cudaStream_t s);
template <class Lat>
void quad_pipe(const sck_plan* plan, const QuadPipeParams& pp, unsigned blocks, cudaStream_t s);
template <class Lat>
void quad_obs(const sck_plan* plan, const QuadObsParams& p, dim3 grid, cudaStream_t s);

}  // namespace sck

#ifdef SCK_QUAD_KERNELS
namespace sck {

// Sums one thread adds to a measure sweep: per lane j, the site's energy share and its N components. The
// pipeline kernel adds several sites per thread in FP64 (T = double); a class launch has one site per thread and
// keeps its float32 values as they are (0 + x is exact) until the block sum converts them to FP64.
template <int N, class T = double>
struct MeasureAcc {
  T v[4][1 + N];
};

// Residue (0 .. P-1) along x of the class's sites in row (y, z) of the launch's sublattice, or -1 when the row
// holds none. The colour of a site is K c + o_alpha per factor (mixed radix); stepping x by one adds K[r][0].
template <int P>
__device__ __forceinline__ int class_residue(const QuadParams& p, int colour, int alpha, int y, int z) {
  int gr[SCK_MAX_FACTORS];
#pragma unroll
  for (int r = 0; r < SCK_MAX_FACTORS; ++r) {
    if (r < p.col.r) {
      const uint32_t v = (uint32_t)(p.col.K[r][1] * y + p.col.K[r][2] * z + p.col.o[alpha][r]);
      gr[r] = (int)(v - fdiv(v, p.fd_m[r]) * (uint32_t)p.col.m[r]);
    }
  }
#pragma unroll
  for (int q = 0; q < P; ++q) {
    int idx = 0;
#pragma unroll
    for (int r = 0; r < SCK_MAX_FACTORS; ++r) {
      if (r < p.col.r) {
        idx = idx * p.col.m[r] + gr[r];
        gr[r] += p.col.K[r][0];
        if (gr[r] >= p.col.m[r]) gr[r] -= p.col.m[r];
      }
    }
    if (idx == colour) return q;
  }
  return -1;
}

__device__ __forceinline__ int wrap_once(int v, int L) {
  v += v < 0 ? L : 0;
  v -= v >= L ? L : 0;
  return v;
}

// Compile-time box extents of a kernel instantiation: L1C > 0 fixes the row length L1; L1C < 0 fixes a cubic
// box of edge -L1C (a power of two: L1 = L2 = L3, so the y and z wraps are bit masks and every extent, plane
// and site count is a constant); 0 leaves everything to the runtime geometry.
template <int L1C>
struct QDim {
  static constexpr int E = L1C < 0 ? -L1C : L1C;
  static constexpr bool cube = L1C < 0;
  __device__ __forceinline__ static int L1(const Geometry& g) { return E ? E : g.L1; }
  __device__ __forceinline__ static int L2(const Geometry& g) { return cube ? E : g.L2; }
  __device__ __forceinline__ static int L3(const Geometry& g) { return cube ? E : g.L3; }
  // v in [-1, L]: one step outside the box at most
  __device__ __forceinline__ static int wrap_y(int v, const Geometry& g) {
    return cube ? (v & (E - 1)) : wrap_once(v, g.L2);
  }
  __device__ __forceinline__ static int wrap_z(int v, const Geometry& g) {
    return cube ? (v & (E - 1)) : wrap_once(v, g.L3);
  }
};

// Float4 offsets (within one quad) of the rows and row positions around a site: rowo[dz][dy] for offsets
// -R..R (periodic wrap), xo[dx] = the element of x + dx within its component row.
template <class Lat, int N, int P, int L1C>
struct QuadAround {
  static constexpr int R = Lat::reach;
  int rowo[2 * R + 1][2 * R + 1];
  int xo[2 * R + 1];
  int plane_a;   // elements of one sublattice

  __device__ __forceinline__ QuadAround(const Geometry& g, int hp, int h, int ph, int y, int z) {
    using D = QDim<L1C>;
    const int L1 = D::L1(g);
    const int HP = D::E ? D::E / P : hp;
    const int RS = N * L1;
    plane_a = D::L3(g) * D::L2(g) * RS;
#pragma unroll
    for (int dz = -R; dz <= R; ++dz) {
      const int zz = Lat::dim == 3 ? D::wrap_z(z + dz, g) : z;
#pragma unroll
      for (int dy = -R; dy <= R; ++dy) rowo[dz + R][dy + R] = (zz * D::L2(g) + D::wrap_y(y + dy, g)) * RS;
    }
#pragma unroll
    for (int dx = -R; dx <= R; ++dx) {
      const int s = ph + dx;
      int res, carry;
      if constexpr (P == 1) {
        res = 0;
        carry = s;
      } else {
        res = s & 1;                 // P = 2: floor division by 2 of -1 .. 2
        carry = s >> 1;
      }
      xo[dx + R] = res * HP + wrap_once(h + carry, HP);
    }
  }
  __device__ __forceinline__ int elem(const BondC b) const {
    return b.a2 * plane_a + rowo[b.dz + R][b.dy + R] + xo[b.dx + R];
  }
};

__device__ __forceinline__ float2 lo2(float4 v) { return make_float2(v.x, v.y); }
__device__ __forceinline__ float2 hi2(float4 v) { return make_float2(v.z, v.w); }

// One class site (row segment position h, residue ph, row (y, z), sublattice A) of the four replicas of quad q.
// MEASURE: also the site's share of the energy of the configuration the sweep leaves, -s'.(v_low + h) +
// anisotropy(s') with v_low the coupling-group fields of the neighbours updated earlier in the sweep (each bond
// is counted once, at its later endpoint, when both its spins are final), and its components s', added in FP64.
// NC: neighbour loads through the non-coherent read-only path, for kernels in which no neighbour is written (a
// class launch); the pipeline kernel, whose later tasks read what earlier tasks of the same launch wrote, keeps
// coherent loads. LOW: the class's lower coupling groups as a compile-time mask (-1: p.lower_groups at run time);
// when every group is lower the measure field is the Metropolis field itself and needs no registers of its own.
template <class Lat, int A, int N, int P, int L1C, bool MEASURE, bool NC = false, int LOW = -1, class Acc>
__device__ __forceinline__ void quad_site(const QuadParams& p, int q, int h, int ph, int y, int z, int32_t key,
                                          Acc& m) {
  const Geometry& g = p.g;
  using D = QDim<L1C>;
  const int L1 = D::L1(g);
  const int plane = D::cube ? D::E * D::E * D::E : g.plane;        // sites of one sublattice
  const int nsite = D::cube ? Lat::b * plane : g.nsite;
  float4* base = p.spins + (size_t)q * N * nsite;
  const QuadAround<Lat, N, P, L1C> nb(g, p.hp, h, ph, y, z);
  const int own_e = A * nb.plane_a + nb.rowo[Lat::reach][Lat::reach] + nb.xo[Lat::reach];
  const int x = h * P + ph;
  const int own = A * plane + (z * D::L2(g) + y) * L1 + x;    // the reference's site index (Philox counter)
  float4 s4[N];
#pragma unroll
  for (int k = 0; k < N; ++k) s4[k] = base[own_e + k * L1];
  constexpr bool kFullLow = LOW == (1 << Lat::groups) - 1;
  float2 vl[N], vh[N], wl[N], wh[N];
#pragma unroll
  for (int k = 0; k < N; ++k) vl[k] = vh[k] = wl[k] = wh[k] = f2(0.0f);
  static_for<0, Lat::groups>([&](auto gc) {
    constexpr int gi = decltype(gc)::value;
    using Rg = GroupRange<Lat, A, gi>;
    float2 gl[N], gh[N];
#pragma unroll
    for (int k = 0; k < N; ++k) gl[k] = gh[k] = f2(0.0f);
    static_for<Rg::begin, Rg::end>([&](auto ic) {
      constexpr BondC bd = Lat::bond(A, decltype(ic)::value);
      const float4* pq = base + nb.elem(bd);
#pragma unroll
      for (int k = 0; k < N; ++k) {
        const float4 t = NC ? __ldg(pq + k * L1) : pq[k * L1];
        gl[k] = __fadd2_rn(gl[k], lo2(t));
        gh[k] = __fadd2_rn(gh[k], hi2(t));
      }
    });
    const float2 J = f2(p.J[A][gi]);
#pragma unroll
    for (int k = 0; k < N; ++k) {
      vl[k] = __fadd2_rn(vl[k], __fmul2_rn(J, gl[k]));
      vh[k] = __fadd2_rn(vh[k], __fmul2_rn(J, gh[k]));
    }
    if constexpr (MEASURE && !kFullLow) {
      if (LOW >= 0 ? ((LOW >> gi) & 1) != 0 : ((p.lower_groups >> gi) & 1u) != 0) {
#pragma unroll
        for (int k = 0; k < N; ++k) {
          wl[k] = __fadd2_rn(wl[k], __fmul2_rn(J, gl[k]));
          wh[k] = __fadd2_rn(wh[k], __fmul2_rn(J, gh[k]));
        }
      }
    }
  });
#pragma unroll
  for (int k = 0; k < N; ++k)
    if (p.hnz[k]) {
      vl[k] = __fadd2_rn(vl[k], f2(p.h[k]));
      vh[k] = __fadd2_rn(vh[k], f2(p.h[k]));
      if constexpr (MEASURE && !kFullLow) {
        wl[k] = __fadd2_rn(wl[k], f2(p.h[k]));
        wh[k] = __fadd2_rn(wh[k], f2(p.h[k]));
      }
    }
  float2 sl[N], sh[N], tl[N], th[N];
#pragma unroll
  for (int k = 0; k < N; ++k) {
    sl[k] = lo2(s4[k]);
    sh[k] = hi2(s4[k]);
  }
  const bool cubic = N == 3 && g.has_cubic;
  const float k1 = cubic ? p.k1[own] : 0.0f;
  const float4 b4 = reinterpret_cast<const float4*>(p.beta)[q];
  const uint32_t c0 = counter_of(4 * q, nsite, own);
  const uint32_t ns = (uint32_t)nsite;
  bool a0, a1, a2, a3;
  // measure: the float32 energy share of each lane's final spin, -s'.w + anisotropy(s'), from the products of
  // both candidates, taken as soon as each pair's decision is known
  FinishMeasure fl, fh;
  auto share = [](bool acc, float es, float et, float as, float at) {
    return acc ? __fadd_rn(-et, at) : __fadd_rn(-es, as);
  };
  float2 el, eh;
  finish_values<N, MEASURE>(g.acceptance, cubic, f2(k1), p.k2, c0, c0 + ns, true, make_float2(b4.x, b4.y), key, sl,
                            vl, tl, a0, a1, kFullLow ? &vl : &wl, &fl);
  if constexpr (MEASURE)
    el = make_float2(share(a0, fl.es.x, fl.et.x, fl.as.x, fl.at.x), share(a1, fl.es.y, fl.et.y, fl.as.y, fl.at.y));
  finish_values<N, MEASURE>(g.acceptance, cubic, f2(k1), p.k2, c0 + 2 * ns, c0 + 3 * ns, true,
                            make_float2(b4.z, b4.w), key, sh, vh, th, a2, a3, kFullLow ? &vh : &wh, &fh);
  if constexpr (MEASURE)
    eh = make_float2(share(a2, fh.es.x, fh.et.x, fh.as.x, fh.at.x), share(a3, fh.es.y, fh.et.y, fh.as.y, fh.at.y));
  float4 n4[N];
#pragma unroll
  for (int k = 0; k < N; ++k)
    n4[k] = make_float4(a0 ? tl[k].x : s4[k].x, a1 ? tl[k].y : s4[k].y, a2 ? th[k].x : s4[k].z,
                        a3 ? th[k].y : s4[k].w);
  if (a0 | a1 | a2 | a3) {
#pragma unroll
    for (int k = 0; k < N; ++k) base[own_e + k * L1] = n4[k];
  }
  if constexpr (MEASURE) {
    // the lanes' shares and components
    m.v[0][0] += el.x;
    m.v[1][0] += el.y;
    m.v[2][0] += eh.x;
    m.v[3][0] += eh.y;
#pragma unroll
    for (int k = 0; k < N; ++k) {
      m.v[0][1 + k] += n4[k].x;
      m.v[1][1 + k] += n4[k].y;
      m.v[2][1 + k] += n4[k].z;
      m.v[3][1 + k] += n4[k].w;
    }
  }
}

template <int V>
__device__ __forceinline__ void block_sum(double (&x)[V], double (*red)[8]);

// FP64 warp sums of 8 values per lane by recursive halving: at offset o (16, 8, 4) each lane keeps one half of its
// remaining values, sends the other half to lane ^ o and adds what it receives; offsets 2 and 1 then add the single
// values of the lane groups. Lane l ends with the warp total of value (l >> 2) & 7, the same fixed binary tree of
// additions on every call.
__device__ __forceinline__ double warp_halving_sum8(double (&x)[8]) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 16, h = 4; o >= 4; o >>= 1, h >>= 1) {
    const bool hi = (lane & o) != 0;
#pragma unroll
    for (int i = 0; i < h; ++i) {
      const double keep = hi ? x[i + h] : x[i];
      const double send = hi ? x[i] : x[i + h];
      x[i] = keep + __shfl_xor_sync(0xFFFFFFFFu, send, o);
    }
  }
  x[0] += __shfl_xor_sync(0xFFFFFFFFu, x[0], 2);
  x[0] += __shfl_xor_sync(0xFFFFFFFFu, x[0], 1);
  return x[0];
}

// Measure-step epilogue of a block of 256 threads: the block totals of the (1 + N) values of each of the four
// lanes of a quad, in a fixed order (two warp halving sums, of lanes 0-1 and of lanes 2-3, each converting its
// eight values to FP64 only when it runs; then the 8 warps in order); thread v < 4 (1 + N) gets value v (lane
// v / (1 + N), component v % (1 + N)), the other threads 0. Every thread of the block must call it.
template <int N, class T>
__device__ __forceinline__ double measure_block_sum(const MeasureAcc<N, T>& m) {
  __shared__ double red[8][16];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int pass = 0; pass < 2; ++pass) {
    double x[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) x[i] = 0.0;
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
      for (int v = 0; v <= N; ++v) x[j * (1 + N) + v] = (double)m.v[2 * pass + j][v];
    const double t = warp_halving_sum8(x);
    if ((lane & 3) == 0) red[warp][pass * 8 + (lane >> 2)] = t;
  }
  __syncthreads();
  double v = 0.0;
  if (threadIdx.x < 4 * (1 + N)) {
    const int j = threadIdx.x / (1 + N), c = threadIdx.x - j * (1 + N);
    const int slot = (j >> 1) * 8 + (j & 1) * (1 + N) + c;
#pragma unroll
    for (int w = 0; w < 8; ++w) v += red[w][slot];
  }
  return v;
}

// Blocks of 256 threads per SM the class and pipeline kernels are compiled for (3: at most 85 registers).
#ifndef SCK_QUAD_MIN_BLOCKS
#define SCK_QUAD_MIN_BLOCKS 3
#endif
#ifndef SCK_QUAD_MEASURE_MIN_BLOCKS
#define SCK_QUAD_MEASURE_MIN_BLOCKS 3
#endif
#ifndef SCK_QUAD_CUBE_MEASURE_MIN_BLOCKS
#define SCK_QUAD_CUBE_MEASURE_MIN_BLOCKS 3
#endif

// Grid (ceil(L3 L2 L1 / P / 256), quads of this launch). Thread -> (row, position in the row's class segment).
// The cubic instantiations run four blocks per SM (64 registers): 78 against 77 attempts/ns at three on the 3D
// Heisenberg bcc J1-J2 workload.
// Measure kernels of the cubic boxes take the class's lower coupling groups as a compile-time mask LOW; the
// others read them at run time (LOW = -1). Both run three blocks per SM: at four (64 registers) the measure
// kernels spill 140-244 bytes a thread, and a measure sweep of the 3D Heisenberg bcc J1-J2 workload ran at 60
// attempts/ns against 64 at three (12-44 bytes).
template <class Lat, int N, int P, int L1C, bool MEASURE, int LOW = -1>
__global__ void __launch_bounds__(256, MEASURE ? (LOW >= 0 ? SCK_QUAD_CUBE_MEASURE_MIN_BLOCKS
                                                            : SCK_QUAD_MEASURE_MIN_BLOCKS)
                                               : (L1C < 0 ? 4 : SCK_QUAD_MIN_BLOCKS))
    quad_class_kernel(const __grid_constant__ QuadParams p) {
  const Geometry& g = p.g;
  using D = QDim<L1C>;
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t row, h;
  if constexpr (D::cube && D::E / P == 32) {
    // a cubic box with 32 class sites per row: a block takes 2 rows of 4 planes (neighbour rows shared in L1)
    const uint32_t tile = blockIdx.x, lz = threadIdx.x >> 6, ly = (threadIdx.x >> 5) & 1;
    h = threadIdx.x & 31;
    row = ((tile / (D::E / 2)) * 4 + lz) * D::E + (tile % (D::E / 2)) * 2 + ly;
  } else if constexpr (D::E > 0) {
    row = t / (uint32_t)(D::E / P);
    h = t - row * (uint32_t)(D::E / P);
  } else {
    row = fdiv(t, p.fd_hp);
    h = t - row * (uint32_t)p.hp;
  }
  const int q = p.q0 + (int)blockIdx.y;
  MeasureAcc<N, float> m;
  if constexpr (MEASURE) {
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int v = 0; v <= N; ++v) m.v[j][v] = 0.0f;
  }
  if (row < (uint32_t)(D::L3(g) * D::L2(g))) {
    const int z = D::cube ? (int)(row / (uint32_t)D::E) : (int)fdiv(row, p.fd_L2);
    const int y = (int)row - z * D::L2(g);
    const int ph = class_residue<P>(p, p.colour, p.alpha, y, z);
    if (ph >= 0) {
      const int32_t key = sweep_key_at(p.state, p.sweep_offset);
      static_for<0, Lat::b>([&](auto ac) {
        constexpr int a = decltype(ac)::value;
        if (a == p.alpha) quad_site<Lat, a, N, P, L1C, MEASURE, true, LOW>(p, q, (int)h, ph, y, z, key, m);
      });
    }
  }
  if constexpr (MEASURE) {
    // every thread of the block reaches here: block sums in a fixed order, one partial per (replica, value)
    const double val = measure_block_sum(m);
    if (threadIdx.x < 4 * (1 + N)) {
      const int j = threadIdx.x / (1 + N), v = threadIdx.x - j * (1 + N);
      const int rep = 4 * q + j;
      if (rep < p.B)
        p.partial[(((size_t)rep * p.n_classes + p.measure_ci) * p.blocks_x + blockIdx.x) * (1 + N) + v] = val;
    }
  }
}


// ------------------------------------------------------------------------------------------ L2 pipeline
__device__ __forceinline__ unsigned ld_acquire_gpu(const unsigned* a) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(a) : "memory");
  return v;
}

struct PipeTask {
  int go, has, q, ci, sweep, done_idx, chunk;
};

template <class Lat, int N, int P, int L1C, bool MEASURE>
__global__ void __launch_bounds__(256, SCK_QUAD_MIN_BLOCKS) quad_pipe_kernel(const __grid_constant__ QuadPipeParams pp) {
  __shared__ PipeTask s;
  if (threadIdx.x == 0) {
    const unsigned tk = atomicAdd(pp.ticket, 1u);
    const unsigned per_pos = (unsigned)(pp.C / pp.D) * (unsigned)pp.T;
    const unsigned pos = tk / per_pos;
    const unsigned rem = tk - pos * per_pos;
    const int i = (int)(rem / (unsigned)pp.T), j = (int)(rem - (unsigned)i * (unsigned)pp.T);
    const int ci = (int)(pos % (unsigned)pp.D) + i * pp.D;
    const int num = (int)pos - ci;
    s.has = 0;
    s.go = 0;
    if (num >= 0 && num / pp.D < pp.units) {
      const int u = num / pp.D;
      const int sw = u / pp.ngroups, g = u - sw * pp.ngroups;
      const int qi = j / pp.tq;
      s.has = 1;
      s.q = g * pp.group + qi;
      s.chunk = j - qi * pp.tq;
      s.ci = ci;
      s.sweep = pp.sweep_base + sw;
      s.done_idx = g * pp.C + ci;
      const unsigned* dep = nullptr;
      unsigned need = 0;
      if (ci > 0) {
        dep = pp.done + s.done_idx - 1;
        need = (unsigned)(sw + 1) * (unsigned)pp.T;
      } else if (sw > 0) {
        dep = pp.done + g * pp.C + pp.C - 1;
        need = (unsigned)sw * (unsigned)pp.T;
      }
      int go = 1;
      if (dep != nullptr) {
        unsigned polls = 0;
        while (ld_acquire_gpu(dep) < need) {
          if (++polls > pp.wait_limit) {
            go = 0;
            atomicExch_system(pp.giveup, 1);
            break;
          }
          __nanosleep(64);
        }
      }
      s.go = go && s.q < pp.Q;
    }
  }
  __syncthreads();
  if (!s.has) return;                                   // the pipeline's fill and drain: no task
  // the measure step's partial sums: the launch's last sweep only (a block-uniform condition)
  const bool measuring = MEASURE && s.sweep == pp.sweep_base + pp.units / pp.ngroups - 1;
  MeasureAcc<N> m;
  if constexpr (MEASURE) {
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int v = 0; v <= N; ++v) m.v[j][v] = 0.0;
  }
  if (s.go) {
    const QuadParams& p = pp.p;
    const Geometry& g = p.g;
#pragma unroll 1
    for (int c = 0; c < pp.cpt; ++c) {
    const int chunk = s.chunk * pp.cpt + c;
    if (chunk >= pp.blocks_x) break;
    const uint32_t t = (uint32_t)chunk * 256u + threadIdx.x;
    uint32_t row, h;
    if constexpr (QDim<L1C>::E > 0) {
      row = t / (uint32_t)(QDim<L1C>::E / P);
      h = t - row * (uint32_t)(QDim<L1C>::E / P);
    } else {
      row = fdiv(t, p.fd_hp);
      h = t - row * (uint32_t)p.hp;
    }
    if (row < (uint32_t)(g.L3 * g.L2)) {
      const int colour = pp.cls[s.ci][0], alpha = pp.cls[s.ci][1];
      const int z = (int)fdiv(row, p.fd_L2);
      const int y = (int)row - z * g.L2;
      const int ph = class_residue<P>(p, colour, alpha, y, z);
      if (ph >= 0) {
        const int32_t key = sweep_key_at(p.state, s.sweep);
        static_for<0, Lat::b>([&](auto ac) {
          constexpr int a = decltype(ac)::value;
          if (a == alpha) {
            if (measuring) {
              QuadParams pm = p;
              pm.lower_groups = pp.lower_groups[s.ci];
              quad_site<Lat, a, N, P, L1C, MEASURE>(pm, s.q, (int)h, ph, y, z, key, m);
            } else {
              quad_site<Lat, a, N, P, L1C, false>(p, s.q, (int)h, ph, y, z, key, m);
            }
          }
        });
      }
    }
    }
  }
  if constexpr (MEASURE) {
    if (measuring) {
      const double val = measure_block_sum(m);
      if (threadIdx.x < 4 * (1 + N) && s.q < pp.Q) {
        const int j = threadIdx.x / (1 + N), v = threadIdx.x - j * (1 + N);
        const int rep = 4 * s.q + j;
        if (rep < pp.B) pp.partial[(((size_t)rep * pp.C + s.ci) * pp.tq + s.chunk) * (1 + N) + v] = val;
      }
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    // finished (or given up): later tasks of this group may start. The barrier orders every thread's stores
    // before this release (cumulativity), so a block that acquires the count sees them.
    asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(pp.done + s.done_idx) : "memory");
  }
}


template <int V>
__device__ __forceinline__ void block_sum(double (&x)[V], double (*red)[8]) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int i = 0; i < V; ++i) {
    double v = x[i];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xFFFFFFFFu, v, off);
    if (lane == 0) red[i][warp] = v;
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < V; ++i) {
    double v = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) v += red[i][w];
    x[i] = v;
  }
  __syncthreads();
}

template <class Lat, int N, int P>
__global__ void __launch_bounds__(256) quad_observables_kernel(const __grid_constant__ QuadObsParams p) {
  const Geometry& g = p.g;
  const int q = blockIdx.y;
  const float4* base = p.spins + (size_t)q * N * g.nsite;
  const int per_a = g.L3 * g.L2 * g.L1;   // sites of one sublattice
  __shared__ double red[4 * (1 + N)][8];
  double E[4] = {0.0, 0.0, 0.0, 0.0};
  static_for<0, Lat::b>([&](auto ac) {
    constexpr int A = decltype(ac)::value;
    double acc[4 * (1 + N)];
#pragma unroll
    for (int i = 0; i < 4 * (1 + N); ++i) acc[i] = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < per_a; i += p.blocks_per_quad * blockDim.x) {
      // i runs over (z, y, storage position) so that a warp reads consecutive float4s of a component row
      const int row = i / g.L1, xs = i - row * g.L1;
      const int z = row / g.L2, y = row - z * g.L2;
      const int res = xs / p.hp, h = xs - res * p.hp;
      const int x = h * P + res;
      const QuadAround<Lat, N, P, 0> nb(g, p.hp, h, res, y, z);
      const int own_e = A * nb.plane_a + nb.rowo[Lat::reach][Lat::reach] + nb.xo[Lat::reach];
      double s[4][N];
#pragma unroll
      for (int k = 0; k < N; ++k) {
        const float4 v = base[own_e + k * g.L1];
        s[0][k] = v.x;
        s[1][k] = v.y;
        s[2][k] = v.z;
        s[3][k] = v.w;
      }
      double e[4] = {0.0, 0.0, 0.0, 0.0};
      static_for<0, Lat::n_bonds(A)>([&](auto ic) {
        constexpr int bi = decltype(ic)::value;
        if constexpr (forward_bond<Lat, A>(bi)) {
          constexpr BondC bd = Lat::bond(A, bi);
          const float4* pq = base + nb.elem(bd);
          double dot[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
          for (int k = 0; k < N; ++k) {
            const float4 t = pq[k * g.L1];
            dot[0] += s[0][k] * (double)t.x;
            dot[1] += s[1][k] * (double)t.y;
            dot[2] += s[2][k] * (double)t.z;
            dot[3] += s[3][k] * (double)t.w;
          }
          const double J = p.obs[A].J[bi];
#pragma unroll
          for (int j = 0; j < 4; ++j) e[j] -= J * dot[j];
        }
      });
      const double k1 = (N == 3 && g.has_cubic) ? (double)p.k1[A * per_a + (z * g.L2 + y) * g.L1 + x] : 0.0;
#pragma unroll
      for (int j = 0; j < 4; ++j) {
#pragma unroll
        for (int k = 0; k < N; ++k) e[j] -= p.h64[k] * s[j][k];
        if constexpr (N == 3) {
          if (g.has_cubic) {
            const double xy = s[j][0] * s[j][1], xz = s[j][0] * s[j][2], yz = s[j][1] * s[j][2];
            const double xyz = s[j][0] * s[j][1] * s[j][2];
            e[j] += k1 * (xy * xy + xz * xz + yz * yz) + p.k2 * xyz * xyz;
          }
        }
        acc[j * (1 + N)] += e[j];
#pragma unroll
        for (int k = 0; k < N; ++k) acc[j * (1 + N) + 1 + k] += s[j][k];
      }
    }
    block_sum<4 * (1 + N)>(acc, red);
    if (threadIdx.x == 0) {
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        E[j] += acc[j * (1 + N)];
        const int rep = 4 * q + j;
        if (rep < p.B) {
          double* out = p.partial + ((size_t)rep * p.blocks_per_quad + blockIdx.x) * OBS_VALUES;
#pragma unroll
          for (int k = 0; k < N; ++k) out[1 + A * N + k] = acc[j * (1 + N) + 1 + k];
        }
      }
    }
  });
  if (threadIdx.x == 0) {
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int rep = 4 * q + j;
      if (rep < p.B) p.partial[((size_t)rep * p.blocks_per_quad + blockIdx.x) * OBS_VALUES] = E[j];
    }
  }
}


// ------------------------------------------------------------------------------------------- launchers
// Measure launch with the compile-time mask of p.lower_groups, tried from LOW down to 0 (-1: the run-time mask).
template <class Lat, int N, int P, int L1C, int LOW>
inline void launch_measure_low(const QuadParams& p, dim3 grid, cudaStream_t s) {
  if constexpr (LOW < 0) {
    quad_class_kernel<Lat, N, P, L1C, true, -1><<<grid, 256, 0, s>>>(p);
  } else {
    if (p.lower_groups == (unsigned)LOW) quad_class_kernel<Lat, N, P, L1C, true, LOW><<<grid, 256, 0, s>>>(p);
    else launch_measure_low<Lat, N, P, L1C, LOW - 1>(p, grid, s);
  }
}

template <class Lat, int N, int P, int L1C>
inline void launch_quad_t(const QuadParams& p, dim3 grid, cudaStream_t s) {
  if (p.partial != nullptr) {
    if constexpr (L1C < 0 && N == 3) launch_measure_low<Lat, N, P, L1C, (1 << Lat::groups) - 1>(p, grid, s);
    else quad_class_kernel<Lat, N, P, L1C, true><<<grid, 256, 0, s>>>(p);
  } else {
    quad_class_kernel<Lat, N, P, L1C, false><<<grid, 256, 0, s>>>(p);
  }
}

template <class Lat, int N, int P>
inline void launch_quad_l1(const QuadParams& p, dim3 grid, cudaStream_t s) {
  if constexpr (Lat::dim == 3) {
    if (p.g.L1 == 64 && p.g.L2 == 64 && p.g.L3 == 64) return launch_quad_t<Lat, N, P, -64>(p, grid, s);
  }
  if (p.g.L1 == 64) return launch_quad_t<Lat, N, P, 64>(p, grid, s);
  if (p.g.L1 == 32) return launch_quad_t<Lat, N, P, 32>(p, grid, s);
  if (p.g.L1 == 128) return launch_quad_t<Lat, N, P, 128>(p, grid, s);
  launch_quad_t<Lat, N, P, 0>(p, grid, s);
}

template <class Lat, int N>
inline void launch_quad_p(const sck_plan* plan, const QuadParams& p, dim3 grid, cudaStream_t s) {
  if (plan->P == 1) launch_quad_l1<Lat, N, 1>(p, grid, s);
  else launch_quad_l1<Lat, N, 2>(p, grid, s);
}

template <class Lat>
inline void launch_quad_n(const sck_plan* plan, const QuadParams& p, dim3 grid, cudaStream_t s) {
  if (plan->geom.n == 2) launch_quad_p<Lat, 2>(plan, p, grid, s);
  else launch_quad_p<Lat, 3>(plan, p, grid, s);
}


template <class Lat, int N>
inline void launch_qobs_n(const sck_plan* plan, const QuadObsParams& p, dim3 grid, cudaStream_t s) {
  if (plan->P == 1) quad_observables_kernel<Lat, N, 1><<<grid, 256, 0, s>>>(p);
  else quad_observables_kernel<Lat, N, 2><<<grid, 256, 0, s>>>(p);
}

template <class Lat>
inline void launch_qobs(const sck_plan* plan, const QuadObsParams& p, dim3 grid, cudaStream_t s) {
  if (plan->geom.n == 2) launch_qobs_n<Lat, 2>(plan, p, grid, s);
  else launch_qobs_n<Lat, 3>(plan, p, grid, s);
}

// FP64 observables of the first `batch` replicas of interleaved storage; `workspace` holds
// batch x quad_obs_blocks x OBS_VALUES doubles.

template <class Lat, int N, int P, int L1C>
inline void launch_pipe_t(const QuadPipeParams& pp, unsigned blocks, cudaStream_t s) {
  if (pp.partial != nullptr)
    quad_pipe_kernel<Lat, N, P, L1C, true><<<blocks, 256, 0, s>>>(pp);
  else
    quad_pipe_kernel<Lat, N, P, L1C, false><<<blocks, 256, 0, s>>>(pp);
}

template <class Lat, int N, int P>
inline void launch_pipe_l1(const QuadPipeParams& pp, unsigned blocks, cudaStream_t s) {
  if (pp.p.g.L1 == 64) launch_pipe_t<Lat, N, P, 64>(pp, blocks, s);
  else if (pp.p.g.L1 == 32) launch_pipe_t<Lat, N, P, 32>(pp, blocks, s);
  else if (pp.p.g.L1 == 128) launch_pipe_t<Lat, N, P, 128>(pp, blocks, s);
  else launch_pipe_t<Lat, N, P, 0>(pp, blocks, s);
}

template <class Lat>
inline void launch_pipe_lat(const sck_plan* plan, const QuadPipeParams& pp, unsigned blocks, cudaStream_t s) {
  if (plan->geom.n == 2) {
    if (plan->P == 1) launch_pipe_l1<Lat, 2, 1>(pp, blocks, s);
    else launch_pipe_l1<Lat, 2, 2>(pp, blocks, s);
  } else {
    if (plan->P == 1) launch_pipe_l1<Lat, 3, 1>(pp, blocks, s);
    else launch_pipe_l1<Lat, 3, 2>(pp, blocks, s);
  }
}

// n sweeps of the pipeline (one launch per chunk of sweeps that keeps the ticket count below 2^30); state[1] is
// advanced by the caller. The counters are zeroed before every launch. With `partial` (a measure step, which
// needs quad_measure_fused), the last sweep also writes the measure sweep's partial sums.

template <class Lat>
void quad_grid(const sck_plan* plan, const QuadParams& p, dim3 grid, cudaStream_t s) {
  launch_quad_n<Lat>(plan, p, grid, s);
}
template <class Lat>
void quad_pipe(const sck_plan* plan, const QuadPipeParams& pp, unsigned blocks, cudaStream_t s) {
  launch_pipe_lat<Lat>(plan, pp, blocks, s);
}
template <class Lat>
void quad_obs(const sck_plan* plan, const QuadObsParams& p, dim3 grid, cudaStream_t s) {
  launch_qobs<Lat>(plan, p, grid, s);
}

}  // namespace sck

#define SCK_QUAD_INSTANTIATE(LAT)                                                                        \
  namespace sck {                                                                                          \
  template void quad_grid<LAT>(const sck_plan*, const QuadParams&, dim3, cudaStream_t);                    \
  template void quad_pipe<LAT>(const sck_plan*, const QuadPipeParams&, unsigned, cudaStream_t);            \
  template void quad_obs<LAT>(const sck_plan*, const QuadObsParams&, dim3, cudaStream_t);                  \
  }
#endif
