// Interleaved storage for vector models (SCK_MODE_QUAD) and its class kernels, layout conversions and FP64
// observables.
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
#include <string.h>

#include <string>

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

// FP64 sums one thread adds to a measure sweep: per lane j, the site's energy share and its N components.
template <int N>
struct MeasureAcc {
  double v[4][1 + N];
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

// Float4 offsets (within one quad) of the rows and row positions around a site: rowo[dz][dy] for offsets
// -R..R (periodic wrap), xo[dx] = the element of x + dx within its component row.
template <class Lat, int N, int P, int L1C>
struct QuadAround {
  static constexpr int R = Lat::reach;
  int rowo[2 * R + 1][2 * R + 1];
  int xo[2 * R + 1];
  int plane_a;   // elements of one sublattice

  __device__ __forceinline__ QuadAround(const Geometry& g, int hp, int h, int ph, int y, int z) {
    const int L1 = L1C ? L1C : g.L1;
    const int HP = L1C ? L1C / P : hp;
    const int RS = N * L1;
    plane_a = g.L3 * g.L2 * RS;
#pragma unroll
    for (int dz = -R; dz <= R; ++dz) {
      const int zz = Lat::dim == 3 ? wrap_once(z + dz, g.L3) : z;
#pragma unroll
      for (int dy = -R; dy <= R; ++dy) rowo[dz + R][dy + R] = (zz * g.L2 + wrap_once(y + dy, g.L2)) * RS;
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
// MEASURE: also the site's share of the energy of the configuration the sweep leaves, -s'.v_low - h.s' +
// anisotropy(s') with v_low the coupling-group fields of the neighbours updated earlier in the sweep (each bond
// is counted once, at its later endpoint, when both its spins are final), and its components s', added in FP64.
template <class Lat, int A, int N, int P, int L1C, bool MEASURE>
__device__ __forceinline__ void quad_site(const QuadParams& p, int q, int h, int ph, int y, int z, int32_t key,
                                          MeasureAcc<N>& m) {
  const Geometry& g = p.g;
  const int L1 = L1C ? L1C : g.L1;
  float4* base = p.spins + (size_t)q * N * g.nsite;
  const QuadAround<Lat, N, P, L1C> nb(g, p.hp, h, ph, y, z);
  const int own_e = A * nb.plane_a + nb.rowo[Lat::reach][Lat::reach] + nb.xo[Lat::reach];
  const int x = h * P + ph;
  const int own = A * g.plane + (z * g.L2 + y) * g.L1 + x;    // the reference's site index (Philox counter)
  float4 s4[N];
#pragma unroll
  for (int k = 0; k < N; ++k) s4[k] = base[own_e + k * L1];
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
        const float4 t = pq[k * L1];
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
    if constexpr (MEASURE) {
      if ((p.lower_groups >> gi) & 1u) {
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
  const uint32_t c0 = counter_of(4 * q, g.nsite, own);
  const uint32_t ns = (uint32_t)g.nsite;
  bool a0, a1, a2, a3;
  finish_values<N>(g.acceptance, cubic, f2(k1), p.k2, c0, c0 + ns, true, make_float2(b4.x, b4.y), key, sl, vl, tl,
                   a0, a1);
  finish_values<N>(g.acceptance, cubic, f2(k1), p.k2, c0 + 2 * ns, c0 + 3 * ns, true, make_float2(b4.z, b4.w), key,
                   sh, vh, th, a2, a3);
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
    // float32 share of the site in each lane, then FP64 sums
    auto share = [&](float2 n0, float2 n1, float2 n2, const float2 (&w)[N]) {
      const float2 nn[3] = {n0, n1, n2};
      float2 bond = __fmul2_rn(nn[0], w[0]);
#pragma unroll
      for (int k = 1; k < N; ++k) bond = __fadd2_rn(bond, __fmul2_rn(nn[k], w[k]));
      float2 e = make_float2(-bond.x, -bond.y);
#pragma unroll
      for (int k = 0; k < N; ++k)
        if (p.hnz[k]) e = __fadd2_rn(e, __fmul2_rn(f2(-p.h[k]), nn[k]));
      if (cubic) {
        const float2 q01 = __fmul2_rn(nn[0], nn[1]), q02 = __fmul2_rn(nn[0], nn[2]), q12 = __fmul2_rn(nn[1], nn[2]);
        const float2 tri = __fmul2_rn(q01, nn[2]);
        const float2 quad = __fadd2_rn(__fadd2_rn(__fmul2_rn(q01, q01), __fmul2_rn(q02, q02)), __fmul2_rn(q12, q12));
        e = __fadd2_rn(e, __fadd2_rn(__fmul2_rn(f2(k1), quad), __fmul2_rn(__fmul2_rn(f2(p.k2), tri), tri)));
      }
      return e;
    };
    const float2 el = share(lo2(n4[0]), lo2(n4[1 % N]), N == 3 ? lo2(n4[2 % N]) : f2(0.0f), wl);
    const float2 eh = share(hi2(n4[0]), hi2(n4[1 % N]), N == 3 ? hi2(n4[2 % N]) : f2(0.0f), wh);
    m.v[0][0] += (double)el.x;
    m.v[1][0] += (double)el.y;
    m.v[2][0] += (double)eh.x;
    m.v[3][0] += (double)eh.y;
#pragma unroll
    for (int k = 0; k < N; ++k) {
      m.v[0][1 + k] += (double)n4[k].x;
      m.v[1][1 + k] += (double)n4[k].y;
      m.v[2][1 + k] += (double)n4[k].z;
      m.v[3][1 + k] += (double)n4[k].w;
    }
  }
}

template <int V>
__device__ __forceinline__ void block_sum(double (&x)[V], double (*red)[8]);

// Grid (ceil(L3 L2 L1 / P / 256), quads of this launch). Thread -> (row, position in the row's class segment).
// At most 85 registers (three blocks of 256 threads per SM) for the sweep; 128 for measure launches.
template <class Lat, int N, int P, int L1C, bool MEASURE>
__global__ void __launch_bounds__(256, MEASURE ? 2 : 3) quad_class_kernel(const __grid_constant__ QuadParams p) {
  const Geometry& g = p.g;
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t row, h;
  if constexpr (L1C > 0) {
    row = t / (uint32_t)(L1C / P);
    h = t - row * (uint32_t)(L1C / P);
  } else {
    row = fdiv(t, p.fd_hp);
    h = t - row * (uint32_t)p.hp;
  }
  const int q = p.q0 + (int)blockIdx.y;
  MeasureAcc<N> m;
  if constexpr (MEASURE) {
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int v = 0; v <= N; ++v) m.v[j][v] = 0.0;
  }
  if (row < (uint32_t)(g.L3 * g.L2)) {
    const int z = (int)fdiv(row, p.fd_L2);
    const int y = (int)row - z * g.L2;
    const int ph = class_residue<P>(p, p.colour, p.alpha, y, z);
    if (ph >= 0) {
      const int32_t key = sweep_key_at(p.state, p.sweep_offset);
      static_for<0, Lat::b>([&](auto ac) {
        constexpr int a = decltype(ac)::value;
        if (a == p.alpha) quad_site<Lat, a, N, P, L1C, MEASURE>(p, q, (int)h, ph, y, z, key, m);
      });
    }
  }
  if constexpr (MEASURE) {
    // every thread of the block reaches here: block sums in a fixed order, one partial per (replica, value)
    __shared__ double red[4 * (1 + N)][8];
    double x[4 * (1 + N)];
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int v = 0; v <= N; ++v) x[j * (1 + N) + v] = m.v[j][v];
    block_sum<4 * (1 + N)>(x, red);
    if (threadIdx.x < 4 * (1 + N)) {
      const int j = threadIdx.x / (1 + N), v = threadIdx.x - j * (1 + N);
      const int rep = 4 * q + j;
      if (rep < p.B) {
        double val = 0.0;
#pragma unroll
        for (int i = 0; i < 4 * (1 + N); ++i)
          if (i == (int)threadIdx.x) val = x[i];
        p.partial[(((size_t)rep * p.n_classes + p.measure_ci) * p.blocks_x + blockIdx.x) * (1 + N) + v] = val;
      }
    }
  }
}

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
  int cls[8][2];
  unsigned* ticket;
  unsigned* done;           // finished tickets per (group, class), summed over the launch's sweeps
  unsigned wait_limit;      // polls of a completion counter before giving up
  int* giveup;              // host-mapped flag, set (system scope) when a wait gives up
  // measure step: the launch's last sweep also writes FP64 partial sums [replica][class][site block][1 + N]
  double* partial;
  unsigned lower_groups[8];
  int B;
};

__device__ __forceinline__ unsigned ld_acquire_gpu(const unsigned* a) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(a) : "memory");
  return v;
}

struct PipeTask {
  int go, has, q, ci, sweep, done_idx, chunk;
};

template <class Lat, int N, int P, int L1C, bool MEASURE>
__global__ void __launch_bounds__(256, MEASURE ? 2 : 3) quad_pipe_kernel(const __grid_constant__ QuadPipeParams pp) {
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
      const int qi = j / pp.blocks_x;
      s.has = 1;
      s.q = g * pp.group + qi;
      s.chunk = j - qi * pp.blocks_x;
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
    const uint32_t t = (uint32_t)s.chunk * 256u + threadIdx.x;
    uint32_t row, h;
    if constexpr (L1C > 0) {
      row = t / (uint32_t)(L1C / P);
      h = t - row * (uint32_t)(L1C / P);
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
  if constexpr (MEASURE) {
    if (measuring) {
      __shared__ double red[4 * (1 + N)][8];
      double x[4 * (1 + N)];
#pragma unroll
      for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int v = 0; v <= N; ++v) x[j * (1 + N) + v] = m.v[j][v];
      block_sum<4 * (1 + N)>(x, red);
      if (threadIdx.x < 4 * (1 + N) && s.q < pp.Q) {
        const int j = threadIdx.x / (1 + N), v = threadIdx.x - j * (1 + N);
        const int rep = 4 * s.q + j;
        if (rep < pp.B) {
          double val = 0.0;
#pragma unroll
          for (int i = 0; i < 4 * (1 + N); ++i)
            if (i == (int)threadIdx.x) val = x[i];
          pp.partial[(((size_t)rep * pp.C + s.ci) * pp.blocks_x + s.chunk) * (1 + N) + v] = val;
        }
      }
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    atomicAdd(pp.done + s.done_idx, 1u);   // finished (or given up): later tasks of this group may start
  }
}

// ------------------------------------------------------------------------------------------ layout changes
__device__ __forceinline__ void quad_coords(uint32_t e, const Geometry& g, int hp, int P, int& a, int& z, int& y,
                                            int& k, int& x) {
  // e = element index within a quad: (((a L3 + z) L2 + y) N + k) L1 + xs
  const int xs = (int)(e % (uint32_t)g.L1);
  uint32_t r = e / (uint32_t)g.L1;
  k = (int)(r % (uint32_t)g.n);
  r /= (uint32_t)g.n;
  y = (int)(r % (uint32_t)g.L2);
  r /= (uint32_t)g.L2;
  z = (int)(r % (uint32_t)g.L3);
  a = (int)(r / (uint32_t)g.L3);
  const int res = xs / hp;
  x = (xs - res * hp) * P + res;
}

// float32 S[B][N][b][L3][L2][L1] -> quads (lanes of replicas >= B are zero). Grid (element blocks, quads).
__global__ void quad_pack_kernel(const float* __restrict__ src, float4* __restrict__ dst, Geometry g, int hp, int P,
                                 int B) {
  const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t per = (uint32_t)g.n * (uint32_t)g.nsite;
  if (e >= per) return;
  const int q = blockIdx.y;
  int a, z, y, k, x;
  quad_coords(e, g, hp, P, a, z, y, k, x);
  const size_t site = (size_t)a * g.plane + ((size_t)z * g.L2 + y) * g.L1 + x;
  float v[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int rep = 4 * q + j;
    v[j] = rep < B ? src[((size_t)rep * g.n + k) * g.nsite + site] : 0.0f;
  }
  dst[(size_t)q * per + e] = make_float4(v[0], v[1], v[2], v[3]);
}

__global__ void quad_unpack_kernel(const float4* __restrict__ src, float* __restrict__ dst, Geometry g, int hp, int P,
                                   int B) {
  const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t per = (uint32_t)g.n * (uint32_t)g.nsite;
  if (e >= per) return;
  const int q = blockIdx.y;
  int a, z, y, k, x;
  quad_coords(e, g, hp, P, a, z, y, k, x);
  const size_t site = (size_t)a * g.plane + ((size_t)z * g.L2 + y) * g.L1 + x;
  const float4 v = src[(size_t)q * per + e];
  const float w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int rep = 4 * q + j;
    if (rep < B) dst[((size_t)rep * g.n + k) * g.nsite + site] = w[j];
  }
}

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

// --------------------------------------------------------------------------------------------- host side
static int quad_period(const sck_plan* plan) { return plan->P; }

// The systems the interleaved kernels serve: vector models with a compile-time lattice table, every axis
// periodic, no mask, a colouring of x-period 1 or 2 that divides L1.
bool quad_ok(const sck_plan* plan, std::string* why) {
  auto no = [&](const char* m) {
    if (why) *why = m;
    return false;
  };
  const Geometry& g = plan->geom;
  if (g.n < 2) return no("interleaved storage is for vector models (n = 2 or 3)");
  if (find_spec(plan) == 0)
    return no("interleaved storage needs a crystal with a compile-time bond table (square, triangular, sc, bcc, "
              "bcc J1-J2, fcc) and no extra bond matrices");
  if (g.has_mask) return no("interleaved storage does not take a site mask");
  if (!g.per[0] || !g.per[1] || (g.dim == 3 && !g.per[2])) return no("interleaved storage needs a periodic box");
  if (plan->P != 1 && plan->P != 2) return no("interleaved storage needs a colouring of x-period 1 or 2");
  if (g.L1 % plan->P != 0) return no("the colouring's x-period must divide L1");
  return true;
}

static QuadParams quad_params(const sck_plan* plan, const sck_buffers* buf, int colour, int alpha) {
  QuadParams p;
  memset(&p, 0, sizeof(p));
  p.g = plan->geom;
  p.col = plan->col;
  for (int r = 0; r < SCK_MAX_FACTORS; ++r) p.fd_m[r] = make_fastdiv((uint32_t)plan->col.m[r]);
  p.hp = plan->geom.L1 / quad_period(plan);
  p.fd_hp = make_fastdiv((uint32_t)p.hp);
  p.fd_L2 = make_fastdiv((uint32_t)plan->geom.L2);
  for (int a = 0; a < SCK_MAX_BASIS; ++a)
    for (int gi = 0; gi < SCK_MAX_GROUPS; ++gi) p.J[a][gi] = plan->sub[a].J[gi];
  for (int k = 0; k < 3; ++k) {
    p.h[k] = plan->desc.h[k];
    p.hnz[k] = (k < plan->geom.n && plan->desc.h[k] != 0.0f) ? 1 : 0;
  }
  p.k2 = plan->desc.k2;
  p.spins = (float4*)buf->spins;
  p.k1 = buf->k1;
  p.beta = buf->beta;
  p.state = buf->state;
  p.colour = colour;
  p.alpha = alpha;
  return p;
}

template <class Lat, int N, int P, int L1C>
static void launch_quad_t(const QuadParams& p, dim3 grid, cudaStream_t s) {
  if (p.partial != nullptr)
    quad_class_kernel<Lat, N, P, L1C, true><<<grid, 256, 0, s>>>(p);
  else
    quad_class_kernel<Lat, N, P, L1C, false><<<grid, 256, 0, s>>>(p);
}

template <class Lat, int N, int P>
static void launch_quad_l1(const QuadParams& p, dim3 grid, cudaStream_t s) {
  if (p.g.L1 == 64) return launch_quad_t<Lat, N, P, 64>(p, grid, s);
  if (p.g.L1 == 32) return launch_quad_t<Lat, N, P, 32>(p, grid, s);
  if (p.g.L1 == 128) return launch_quad_t<Lat, N, P, 128>(p, grid, s);
  launch_quad_t<Lat, N, P, 0>(p, grid, s);
}

template <class Lat, int N>
static void launch_quad_p(const sck_plan* plan, const QuadParams& p, dim3 grid, cudaStream_t s) {
  if (plan->P == 1) launch_quad_l1<Lat, N, 1>(p, grid, s);
  else launch_quad_l1<Lat, N, 2>(p, grid, s);
}

template <class Lat>
static void launch_quad_n(const sck_plan* plan, const QuadParams& p, dim3 grid, cudaStream_t s) {
  if (plan->geom.n == 2) launch_quad_p<Lat, 2>(plan, p, grid, s);
  else launch_quad_p<Lat, 3>(plan, p, grid, s);
}

static void launch_quad_grid(const sck_plan* plan, const QuadParams& p, dim3 grid, cudaStream_t s) {
  switch (plan->spec) {
    case Lat_square_1::id: launch_quad_n<Lat_square_1>(plan, p, grid, s); break;
    case Lat_triangular_1::id: launch_quad_n<Lat_triangular_1>(plan, p, grid, s); break;
    case Lat_sc_1::id: launch_quad_n<Lat_sc_1>(plan, p, grid, s); break;
    case Lat_bcc_1::id: launch_quad_n<Lat_bcc_1>(plan, p, grid, s); break;
    case Lat_bcc_1_2::id: launch_quad_n<Lat_bcc_1_2>(plan, p, grid, s); break;
    default: launch_quad_n<Lat_fcc_1>(plan, p, grid, s); break;
  }
}

static int quad_blocks_x(const sck_plan* plan) {
  const uint32_t per = (uint32_t)plan->geom.L3 * plan->geom.L2 * (plan->geom.L1 / plan->P);
  return (int)((per + 255) / 256);
}

static int launch_quad_params(const sck_plan* plan, QuadParams& p, cudaStream_t s) {
  const int Q = plan->Bp / 4;
  for (int q0 = 0; q0 < Q; q0 += 65535) {
    p.q0 = q0;
    const int nq = Q - q0 < 65535 ? Q - q0 : 65535;
    launch_quad_grid(plan, p, dim3((unsigned)quad_blocks_x(plan), (unsigned)nq), s);
    const int rc = cuda_status(cudaGetLastError(), "interleaved class launch");
    if (rc != SCK_OK) return rc;
  }
  return SCK_OK;
}

// One class of every quad (sweep offset 0: the sweep state[1] names).
int launch_quad_class(const sck_plan* plan, const sck_buffers* buf, int colour, int alpha, cudaStream_t s) {
  QuadParams p = quad_params(plan, buf, colour, alpha);
  return launch_quad_params(plan, p, s);
}

// ------------------------------------------------------------------------------------------ measure sweeps
// The coupling groups of class ci's sublattice whose bonds all reach classes earlier in the sweep order, or
// false when some group mixes earlier and later neighbours. For a linear colouring the neighbour's colour along
// bond (alpha -> alpha2, delta) is the site's colour shifted by K delta + o_alpha2 - o_alpha in every factor,
// the same for every site of the class, so the answer is one per (class, bond).
static bool class_lower_groups(const sck_plan* plan, int ci, unsigned* mask) {
  const sck_system_desc& d = plan->desc;
  const Colouring& col = plan->col;
  const int colour = d.classes[ci][0], alpha = d.classes[ci][1];
  int digit[SCK_MAX_FACTORS] = {0, 0, 0, 0};
  for (int r = col.r - 1, c = colour; r >= 0; --r) {
    digit[r] = c % col.m[r];
    c /= col.m[r];
  }
  const sck_sublattice& sub = d.sub[alpha];
  unsigned out = 0;
  int bi = 0;
  for (int gi = 0; gi < sub.n_groups; ++gi) {
    int lower = 0, later = 0;
    for (; bi < sub.group_end[gi]; ++bi) {
      const sck_bond& bd = sub.bonds[bi];
      int c2 = 0;
      for (int r = 0; r < col.r; ++r) {
        long long v = digit[r] + (long long)col.K[r][0] * bd.d[0] + (long long)col.K[r][1] * bd.d[1] +
                      (long long)col.K[r][2] * bd.d[2] + col.o[bd.alpha2][r] - col.o[alpha][r];
        v %= col.m[r];
        if (v < 0) v += col.m[r];
        c2 = c2 * col.m[r] + (int)v;
      }
      int idx = -1;
      for (int j = 0; j < d.n_classes; ++j)
        if (d.classes[j][0] == c2 && d.classes[j][1] == bd.alpha2) idx = j;
      if (idx < 0 || idx == ci) return false;   // a neighbour in no class, or in its own class: not a colouring
      (idx < ci ? lower : later) += 1;
    }
    if (lower && later) return false;
    if (lower) out |= 1u << gi;
  }
  *mask = out;
  return true;
}

bool quad_measure_fused(const sck_plan* plan) {
  if (plan->desc.n_classes > 64) return false;
  unsigned m = 0;
  for (int ci = 0; ci < plan->desc.n_classes; ++ci)
    if (!class_lower_groups(plan, ci, &m)) return false;
  return true;
}

size_t quad_measure_workspace(const sck_plan* plan) {
  const size_t fused = (size_t)plan->batch * plan->desc.n_classes * quad_blocks_x(plan) * (1 + plan->geom.n);
  const size_t exact = (size_t)plan->batch * quad_obs_blocks(plan) * OBS_VALUES;
  return (fused > exact ? fused : exact) * sizeof(double);
}

struct MeasureFinishParams {
  int n_classes, blocks_x, n, b;
  int cls_alpha[64];
};

// E[r] = sum of every class's and block's energy shares, M[r][alpha][k] = sum over the classes of sublattice
// alpha; one block per replica, fixed-order sums.
__global__ void __launch_bounds__(128) quad_measure_finish(const double* __restrict__ partial,
                                                           const __grid_constant__ MeasureFinishParams f,
                                                           double* __restrict__ E, double* __restrict__ M) {
  const int rep = blockIdx.x;
  const int V = 1 + f.n;
  const int per = f.n_classes * f.blocks_x;
  double acc[1 + SCK_MAX_BASIS * 3];
#pragma unroll
  for (int i = 0; i < 1 + SCK_MAX_BASIS * 3; ++i) acc[i] = 0.0;
  const double* src = partial + (size_t)rep * per * V;
  for (int i = threadIdx.x; i < per; i += blockDim.x) {
    const int a = f.cls_alpha[i / f.blocks_x];
    acc[0] += src[(size_t)i * V];
#pragma unroll
    for (int aa = 0; aa < SCK_MAX_BASIS; ++aa)
      if (aa == a)
#pragma unroll
        for (int k = 0; k < 3; ++k)
          if (k < f.n) acc[1 + aa * 3 + k] += src[(size_t)i * V + 1 + k];
  }
  __shared__ double red[1 + SCK_MAX_BASIS * 3][8];
  block_sum<1 + SCK_MAX_BASIS * 3>(acc, red);
  if (threadIdx.x == 0) {
    if (E != nullptr) E[rep] = acc[0];
    if (M != nullptr)
      for (int a = 0; a < f.b; ++a)
        for (int k = 0; k < f.n; ++k) M[((size_t)rep * f.b + a) * f.n + k] = acc[1 + a * 3 + k];
  }
}

// One sweep whose class launches also accumulate the FP64 observables of the configuration it leaves (E and M
// of the first plan->batch replicas), then the counter advance. Needs quad_measure_fused(plan).
static int launch_measure_finish(const sck_plan* plan, const void* workspace, double* E, double* M, cudaStream_t s);

int launch_quad_measure_sweep(const sck_plan* plan, const sck_buffers* buf, double* E, double* M, void* workspace,
                              cudaStream_t s) {
  const int C = plan->desc.n_classes;
  for (int ci = 0; ci < C; ++ci) {
    QuadParams p = quad_params(plan, buf, plan->desc.classes[ci][0], plan->desc.classes[ci][1]);
    if (!class_lower_groups(plan, ci, &p.lower_groups)) {
      set_error("measure sweep: a coupling group mixes earlier and later classes");
      return SCK_ERR_UNSUPPORTED;
    }
    p.measure_ci = ci;
    p.n_classes = C;
    p.blocks_x = quad_blocks_x(plan);
    p.B = plan->batch;
    p.partial = (double*)workspace;
    const int rc = launch_quad_params(plan, p, s);
    if (rc != SCK_OK) return rc;
  }
  const int rc = launch_advance(buf->state, 1, s);
  if (rc != SCK_OK) return rc;
  return launch_measure_finish(plan, workspace, E, M, s);
}

static int launch_measure_finish(const sck_plan* plan, const void* workspace, double* E, double* M, cudaStream_t s) {
  const int C = plan->desc.n_classes;
  MeasureFinishParams f;
  memset(&f, 0, sizeof(f));
  f.n_classes = C;
  f.blocks_x = quad_blocks_x(plan);
  f.n = plan->geom.n;
  f.b = plan->geom.b;
  for (int ci = 0; ci < C; ++ci) f.cls_alpha[ci] = plan->desc.classes[ci][1];
  quad_measure_finish<<<plan->batch, 128, 0, s>>>((const double*)workspace, f, E, M);
  return cuda_status(cudaGetLastError(), "measure sweep finish");
}

// Reference layout <-> interleaved storage: to_flat = 0 packs `flat` (B x N x sites floats) into `quads`,
// to_flat = 1 unpacks `quads` into `flat` (padding lanes are dropped).
int launch_quad_convert(const sck_plan* plan, float* flat, float4* quads, int to_flat, cudaStream_t s) {
  const Geometry& g = plan->geom;
  const uint32_t per = (uint32_t)g.n * (uint32_t)g.nsite;
  const int Q = plan->Bp / 4;
  const int hp = g.L1 / plan->P;
  for (int q0 = 0; q0 < Q; q0 += 65535) {
    const int nq = Q - q0 < 65535 ? Q - q0 : 65535;
    const dim3 grid((per + 255) / 256, (unsigned)nq);
    const size_t off4 = (size_t)q0 * per;
    if (to_flat)
      quad_unpack_kernel<<<grid, 256, 0, s>>>(quads + off4, flat + off4 * 4, g, hp, plan->P, plan->batch - 4 * q0);
    else
      quad_pack_kernel<<<grid, 256, 0, s>>>(flat + off4 * 4, quads + off4, g, hp, plan->P, plan->batch - 4 * q0);
    const int rc = cuda_status(cudaGetLastError(), to_flat ? "interleaved unpack" : "interleaved pack");
    if (rc != SCK_OK) return rc;
  }
  return SCK_OK;
}

int quad_obs_blocks(const sck_plan* plan) {
  const int Q = plan->Bp / 4;
  const int per_a = plan->geom.L3 * plan->geom.L2 * plan->geom.L1;
  const int most = (per_a + 255) / 256;
  const int want = (148 * 8 + Q - 1) / Q;
  return want < most ? (want < 1 ? 1 : want) : most;
}

template <class Lat, int N>
static void launch_qobs_n(const sck_plan* plan, const QuadObsParams& p, dim3 grid, cudaStream_t s) {
  if (plan->P == 1) quad_observables_kernel<Lat, N, 1><<<grid, 256, 0, s>>>(p);
  else quad_observables_kernel<Lat, N, 2><<<grid, 256, 0, s>>>(p);
}

template <class Lat>
static void launch_qobs(const sck_plan* plan, const QuadObsParams& p, dim3 grid, cudaStream_t s) {
  if (plan->geom.n == 2) launch_qobs_n<Lat, 2>(plan, p, grid, s);
  else launch_qobs_n<Lat, 3>(plan, p, grid, s);
}

// FP64 observables of the first `batch` replicas of interleaved storage; `workspace` holds
// batch x quad_obs_blocks x OBS_VALUES doubles.
int launch_quad_observables(const sck_plan* plan, const void* spins, int batch, const float* k1, double* E, double* M,
                            void* workspace, cudaStream_t s) {
  QuadObsParams p;
  memset(&p, 0, sizeof(p));
  p.g = plan->geom;
  for (int a = 0; a < SCK_MAX_BASIS; ++a) p.obs[a] = plan->obs[a];
  for (int k = 0; k < 3; ++k) p.h64[k] = plan->desc.h64[k];
  p.k2 = plan->desc.k2_64;
  p.hp = plan->geom.L1 / plan->P;
  p.blocks_per_quad = quad_obs_blocks(plan);
  p.B = batch;
  p.spins = (const float4*)spins;
  p.k1 = k1;
  p.partial = (double*)workspace;
  const int Q = (batch + 3) / 4;
  if (Q > 65535) return cuda_status(cudaErrorInvalidConfiguration, "interleaved observables: too many quads");
  const dim3 grid((unsigned)p.blocks_per_quad, (unsigned)Q);
  switch (plan->spec) {
    case Lat_square_1::id: launch_qobs<Lat_square_1>(plan, p, grid, s); break;
    case Lat_triangular_1::id: launch_qobs<Lat_triangular_1>(plan, p, grid, s); break;
    case Lat_sc_1::id: launch_qobs<Lat_sc_1>(plan, p, grid, s); break;
    case Lat_bcc_1::id: launch_qobs<Lat_bcc_1>(plan, p, grid, s); break;
    case Lat_bcc_1_2::id: launch_qobs<Lat_bcc_1_2>(plan, p, grid, s); break;
    default: launch_qobs<Lat_fcc_1>(plan, p, grid, s); break;
  }
  const int rc = cuda_status(cudaGetLastError(), "interleaved observables");
  if (rc != SCK_OK) return rc;
  return launch_observables_finish(p.partial, batch, p.blocks_per_quad, plan->geom.b, plan->geom.n, E, M, s);
}

// ---------------------------------------------------------------------------------------- pipeline host
size_t quad_pipe_counter_bytes(const sck_plan* plan) {
  const int Q = plan->Bp / 4;
  const int ngroups = (Q + plan->quad_group - 1) / plan->quad_group;
  return (size_t)(1 + ngroups * plan->desc.n_classes) * sizeof(unsigned);
}

template <class Lat, int N, int P, int L1C>
static void launch_pipe_t(const QuadPipeParams& pp, unsigned blocks, cudaStream_t s) {
  if (pp.partial != nullptr)
    quad_pipe_kernel<Lat, N, P, L1C, true><<<blocks, 256, 0, s>>>(pp);
  else
    quad_pipe_kernel<Lat, N, P, L1C, false><<<blocks, 256, 0, s>>>(pp);
}

template <class Lat, int N, int P>
static void launch_pipe_l1(const QuadPipeParams& pp, unsigned blocks, cudaStream_t s) {
  if (pp.p.g.L1 == 64) launch_pipe_t<Lat, N, P, 64>(pp, blocks, s);
  else if (pp.p.g.L1 == 32) launch_pipe_t<Lat, N, P, 32>(pp, blocks, s);
  else if (pp.p.g.L1 == 128) launch_pipe_t<Lat, N, P, 128>(pp, blocks, s);
  else launch_pipe_t<Lat, N, P, 0>(pp, blocks, s);
}

template <class Lat>
static void launch_pipe_lat(const sck_plan* plan, const QuadPipeParams& pp, unsigned blocks, cudaStream_t s) {
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
int launch_quad_pipeline(const sck_plan* plan, const sck_buffers* buf, int n_sweeps, cudaStream_t s,
                         double* partial) {
  if (plan->pipe_counters == nullptr || plan->giveup_dev == nullptr) {
    set_error("the interleaved pipeline has no counters: call sck_plan_pipeline on this device");
    return SCK_ERR_INVALID;
  }
  QuadPipeParams pp;
  memset(&pp, 0, sizeof(pp));
  pp.p = quad_params(plan, buf, 0, 0);
  const int C = plan->desc.n_classes;
  pp.C = C;
  pp.D = plan->quad_skew;
  pp.group = plan->quad_group;
  pp.Q = plan->Bp / 4;
  pp.ngroups = (pp.Q + pp.group - 1) / pp.group;
  pp.blocks_x = quad_blocks_x(plan);
  pp.T = pp.group * pp.blocks_x;
  for (int ci = 0; ci < C; ++ci) {
    pp.cls[ci][0] = plan->desc.classes[ci][0];
    pp.cls[ci][1] = plan->desc.classes[ci][1];
  }
  pp.ticket = (unsigned*)plan->pipe_counters;
  pp.done = pp.ticket + 1;
  pp.wait_limit = plan->wait_limit;
  pp.giveup = plan->giveup_dev;
  pp.B = plan->batch;
  if (partial != nullptr)
    for (int ci = 0; ci < C; ++ci)
      if (!class_lower_groups(plan, ci, &pp.lower_groups[ci])) {
        set_error("measure sweep: a coupling group mixes earlier and later classes");
        return SCK_ERR_UNSUPPORTED;
      }
  const long long per_pos = (long long)(C / pp.D) * pp.T;
  const long long units_max = ((1ll << 30) / per_pos - C) / pp.D;
  const long long sweeps_per_launch = units_max / pp.ngroups;
  if (sweeps_per_launch < 1) return cuda_status(cudaErrorInvalidConfiguration, "interleaved pipeline: too many tickets");
  const size_t bytes = quad_pipe_counter_bytes(plan);
  for (int sw0 = 0; sw0 < n_sweeps; sw0 += (int)sweeps_per_launch) {
    const int n = (int)((long long)(n_sweeps - sw0) < sweeps_per_launch ? n_sweeps - sw0 : sweeps_per_launch);
    pp.units = n * pp.ngroups;
    pp.sweep_base = sw0;
    pp.partial = (partial != nullptr && sw0 + n == n_sweeps) ? partial : nullptr;
    int rc = cuda_status(cudaMemsetAsync(plan->pipe_counters, 0, bytes, s), "interleaved pipeline counters");
    if (rc != SCK_OK) return rc;
    const long long positions = (long long)pp.D * (pp.units - 1) + C;
    const unsigned blocks = (unsigned)(positions * per_pos);
    switch (plan->spec) {
      case Lat_square_1::id: launch_pipe_lat<Lat_square_1>(plan, pp, blocks, s); break;
      case Lat_triangular_1::id: launch_pipe_lat<Lat_triangular_1>(plan, pp, blocks, s); break;
      case Lat_sc_1::id: launch_pipe_lat<Lat_sc_1>(plan, pp, blocks, s); break;
      case Lat_bcc_1::id: launch_pipe_lat<Lat_bcc_1>(plan, pp, blocks, s); break;
      case Lat_bcc_1_2::id: launch_pipe_lat<Lat_bcc_1_2>(plan, pp, blocks, s); break;
      default: launch_pipe_lat<Lat_fcc_1>(plan, pp, blocks, s); break;
    }
    rc = cuda_status(cudaGetLastError(), "interleaved pipeline launch");
    if (rc != SCK_OK) return rc;
  }
  return SCK_OK;
}

// A measure step through the pipeline: n sweeps, the last one measured, the counter advance and the sums.
int launch_quad_pipeline_measure(const sck_plan* plan, const sck_buffers* buf, int n_sweeps, double* E, double* M,
                                 void* workspace, cudaStream_t s) {
  int rc = launch_quad_pipeline(plan, buf, n_sweeps, s, (double*)workspace);
  if (rc != SCK_OK) return rc;
  rc = launch_advance(buf->state, n_sweeps, s);
  if (rc != SCK_OK) return rc;
  return launch_measure_finish(plan, workspace, E, M, s);
}

}  // namespace sck
