// Row kernels for vector models on lattices whose colour classes alternate along x (x-period 2: square, sc,
// bcc with one or two shells), in periodic boxes without a mask and with L1 a multiple of 64.
//
// A warp owns a 64-cell segment of one row (z, y) of its class's sublattice: lane l owns the class site
// x = xs + 2 l + p, p in {0, 1} being the row's class residue. Every row the update reads is fetched as
// consecutive cell pairs (xs + 2 l, xs + 2 l + 1), one 8-byte load per lane, so a warp load covers two full
// 128-byte lines with nothing wasted; a neighbour at x - 1 or x + 1 that falls in the adjacent lane's pair
// comes through a warp shuffle, and rows shared by several bonds are loaded once (compile-time dedupe over the
// bond table). The arithmetic is the specialised kernel's (two replicas per lane in float32x2).
#include "spec.cuh"

namespace sck {

constexpr unsigned kFull = 0xFFFFFFFFu;

// First bond of sublattice A that reads the same row (sublattice, dy, dz) as bond i.
template <class Lat, int A>
__host__ __device__ constexpr int first_same_row(int i) {
  const BondC b = Lat::bond(A, i);
  for (int j = 0; j < i; ++j) {
    const BondC c = Lat::bond(A, j);
    if (c.a2 == b.a2 && c.dy == b.dy && c.dz == b.dz) return j;
  }
  return i;
}

template <class Lat, int A>
__host__ __device__ constexpr bool own_row(int i) {
  const BondC b = Lat::bond(A, i);
  return b.a2 == A && b.dy == 0 && b.dz == 0;
}

// Cell xs + 2 lane + j of a row held as lane pairs (j in -1..2, warp-uniform). Lanes at the segment edges read
// the neighbouring segment's cell from memory when the row has several segments.
__device__ __forceinline__ float pick(float2 pr, int j, int lane, const float* row, int xs, int L1, int segs) {
  if (j == 0) return pr.x;
  if (j == 1) return pr.y;
  if (j < 0) {
    float v = __shfl_sync(kFull, pr.y, (lane + 31) & 31);
    if (segs > 1 && lane == 0) v = row[(xs == 0 ? L1 : xs) - 1];
    return v;
  }
  float v = __shfl_sync(kFull, pr.x, (lane + 1) & 31);
  if (segs > 1 && lane == 31) v = row[xs + 64 == L1 ? 0 : xs + 64];
  return v;
}

template <class Lat, int A, int N>
__device__ __forceinline__ void row_pair_site(const SpecParams& p, int rep0, bool two, int y, int z, int xs, int pq,
                                              int lane, int32_t key) {
  const Common& c = p.c;
  const Geometry& g = c.g;
  const int L1 = g.L1, L2 = g.L2, L3 = g.L3, segs = p.segs_per_row;
  const size_t NS = (size_t)g.nsite, RS = two ? (size_t)N * NS : 0;
  const float* base = (const float*)c.src + (size_t)rep0 * N * NS;
  const int rep1 = two ? rep0 + 1 : rep0;
  const int x = xs + 2 * lane + pq;
  const int own = A * g.plane + (z * L2 + y) * L1 + x;
  const int ym = y == 0 ? L2 - 1 : y - 1, yp = y == L2 - 1 ? 0 : y + 1;
  const int zm = g.dim == 3 ? (z == 0 ? L3 - 1 : z - 1) : z, zp = g.dim == 3 ? (z == L3 - 1 ? 0 : z + 1) : z;
  auto row_start = [&](int a2, int dy, int dz) {
    const int yy = dy < 0 ? ym : (dy > 0 ? yp : y);
    const int zz = dz < 0 ? zm : (dz > 0 ? zp : z);
    return a2 * g.plane + (zz * L2 + yy) * L1;
  };
  // own row: the site's spin and its same-row neighbours
  const int own_row_start = A * g.plane + (z * L2 + y) * L1;
  float2 orow[N][2];
#pragma unroll
  for (int k = 0; k < N; ++k) {
    const float* r = base + k * NS + own_row_start;
    orow[k][0] = *reinterpret_cast<const float2*>(r + xs + 2 * lane);
    orow[k][1] = *reinterpret_cast<const float2*>(r + RS + xs + 2 * lane);
  }
  float2 s[N], v[N];
#pragma unroll
  for (int k = 0; k < N; ++k) {
    s[k] = pq == 0 ? make_float2(orow[k][0].x, orow[k][1].x) : make_float2(orow[k][0].y, orow[k][1].y);
    v[k] = f2(0.0f);
  }
  constexpr int MB = Lat::max_bonds;
  float2 rows[MB][N][2];
  int starts[MB];
  static_for<0, Lat::groups>([&](auto gc) {
    constexpr int gi = decltype(gc)::value;
    using R = GroupRange<Lat, A, gi>;
    float2 gs[N];
#pragma unroll
    for (int k = 0; k < N; ++k) gs[k] = f2(0.0f);
    static_for<R::begin, R::end>([&](auto ic) {
      constexpr int i = decltype(ic)::value;
      constexpr BondC bd = Lat::bond(A, i);
      constexpr int src = first_same_row<Lat, A>(i);
      constexpr bool own_r = own_row<Lat, A>(i);
      if constexpr (!own_r && src == i) {
        starts[i] = row_start(bd.a2, bd.dy, bd.dz);
#pragma unroll
        for (int k = 0; k < N; ++k) {
          const float* r = base + k * NS + starts[i];
          rows[i][k][0] = *reinterpret_cast<const float2*>(r + xs + 2 * lane);
          rows[i][k][1] = *reinterpret_cast<const float2*>(r + RS + xs + 2 * lane);
        }
      }
      const int j = pq + bd.dx;
#pragma unroll
      for (int k = 0; k < N; ++k) {
        const float2* pr = own_r ? orow[k] : rows[src][k];
        const float* r0 = base + k * NS + (own_r ? own_row_start : starts[src]);
        const float a = pick(pr[0], j, lane, r0, xs, L1, segs);
        const float b = pick(pr[1], j, lane, r0 + RS, xs, L1, segs);
        gs[k] = __fadd2_rn(gs[k], make_float2(a, b));
      }
    });
#pragma unroll
    for (int k = 0; k < N; ++k) v[k] = __fadd2_rn(v[k], __fmul2_rn(f2(p.J[A][gi]), gs[k]));
  });
#pragma unroll
  for (int k = 0; k < N; ++k)
    if (c.hnz[k]) v[k] = __fadd2_rn(v[k], f2(c.h[k]));
  float2 t[N];
  bool acc0, acc1;
  finish_pair<N>(c, own, rep0, rep1, two, key, s, v, t, acc0, acc1);
  float* po = (float*)c.dst + (size_t)rep0 * N * NS + own;
  if (acc0) {
#pragma unroll
    for (int k = 0; k < N; ++k) po[k * NS] = t[k].x;
  }
  if (two && acc1) {
#pragma unroll
    for (int k = 0; k < N; ++k) po[k * NS + RS] = t[k].y;
  }
}

// Grid (ceil(row segments / 8), n_tasks * units_per_task); 8 warps per block, one row segment per warp.
template <class Lat, int N>
__global__ void __launch_bounds__(256) row_task_kernel(const __grid_constant__ SpecParams p) {
  const int lane = threadIdx.x & 31;
  const int seg = blockIdx.x * 8 + (threadIdx.x >> 5);
  if (seg >= p.c.rows * p.segs_per_row) return;
  const int ti = blockIdx.y / p.units_per_task;
  const int unit = blockIdx.y - ti * p.units_per_task;
  const Task task = p.tasks[ti];
  const int rep = task.rep_begin + 2 * unit;
  if (rep >= task.rep_end) return;
  const int row = seg / p.segs_per_row;
  const int xs = (seg - row * p.segs_per_row) * 64;
  int x0, y, z;
  if (!class_site(p.c, task.colour, task.alpha, (uint32_t)row * (uint32_t)p.c.bx, x0, y, z)) return;
  const int32_t key = sweep_key_at(p.c.state, task.sweep_offset);
  static_for<0, Lat::b>([&](auto ac) {
    constexpr int a = decltype(ac)::value;
    if (a != task.alpha) return;
    row_pair_site<Lat, a, N>(p, rep, rep + 1 < task.rep_end, y, z, xs, x0, lane, key);
  });
}

bool row_kernel_ok(const sck_plan* plan) {
  const Geometry& g = plan->geom;
  if (!plan->row_kernels || plan->mode != SCK_MODE_F32 || g.n < 2 || g.has_mask || plan->P != 2) return false;
  if (g.L1 % 64 != 0 || !g.per[0] || !g.per[1] || (g.dim == 3 && !g.per[2])) return false;
  return plan->spec == Lat_square_1::id || plan->spec == Lat_sc_1::id || plan->spec == Lat_bcc_1::id ||
         plan->spec == Lat_bcc_1_2::id;
}

template <class Lat>
static void launch_row_lat(const sck_plan* plan, const SpecParams& p, dim3 grid, cudaStream_t s) {
  if (plan->geom.n == 2)
    row_task_kernel<Lat, 2><<<grid, 256, 0, s>>>(p);
  else
    row_task_kernel<Lat, 3><<<grid, 256, 0, s>>>(p);
}

int launch_row_tasks(const sck_plan* plan, const SpecParams& p, int ys, cudaStream_t s) {
  const int nseg = plan->geom.L3 * plan->geom.L2 * (plan->geom.L1 / 64);
  const dim3 grid((nseg + 7) / 8, (unsigned)ys);
  switch (plan->spec) {
    case Lat_square_1::id: launch_row_lat<Lat_square_1>(plan, p, grid, s); break;
    case Lat_sc_1::id: launch_row_lat<Lat_sc_1>(plan, p, grid, s); break;
    case Lat_bcc_1::id: launch_row_lat<Lat_bcc_1>(plan, p, grid, s); break;
    default: launch_row_lat<Lat_bcc_1_2>(plan, p, grid, s); break;
  }
  return cuda_status(cudaGetLastError(), "row class launch");
}

}  // namespace sck
