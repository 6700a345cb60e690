// Segment kernels: the class update of vector models (n = 2, 3) on a periodic box with a compile-time bond
// table (lattices.h) and a colouring whose classes alternate along x (x-period 2).
//
// A thread owns an aligned 4-site x-segment of one row of one replica, whose two sites of the class sit at
// x0 + d and x0 + d + 2 (d = 0 or 1 by row). For every distinct neighbour row of the sublattice's bond table
// (own row first) it loads the segment of each component with one 128-bit load (the lanes of a warp read
// consecutive 16-byte pieces of a row, so every sector fetched is used whole), plus the one site past either
// end that an x-offset of -1 or +1 reaches, and adds each bond's neighbour to the coupling-group sums of both
// sites. Compared with one site and two replicas per thread this halves the load instructions and shares the
// row addressing between the two sites. The group sums run in row order rather than the reference's bond
// order, so local fields differ from the reference's by float32 rounding only; the
// proposal, energy change and acceptance keep the reference's operation order (finish_core in spec.cuh). Lanes
// are mapped to rows so that the rows of a warp share d (rows of one y parity are consecutive), which keeps the
// two compile-time variants of a warp from diverging.
#include "spec.cuh"

namespace sck {

// ------------------------------------------------------------------------ compile-time rows of a bond table
template <class Lat, int A>
struct SegRows {
  static constexpr int nb = Lat::n_bonds(A);
  __host__ __device__ static constexpr bool same_row(const BondC& b, int a2, int dy, int dz) {
    return b.a2 == a2 && b.dy == dy && b.dz == dz;
  }
  // is bond i the first to read its row (the own row (A, 0, 0) is row 0 and never "first")
  __host__ __device__ static constexpr bool first(int i) {
    const BondC b = Lat::bond(A, i);
    if (same_row(b, A, 0, 0)) return false;
    for (int j = 0; j < i; ++j)
      if (same_row(Lat::bond(A, j), b.a2, b.dy, b.dz)) return false;
    return true;
  }
  __host__ __device__ static constexpr int count() {
    int n = 1;
    for (int i = 0; i < nb; ++i) n += first(i) ? 1 : 0;
    return n;
  }
  __host__ __device__ static constexpr BondC row(int r) {
    if (r == 0) return BondC{A, 0, 0, 0};
    int n = 0;
    for (int i = 0; i < nb; ++i)
      if (first(i) && ++n == r) return Lat::bond(A, i);
    return BondC{A, 0, 0, 0};
  }
  __host__ __device__ static constexpr int row_of_bond(int i) {
    const BondC b = Lat::bond(A, i);
    for (int r = 0; r < count(); ++r) {
      const BondC q = row(r);
      if (same_row(b, q.a2, q.dy, q.dz)) return r;
    }
    return -1;
  }
  __host__ __device__ static constexpr bool has_dx(int r, int dx) {
    for (int i = 0; i < nb; ++i)
      if (row_of_bond(i) == r && Lat::bond(A, i).dx == dx) return true;
    return false;
  }
  __host__ __device__ static constexpr int group_of(int i) {
    int g = 0;
    while (g < Lat::groups && Lat::group_end(A, g) <= i) ++g;
    return g;
  }
  __host__ __device__ static constexpr bool reach_one() {
    for (int i = 0; i < nb; ++i) {
      const BondC b = Lat::bond(A, i);
      if (b.dx < -1 || b.dx > 1 || b.dy < -1 || b.dy > 1 || b.dz < -1 || b.dz > 1) return false;
    }
    return true;
  }
};

__device__ __forceinline__ int wrap1(int v, int L) { return v < 0 ? v + L : (v >= L ? v - L : v); }

// the two class sites x0 + D and x0 + D + 2 of row (y, z), sublattice A, replica rep; NSL > 0: the replica has
// 2^NSL sites and the component planes sit at compile-time offsets from one address
template <class Lat, int A, int N, int D, int NSL>
__device__ __forceinline__ void seg_sites(const Common& c, const float (&J)[SCK_MAX_GROUPS], int rep, int y, int z,
                                          int x0, int32_t key) {
  using R = SegRows<Lat, A>;
  const Geometry& g = c.g;
  const size_t NS = NSL ? ((size_t)1 << NSL) : (size_t)g.nsite;
  const float* base = (const float*)c.src + (size_t)rep * N * NS;
  float* obase = (float*)c.dst + (size_t)rep * N * NS;
  const float* bk[N];   // component planes of the replica: each load is one 32-bit index off these
#pragma unroll
  for (int k = 0; k < N; ++k) bk[k] = base + k * NS;
  // scalar group sums per site: the two sites of a pair sit two registers apart in a 128-bit load, so packing
  // them for float32x2 adds would cost a move per add
  float gs[Lat::groups][N][2];
#pragma unroll
  for (int gi = 0; gi < Lat::groups; ++gi)
#pragma unroll
    for (int k = 0; k < N; ++k) gs[gi][k][0] = gs[gi][k][1] = 0.0f;
  float2 s[N];
  const int xl = x0 == 0 ? g.L1 - 1 : x0 - 1;
  const int xr = x0 + 4 == g.L1 ? 0 : x0 + 4;
  static_for<0, R::count()>([&](auto rc) {
    constexpr int r = decltype(rc)::value;
    constexpr BondC row = R::row(r);
    constexpr bool left = D == 0 && R::has_dx(r, -1);
    constexpr bool right = D == 1 && R::has_dx(r, 1);
    const int yy = wrap1(y + row.dy, g.L2);
    const int zz = Lat::dim == 3 ? wrap1(z + row.dz, g.L3) : 0;
    const int ro = row.a2 * g.plane + (zz * g.L2 + yy) * g.L1;
#pragma unroll
    for (int k = 0; k < N; ++k) {
      const float4 m = *(const float4*)(bk[k] + ro + x0);
      float w[6] = {0.f, m.x, m.y, m.z, m.w, 0.f};
      if (left) w[0] = bk[k][ro + xl];
      if (right) w[5] = bk[k][ro + xr];
      if constexpr (r == 0) s[k] = make_float2(w[1 + D], w[3 + D]);
      static_for<0, R::nb>([&](auto ic) {
        constexpr int i = decltype(ic)::value;
        if constexpr (R::row_of_bond(i) == r) {
          constexpr int o = 1 + D + Lat::bond(A, i).dx;
          constexpr int gi = R::group_of(i);
          gs[gi][k][0] = __fadd_rn(gs[gi][k][0], w[o]);
          gs[gi][k][1] = __fadd_rn(gs[gi][k][1], w[o + 2]);
        }
      });
    }
  });
  float2 v[N];
#pragma unroll
  for (int k = 0; k < N; ++k) {
    float2 acc = f2(0.0f);
#pragma unroll
    for (int gi = 0; gi < Lat::groups; ++gi)
      acc = __fadd2_rn(acc, __fmul2_rn(f2(J[gi]), make_float2(gs[gi][k][0], gs[gi][k][1])));
    if (c.hnz[k]) acc = __fadd2_rn(acc, f2(c.h[k]));
    v[k] = acc;
  }
  const int oa = A * g.plane + (z * g.L2 + y) * g.L1 + x0 + D, ob = oa + 2;
  const float beta = c.beta[rep];
  float2 t[N];
  bool acc0, acc1;
  finish_core<N>(c, counter_of(rep, g.nsite, oa), counter_of(rep, g.nsite, ob), true, oa, ob,
                 make_float2(beta, beta), key, s, v, t, acc0, acc1);
  float* po = obase + oa;
  if (acc0) {
#pragma unroll
    for (int k = 0; k < N; ++k) po[k * NS] = t[k].x;
  }
  if (acc1) {
#pragma unroll
    for (int k = 0; k < N; ++k) po[k * NS + 2] = t[k].y;
  }
}

// Grid (ceil(rows * L1 / 4 / 256), n_tasks * units_per_task); block y-slot -> (task, replica).
template <class Lat, int N, int NSL>
__global__ void __launch_bounds__(256, 4) seg_kernel(const __grid_constant__ SpecParams p) {
  const Common& c = p.c;
  const Geometry& g = c.g;
  const uint32_t segs = (uint32_t)(g.L1 >> 2);
  const uint32_t per = (uint32_t)g.L2 * (uint32_t)g.L3 * segs;
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= per) return;
  const int ti = blockIdx.y / p.units_per_task;
  const Task task = p.tasks[ti];
  const int rep = task.rep_begin + (int)(blockIdx.y - ti * p.units_per_task);
  if (rep >= task.rep_end) return;
  const uint32_t rowi = fdiv(t, p.fd_segs);
  const int x0 = (int)(t - rowi * segs) * 4;
  const int z = (int)fdiv(rowi, c.fd_L2);
  const int i = (int)rowi - z * g.L2;
  // rows of one y parity first (an even L2 keeps each half whole), so a warp's rows share the class offset
  const int y = (g.L2 & 1) ? i : (i < (g.L2 >> 1) ? 2 * i : 2 * (i - (g.L2 >> 1)) + 1);
  const int alpha = task.alpha;
  const int d = first_class_x(c, task.colour, alpha, y, z);
  if (d > 1) return;
  const int32_t key = sweep_key_at(c.state, task.sweep_offset);
  static_for<0, Lat::b>([&](auto ac) {
    constexpr int a = decltype(ac)::value;
    if (a != alpha) return;
    if (d == 0)
      seg_sites<Lat, a, N, 0, NSL>(c, p.J[a], rep, y, z, x0, key);
    else
      seg_sites<Lat, a, N, 1, NSL>(c, p.J[a], rep, y, z, x0, key);
  });
}

template <class Lat>
static constexpr bool lat_reach_one() {
  bool ok = true;
  if constexpr (Lat::b >= 1) ok = ok && SegRows<Lat, 0>::reach_one();
  if constexpr (Lat::b >= 2) ok = ok && SegRows<Lat, 1>::reach_one();
  if constexpr (Lat::b >= 3) ok = ok && SegRows<Lat, 2>::reach_one();
  if constexpr (Lat::b >= 4) ok = ok && SegRows<Lat, 3>::reach_one();
  return ok;
}

bool seg_kernel_ok(const sck_plan* plan) {
  const Geometry& g = plan->geom;
  if (plan->kernel_kind != 2 || plan->mode != SCK_MODE_F32 || g.n < 2 || g.has_mask || plan->P != 2) return false;
  if (g.L1 % 4 != 0 || !g.per[0] || !g.per[1] || g.L2 < 3) return false;
  if (g.dim == 3 && (!g.per[2] || g.L3 < 3)) return false;
  switch (plan->spec) {
    case Lat_square_1::id: return lat_reach_one<Lat_square_1>();
    case Lat_sc_1::id: return lat_reach_one<Lat_sc_1>();
    case Lat_bcc_1::id: return lat_reach_one<Lat_bcc_1>();
    case Lat_bcc_1_2::id: return lat_reach_one<Lat_bcc_1_2>();
    case Lat_fcc_1::id: return lat_reach_one<Lat_fcc_1>();
    default: return false;
  }
}

template <class Lat, int N>
static void launch_seg_n(const sck_plan* plan, const SpecParams& p, dim3 grid, cudaStream_t s) {
  // replicas of 2^16 .. 2^19 sites: component offsets up to 4 MB fit a load's immediate offset
  switch (plan->geom.nsite) {
    case 1 << 16: seg_kernel<Lat, N, 16><<<grid, 256, 0, s>>>(p); break;
    case 1 << 17: seg_kernel<Lat, N, 17><<<grid, 256, 0, s>>>(p); break;
    case 1 << 18: seg_kernel<Lat, N, 18><<<grid, 256, 0, s>>>(p); break;
    case 1 << 19: seg_kernel<Lat, N, 19><<<grid, 256, 0, s>>>(p); break;
    default: seg_kernel<Lat, N, 0><<<grid, 256, 0, s>>>(p); break;
  }
}

template <class Lat>
static void launch_seg_lat(const sck_plan* plan, const SpecParams& p, dim3 grid, cudaStream_t s) {
  if (plan->geom.n == 2)
    launch_seg_n<Lat, 2>(plan, p, grid, s);
  else
    launch_seg_n<Lat, 3>(plan, p, grid, s);
}

int launch_seg_tasks(const sck_plan* plan, SpecParams& p, int ys, cudaStream_t s) {
  const Geometry& g = plan->geom;
  const uint32_t per = (uint32_t)g.L2 * (uint32_t)g.L3 * (uint32_t)(g.L1 >> 2);
  p.fd_segs = make_fastdiv((uint32_t)(g.L1 >> 2));
  const dim3 grid((per + 255) / 256, (unsigned)ys);
  switch (plan->spec) {
    case Lat_square_1::id: launch_seg_lat<Lat_square_1>(plan, p, grid, s); break;
    case Lat_sc_1::id: launch_seg_lat<Lat_sc_1>(plan, p, grid, s); break;
    case Lat_bcc_1::id: launch_seg_lat<Lat_bcc_1>(plan, p, grid, s); break;
    case Lat_bcc_1_2::id: launch_seg_lat<Lat_bcc_1_2>(plan, p, grid, s); break;
    default: launch_seg_lat<Lat_fcc_1>(plan, p, grid, s); break;
  }
  return cuda_status(cudaGetLastError(), "segment class launch");
}

}  // namespace sck
