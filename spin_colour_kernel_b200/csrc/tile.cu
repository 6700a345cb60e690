// Tile kernels: the class update of vector models on a periodic box with a compile-time bond table, reading
// every neighbour from shared memory.
//
// A block of threads owns a brick of one replica: BR_Z planes x BR_Y rows x the whole row length (one plane in
// 2D). It copies the brick plus one halo plane and one halo row on every side (both sublattices, every
// component, float32) into shared memory with one bulk asynchronous copy per row (the copy engine moves the
// bytes; the threads issue one instruction per row and wait on one mbarrier, with a bounded wait), fills the
// halo site at each end of every row from the row itself, and then updates the class sites of the brick. Every
// neighbour is a shared-memory load at a compile-time offset from the site's own shared address: none of the
// 64-bit address arithmetic that the global-memory kernels spend on each neighbour load is left. A thread takes
// two class sites of one row and runs the proposal and acceptance of both in packed float32x2 arithmetic
// (finish_core in spec.cuh). Neighbours are never sites of the class being updated, so the shared copy never
// goes stale within a launch. Group sums run in bond order, so results are those of the lattice kernels.
#include "spec.cuh"

namespace sck {

constexpr int BR_Y = 4;       // rows per brick
constexpr int TILE_PAD = 4;   // floats before x = 0 in a shared row: x = -1 sits at TILE_PAD - 1
constexpr long long kBrickWaitLimit = 1ll << 22;   // mbarrier polls of the drain after a brick gave up

template <class Lat, int N, int L1T, int BZ>
struct BrickDims {
  static_assert(Lat::reach == 1, "tile kernels read neighbours at most one cell away");
  static constexpr int R2 = BR_Y + 2;                   // rows with halo
  static constexpr int P2 = BZ == 1 ? 1 : BZ + 2;       // planes with halo (2D: the one plane)
  static constexpr int ZO = BZ == 1 ? 0 : 1;            // plane index of the brick's first plane
  static constexpr int RS = L1T + 2 * TILE_PAD;         // floats per shared row
  static constexpr int PLANE = R2 * RS;
  static constexpr int COMP = P2 * PLANE;               // one component of one sublattice
  static constexpr int FLOATS = Lat::b * N * COMP;
  static constexpr int ROWS = Lat::b * N * P2 * R2;     // rows copied
  static constexpr int BYTES = FLOATS * 4 + 16;         // + the mbarrier
};

struct TileParams {
  Common c;
  float J[SCK_MAX_BASIS][SCK_MAX_GROUPS];
  int colour, alpha;
};

static __device__ unsigned long long g_wait_timeouts;   // bounded waits that gave up (sck_wait_timeouts)

__device__ __forceinline__ uint32_t saddr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// 32-bit shared-memory load at a compile-time byte offset from a register address
template <int OFF>
__device__ __forceinline__ float lds(uint32_t addr) {
  float v;
  asm volatile("ld.shared.f32 %0, [%1+%2];\n" : "=f"(v) : "r"(addr), "n"(OFF));
  return v;
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t mbar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(mbar), "r"(parity)
      : "memory");
  return ok != 0;
}

// the two class sites xa and xa + P of row y0 + ty, plane z0 + tz (lane .y absent when !two)
template <class Lat, int A, int N, int L1T, int BZ>
__device__ __forceinline__ void brick_pair(const Common& c, const float (&J)[SCK_MAX_GROUPS], uint32_t sbase, int rep,
                                           int tz, int ty, int xa, int y, int z, bool two, int32_t key) {
  using D = BrickDims<Lat, N, L1T, BZ>;
  const Geometry& g = c.g;
  const int xb = two ? xa + c.P : xa;
  const int own_a = A * g.plane + (z * g.L2 + y) * L1T + xa, own_b = own_a + (xb - xa);
  const bool la = !g.has_mask || c.mask[own_a] != 0;
  const bool lb = two && (!g.has_mask || c.mask[own_b] != 0);
  if (!la && !lb) return;
  const int row = (tz + D::ZO) * D::PLANE + (ty + 1) * D::RS + TILE_PAD;
  const uint32_t qa = sbase + 4u * (uint32_t)(row + xa), qb = sbase + 4u * (uint32_t)(row + xb);
  float2 s[N], v[N];
  static_for<0, N>([&](auto kc) {
    constexpr int k = decltype(kc)::value;
    constexpr int o = 4 * (A * N + k) * D::COMP;
    s[k] = make_float2(lds<o>(qa), lds<o>(qb));
    v[k] = f2(0.0f);
  });
  static_for<0, Lat::groups>([&](auto gc) {
    constexpr int gi = decltype(gc)::value;
    using R = GroupRange<Lat, A, gi>;
    float2 gs[N];
#pragma unroll
    for (int k = 0; k < N; ++k) gs[k] = f2(0.0f);
    static_for<R::begin, R::end>([&](auto ic) {
      constexpr BondC bd = Lat::bond(A, decltype(ic)::value);
      constexpr int off = 4 * (bd.a2 * N * D::COMP + bd.dz * D::PLANE + bd.dy * D::RS + bd.dx);
      static_for<0, N>([&](auto kc) {
        constexpr int k = decltype(kc)::value;
        gs[k] = __fadd2_rn(gs[k], make_float2(lds<off + 4 * k * D::COMP>(qa), lds<off + 4 * k * D::COMP>(qb)));
      });
    });
#pragma unroll
    for (int k = 0; k < N; ++k) v[k] = __fadd2_rn(v[k], __fmul2_rn(f2(J[gi]), gs[k]));
  });
#pragma unroll
  for (int k = 0; k < N; ++k)
    if (c.hnz[k]) v[k] = __fadd2_rn(v[k], f2(c.h[k]));
  float2 t[N];
  bool acc0, acc1;
  const float beta = c.beta[rep];
  finish_core<N>(c, counter_of(rep, g.nsite, own_a), counter_of(rep, g.nsite, own_b), two, own_a, own_b,
                 make_float2(beta, beta), key, s, v, t, acc0, acc1);
  const size_t NS = (size_t)g.nsite;
  float* po = (float*)c.dst + (size_t)rep * N * NS;
  if (la && acc0) {
#pragma unroll
    for (int k = 0; k < N; ++k) po[k * NS + own_a] = t[k].x;
  }
  if (lb && acc1) {
#pragma unroll
    for (int k = 0; k < N; ++k) po[k * NS + own_b] = t[k].y;
  }
}

// Grid ((L2 / BR_Y) x (L3 / BZ) bricks, B replicas), 256 threads.
template <class Lat, int N, int L1T, int BZ>
__global__ void __launch_bounds__(256) brick_class_kernel(const __grid_constant__ TileParams p) {
  using D = BrickDims<Lat, N, L1T, BZ>;
  extern __shared__ __align__(128) float sm[];
  const Common& c = p.c;
  const Geometry& g = c.g;
  const int nby = g.L2 / BR_Y;
  const int y0 = (blockIdx.x % nby) * BR_Y, z0 = (blockIdx.x / nby) * BZ;
  const int rep = blockIdx.y;
  const uint32_t sbase = saddr(sm);
  const uint32_t mbar = sbase + 4u * D::FLOATS;
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(mbar) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(mbar), "r"(D::ROWS * L1T * 4)
                 : "memory");
  }
  __syncthreads();
  const float* src = (const float*)c.src + (size_t)rep * N * g.nsite;
  for (int row = threadIdx.x; row < D::ROWS; row += blockDim.x) {
    const int ry = row % D::R2, rest = row / D::R2, pz = rest % D::P2, ak = rest / D::P2, k = ak % N, a = ak / N;
    int y = y0 - 1 + ry;
    y = y < 0 ? y + g.L2 : (y >= g.L2 ? y - g.L2 : y);
    int z = z0 - D::ZO + pz;
    z = z < 0 ? z + g.L3 : (z >= g.L3 ? z - g.L3 : z);
    const float* gr = src + (size_t)k * g.nsite + (size_t)a * g.plane + ((size_t)z * g.L2 + y) * L1T;
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
            sbase + 4u * (uint32_t)(row * D::RS + TILE_PAD)),
        "l"(gr), "r"(L1T * 4), "r"(mbar)
        : "memory");
  }
  long long polls = 0;
  bool ready = false;
  while (polls < (long long)c.wait_limit && !(ready = mbar_try_wait(mbar, 0))) ++polls;
  if (__syncthreads_or(!ready)) {
    // gave up (every thread of the block agrees): count it, raise the plan's flag, wait (bounded again, with the
    // full limit) for the copies still in flight, leave the brick unchanged
    if (threadIdx.x == 0) {
      atomicAdd(&g_wait_timeouts, 1ull);
      if (c.giveup != nullptr) atomicExch_system(c.giveup, 1);
    }
    for (long long i = 0; i < kBrickWaitLimit && !mbar_try_wait(mbar, 0); ++i) {
    }
    return;
  }
  // halo sites: x = -1 is x = L1 - 1, x = L1 is x = 0
  for (int row = threadIdx.x; row < D::ROWS; row += blockDim.x) {
    float* r = sm + row * D::RS + TILE_PAD;
    r[-1] = r[L1T - 1];
    r[L1T] = r[0];
  }
  __syncthreads();
  const int32_t key = sweep_key_at(c.state, 0);
  const int pairs = (c.bx + 1) >> 1;   // pairs of class sites per row
  const int alpha = p.alpha;
  for (int t = threadIdx.x; t < BZ * BR_Y * pairs; t += blockDim.x) {
    const int jp = t % pairs, r2 = t / pairs, ty = r2 % BR_Y, tz = r2 / BR_Y;
    const int y = y0 + ty, z = z0 + tz;
    const int xa = first_class_x(c, p.colour, alpha, y, z) + 2 * c.P * jp;
    if (xa >= L1T) continue;
    const bool two = xa + c.P < L1T;
    static_for<0, Lat::b>([&](auto ac) {
      constexpr int a = decltype(ac)::value;
      if (a == alpha) brick_pair<Lat, a, N, L1T, BZ>(c, p.J[a], sbase, rep, tz, ty, xa, y, z, two, key);
    });
  }
}

template <class Lat, int N, int L1T, int BZ>
static int launch_brick(const TileParams& p, cudaStream_t s) {
  using D = BrickDims<Lat, N, L1T, BZ>;
  const dim3 grid((p.c.g.L2 / BR_Y) * (p.c.g.L3 / BZ), p.c.B);
  const int rc = cuda_status(cudaFuncSetAttribute(brick_class_kernel<Lat, N, L1T, BZ>,
                                                  cudaFuncAttributeMaxDynamicSharedMemorySize, D::BYTES),
                             "tile shared memory");
  if (rc != SCK_OK) return rc;
  brick_class_kernel<Lat, N, L1T, BZ><<<grid, 256, D::BYTES, s>>>(p);
  return cuda_status(cudaGetLastError(), "tile class launch");
}

template <class Lat, int N, int L1T>
static int launch_tile_lnt(const TileParams& p, cudaStream_t s) {
  if constexpr (Lat::dim == 3)
    return launch_brick<Lat, N, L1T, 4>(p, s);
  else
    return launch_brick<Lat, N, L1T, 1>(p, s);
}

template <class Lat, int N>
static int launch_tile_ln(const TileParams& p, cudaStream_t s) {
  switch (p.c.g.L1) {
    case 32: return launch_tile_lnt<Lat, N, 32>(p, s);
    case 64: return launch_tile_lnt<Lat, N, 64>(p, s);
    default: return launch_tile_lnt<Lat, N, 128>(p, s);
  }
}

template <class Lat>
static int launch_tile_l(const TileParams& p, cudaStream_t s) {
  return p.c.g.n == 2 ? launch_tile_ln<Lat, 2>(p, s) : launch_tile_ln<Lat, 3>(p, s);
}

template <class Lat, int N>
static constexpr int tile_bytes_n(int L1) {
  constexpr int BZ = Lat::dim == 3 ? 4 : 1;
  return L1 == 32 ? BrickDims<Lat, N, 32, BZ>::BYTES
                  : (L1 == 64 ? BrickDims<Lat, N, 64, BZ>::BYTES : BrickDims<Lat, N, 128, BZ>::BYTES);
}

template <class Lat>
static constexpr int tile_bytes(int n, int L1) {
  return n == 2 ? tile_bytes_n<Lat, 2>(L1) : tile_bytes_n<Lat, 3>(L1);
}

static int tile_smem(const sck_plan* plan) {
  const int n = plan->geom.n, L1 = plan->geom.L1;
  switch (plan->spec) {
    case Lat_square_1::id: return tile_bytes<Lat_square_1>(n, L1);
    case Lat_triangular_1::id: return tile_bytes<Lat_triangular_1>(n, L1);
    case Lat_sc_1::id: return tile_bytes<Lat_sc_1>(n, L1);
    case Lat_bcc_1::id: return tile_bytes<Lat_bcc_1>(n, L1);
    case Lat_bcc_1_2::id: return tile_bytes<Lat_bcc_1_2>(n, L1);
    default: return tile_bytes<Lat_fcc_1>(n, L1);
  }
}

bool tile_kernel_ok(const sck_plan* plan) {
  const Geometry& g = plan->geom;
  if (plan->kernel_kind != 3 || plan->spec == 0 || plan->mode != SCK_MODE_F32 || g.n < 2) return false;
  if (plan->Bp > 65535) return false;   // one grid row per replica
  if (g.L1 != 32 && g.L1 != 64 && g.L1 != 128) return false;
  if (!g.per[0] || !g.per[1] || g.L2 % BR_Y != 0 || g.L2 < 3) return false;
  if (g.dim == 3 && (!g.per[2] || g.L3 % 4 != 0 || g.L3 < 4)) return false;
  return tile_smem(plan) <= 220 * 1024;
}

int launch_tile_class(const sck_plan* plan, const Common& c, int colour, int alpha, cudaStream_t s) {
  TileParams p;
  memset(&p, 0, sizeof(p));
  p.c = c;
  for (int a = 0; a < SCK_MAX_BASIS; ++a)
    for (int gi = 0; gi < SCK_MAX_GROUPS; ++gi) p.J[a][gi] = plan->sub[a].J[gi];
  p.colour = colour;
  p.alpha = alpha;
  switch (plan->spec) {
    case Lat_square_1::id: return launch_tile_l<Lat_square_1>(p, s);
    case Lat_triangular_1::id: return launch_tile_l<Lat_triangular_1>(p, s);
    case Lat_sc_1::id: return launch_tile_l<Lat_sc_1>(p, s);
    case Lat_bcc_1::id: return launch_tile_l<Lat_bcc_1>(p, s);
    case Lat_bcc_1_2::id: return launch_tile_l<Lat_bcc_1_2>(p, s);
    default: return launch_tile_l<Lat_fcc_1>(p, s);
  }
}

}  // namespace sck

extern "C" int sck_wait_timeouts(int64_t* count) {
  if (count == nullptr) {
    sck::set_error("null output");
    return SCK_ERR_INVALID;
  }
  unsigned long long v = 0, w = 0, x = 0;
  int rc = sck::cuda_status(cudaMemcpyFromSymbol(&v, sck::g_wait_timeouts, sizeof(v)), "wait timeouts");
  if (rc == SCK_OK) rc = sck::made_wait_timeouts(&w);
  if (rc == SCK_OK) rc = sck::stream_wait_timeouts(&x);
  if (rc != SCK_OK) return rc;
  *count = (int64_t)(v + w + x);
  return SCK_OK;
}
