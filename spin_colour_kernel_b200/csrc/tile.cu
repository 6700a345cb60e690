// Tile kernels: the class update of vector models on a periodic box with a compile-time bond table, reading
// every neighbour from shared memory.
//
// A block of threads owns a band of TILE_TY rows of two replicas and marches along z. It keeps three planes of
// the band (z - 1, z, z + 1), each with one halo row on either side and one halo site at either end of every
// row, in shared memory (both sublattices, every component, float32), filled with cp.async. The class sites of
// plane z then read their neighbours with shared-memory loads at compile-time offsets from three per-site
// pointers (one per plane): the 64-bit address arithmetic that the global-memory kernels spend on every
// neighbour load disappears. Two replicas per thread share the addressing and run the proposal and acceptance in
// packed float32x2 arithmetic (finish_core in spec.cuh). Neighbours are never sites of the class being
// updated, so the shared copies never go stale within a launch. Group sums run in bond order, as in the lattice
// kernels.
#include "spec.cuh"

namespace sck {

constexpr int TILE_TY = 8;    // rows per band
constexpr int TILE_PAD = 4;   // floats before x = 0 in a shared row: x = -1 sits at TILE_PAD - 1

template <class Lat, int N, int L1T>
struct TileDims {
  static_assert(Lat::reach == 1, "tile kernels read neighbours at most one cell away");
  static constexpr int R2 = TILE_TY + 2;               // band rows plus halo rows
  static constexpr int RS = L1T + 2 * TILE_PAD;        // floats per shared row
  static constexpr int COMP = R2 * RS;                 // one component of one sublattice
  static constexpr int REP = Lat::b * N * COMP;        // one replica of one plane
  static constexpr int SLOT = 2 * REP;                 // two replicas
  static constexpr int BYTES = 3 * SLOT * 4;
};

struct TileParams {
  Common c;
  float J[SCK_MAX_BASIS][SCK_MAX_GROUPS];
  int colour, alpha;
};

__device__ __forceinline__ void tile_wait_all() {
  asm volatile("cp.async.commit_group;\n" ::);
  asm volatile("cp.async.wait_group 0;\n" ::);
}

// The rows one thread copies are the same on every plane: rows tid / Q + RSTEP i of the slot (replica,
// sublattice, component, band row), 16-byte chunk tid % Q of each, plus the two halo sites of row tid. Their
// global offsets within a plane and their shared addresses are worked out once; a plane adds its z offset.
template <class Lat, int N, int L1T>
struct TileLoader {
  using D = TileDims<Lat, N, L1T>;
  static constexpr int Q = L1T / 4;                       // 16-byte chunks per row
  static constexpr int RSTEP = 256 / Q;                   // rows per pass of the block
  static constexpr int ROWS = 2 * Lat::b * N * D::R2;     // rows of a slot
  static constexpr int MAXR = (ROWS + RSTEP - 1) / RSTEP;
  static_assert(ROWS <= 256, "one thread per row for the halo sites");
  long long goff[MAXR];   // element offset of the chunk within the pair of replicas, without z
  uint32_t soff[MAXR];    // byte offset of the chunk within a slot
  long long hoff;         // halo sites of row tid: element offset of x = 0 of that row, without z
  uint32_t hs;            // byte offset of x = 0 of that row within a slot
  int nrow;
  bool halo;

  __device__ __forceinline__ TileLoader(const Geometry& g, bool two, int y0) {
    const int q = threadIdx.x % Q;
    nrow = 0;
#pragma unroll
    for (int i = 0; i < MAXR; ++i) {
      const int row = threadIdx.x / Q + RSTEP * i;
      goff[i] = 0;
      soff[i] = 0;
      if (row < ROWS) {
        goff[i] = row_offset(g, two, y0, row) + 4 * q;
        soff[i] = 4u * (uint32_t)(row * D::RS + TILE_PAD + 4 * q);
        nrow = i + 1;
      }
    }
    halo = threadIdx.x < ROWS;
    hoff = halo ? row_offset(g, two, y0, threadIdx.x) : 0;
    hs = 4u * (uint32_t)(threadIdx.x * D::RS + TILE_PAD);
  }
  __device__ __forceinline__ static long long row_offset(const Geometry& g, bool two, int y0, int row) {
    const int r = row % D::R2, akj = row / D::R2, k = akj % N, aj = akj / N, a = aj % Lat::b, j = aj / Lat::b;
    int y = y0 - 1 + r;
    y = y < 0 ? y + g.L2 : (y >= g.L2 ? y - g.L2 : y);
    return (long long)(two ? j : 0) * N * g.nsite + (long long)k * g.nsite + (long long)a * g.plane +
           (long long)y * L1T;
  }
  // plane zu (-1 .. L3, wrapped) into the slot at shared address `slot`
  __device__ __forceinline__ void load(const Geometry& g, const float* src, uint32_t slot, int zu) const {
    const int zz = zu < 0 ? zu + g.L3 : (zu >= g.L3 ? zu - g.L3 : zu);
    const float* base = src + (long long)zz * g.L2 * L1T;
#pragma unroll
    for (int i = 0; i < MAXR; ++i)
      if (i < nrow)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(slot + soff[i]), "l"(base + goff[i]));
    if (halo) {
      asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(slot + hs - 4), "l"(base + hoff + L1T - 1));
      asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(slot + hs + 4 * L1T), "l"(base + hoff));
    }
  }
};

// 32-bit shared-memory load at a compile-time byte offset from a register address
template <int OFF>
__device__ __forceinline__ float lds(uint32_t addr) {
  float v;
  asm volatile("ld.shared.f32 %0, [%1+%2];\n" : "=f"(v) : "r"(addr), "n"(OFF));
  return v;
}

template <class Lat, int A, int N, int L1T>
__device__ __forceinline__ void tile_site(const Common& c, const float (&J)[SCK_MAX_GROUPS], const uint32_t (&pl)[3],
                                          int zu, int ty, int x, int y, int rep0, bool two, int32_t key) {
  using D = TileDims<Lat, N, L1T>;
  const Geometry& g = c.g;
  const int own = A * g.plane + (zu * g.L2 + y) * L1T + x;
  if (g.has_mask && c.mask[own] == 0) return;
  const uint32_t site = 4u * (uint32_t)((ty + 1) * D::RS + TILE_PAD + x);
  // one shared address per plane z - 1, z, z + 1; every neighbour is a compile-time offset from one of them
  const uint32_t pz[3] = {pl[0] + site, pl[1] + site, pl[2] + site};
  float2 s[N], v[N];
  static_for<0, N>([&](auto kc) {
    constexpr int k = decltype(kc)::value;
    constexpr int o = 4 * (A * N + k) * D::COMP;
    s[k] = make_float2(lds<o>(pz[1]), lds<o + 4 * D::REP>(pz[1]));
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
      constexpr int off = 4 * (bd.a2 * N * D::COMP + bd.dy * D::RS + bd.dx);
      const uint32_t q = pz[bd.dz + 1];
      static_for<0, N>([&](auto kc) {
        constexpr int k = decltype(kc)::value;
        gs[k] = __fadd2_rn(gs[k], make_float2(lds<off + 4 * k * D::COMP>(q), lds<off + 4 * (D::REP + k * D::COMP)>(q)));
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
  const int rep1 = two ? rep0 + 1 : rep0;
  finish_pair<N>(c, own, rep0, rep1, two, key, s, v, t, acc0, acc1);
  const size_t NS = (size_t)g.nsite;
  float* po = (float*)c.dst + (size_t)rep0 * N * NS + own;
  if (acc0) {
#pragma unroll
    for (int k = 0; k < N; ++k) po[k * NS] = t[k].x;
  }
  if (two && acc1) {
#pragma unroll
    for (int k = 0; k < N; ++k) po[(N + k) * NS] = t[k].y;
  }
}

// Grid (L2 / TILE_TY bands, ceil(B / 2) replica pairs), 256 threads.
template <class Lat, int N, int L1T>
__global__ void __launch_bounds__(256) tile_class_kernel(const __grid_constant__ TileParams p) {
  extern __shared__ __align__(16) float sm[];
  const Common& c = p.c;
  const Geometry& g = c.g;
  const int y0 = blockIdx.x * TILE_TY;
  const int rep0 = 2 * blockIdx.y;
  const bool two = rep0 + 1 < c.B;
  const float* src0 = (const float*)c.src + (size_t)rep0 * N * g.nsite;
  const TileLoader<Lat, N, L1T> ld(g, two, y0);
  const uint32_t sbase = (uint32_t)__cvta_generic_to_shared(sm);
  constexpr uint32_t SLOT_BYTES = 4u * TileDims<Lat, N, L1T>::SLOT;
  ld.load(g, src0, sbase + 2 * SLOT_BYTES, -1);
  ld.load(g, src0, sbase, 0);
  ld.load(g, src0, sbase + SLOT_BYTES, 1);
  tile_wait_all();
  __syncthreads();
  const int32_t key = sweep_key_at(c.state, 0);
  const int spr = c.bx;                      // class sites per row at most
  const int alpha = p.alpha;
  uint32_t pl[3] = {sbase + 2 * SLOT_BYTES, sbase, sbase + SLOT_BYTES};   // planes zu - 1, zu, zu + 1 at zu = 0
  for (int zu = 0; zu < g.L3; ++zu) {
    for (int t = threadIdx.x; t < TILE_TY * spr; t += blockDim.x) {
      const int ty = t / spr, j = t - ty * spr;
      const int y = y0 + ty;
      const int x = first_class_x(c, p.colour, alpha, y, zu) + c.P * j;
      if (x >= L1T) continue;
      static_for<0, Lat::b>([&](auto ac) {
        constexpr int a = decltype(ac)::value;
        if (a == alpha) tile_site<Lat, a, N, L1T>(c, p.J[a], pl, zu, ty, x, y, rep0, two, key);
      });
    }
    const uint32_t rot = pl[0];   // the ring turns: zu's slot becomes z - 1, zu + 1's becomes z
    pl[0] = pl[1];
    pl[1] = pl[2];
    pl[2] = rot;
    __syncthreads();   // every thread is done with plane zu - 1
    if (zu + 1 < g.L3) {
      ld.load(g, src0, pl[2], zu + 2);
      tile_wait_all();
      __syncthreads();
    }
  }
}

template <class Lat, int N, int L1T>
static int launch_tile_lnt(const TileParams& p, cudaStream_t s) {
  using D = TileDims<Lat, N, L1T>;
  const dim3 grid(p.c.g.L2 / TILE_TY, (p.c.B + 1) / 2);
  const int rc = cuda_status(cudaFuncSetAttribute(tile_class_kernel<Lat, N, L1T>,
                                                  cudaFuncAttributeMaxDynamicSharedMemorySize, D::BYTES),
                             "tile shared memory");
  if (rc != SCK_OK) return rc;
  tile_class_kernel<Lat, N, L1T><<<grid, 256, D::BYTES, s>>>(p);
  return cuda_status(cudaGetLastError(), "tile class launch");
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

template <class Lat>
static constexpr int tile_bytes(int n, int L1) {
  return n == 2 ? (L1 == 32 ? TileDims<Lat, 2, 32>::BYTES : L1 == 64 ? TileDims<Lat, 2, 64>::BYTES
                                                                      : TileDims<Lat, 2, 128>::BYTES)
                : (L1 == 32 ? TileDims<Lat, 3, 32>::BYTES : L1 == 64 ? TileDims<Lat, 3, 64>::BYTES
                                                                      : TileDims<Lat, 3, 128>::BYTES);
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
  if (g.L1 != 32 && g.L1 != 64 && g.L1 != 128) return false;
  if (!g.per[0] || !g.per[1] || g.L2 % TILE_TY != 0) return false;
  if (g.dim == 3 && (!g.per[2] || g.L3 < 3)) return false;
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
