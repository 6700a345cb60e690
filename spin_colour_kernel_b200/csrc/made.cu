// Learned block proposal for 3D Ising (include/sck_made.h): a masked autoregressive MLP (MADE) over the 64
// spins of a 4x4x4 block, conditioned on its 96 boundary spins, proposes a joint block update whose exact
// density enters a Metropolis-Hastings ratio. No counterpart in the reference.
//
// Tensor cores run every product: bfloat16 operands, FP32 accumulation, mma.sync.m16n8k16 fed by ldmatrix
// from shared memory.
//   * Training: one tiled GEMM kernel (64x64x32 tiles, cp.async double buffering) in the three layouts of a
//     dense layer's forward, data-gradient and weight-gradient products; the weight gradient reduces over the
//     batch in split-K partials that a finishing kernel sums in a fixed order (deterministic), masks and
//     feeds to Adam, which also rewrites the bfloat16 masked copies.
//   * Sampling: one warp carries 8 blocks through the autoregressive steps as a 16-row tile: rows 0-7 draw the
//     proposal x', rows 8-15 re-evaluate the current spins x under the same weights, so q(x' | b) and
//     q(x | b) come out of the same arithmetic. Step g computes only the hidden units of degree g in each
//     layer (their inputs are final) and the logits of group g, then draws the group's spins. The MMA
//     accumulator of the lane that owns block r holds both its proposal and its current-state logits.
#include <mutex>
#include <string>

#include <cuda_bf16.h>

#include "../../include/sck_made.h"
#include "internal.h"

namespace sck {
namespace made {

constexpr int IN = SCK_MADE_IN, H = SCK_MADE_HIDDEN, NSP = SCK_MADE_SPINS, NBD = SCK_MADE_BOUNDARY;
// layer l (0..3): rows (outputs) and columns (inputs) of its weight matrix
__host__ __device__ constexpr int out_rows(int l) { return l < 3 ? H : NSP; }
__host__ __device__ constexpr int in_cols(int l) { return l == 0 ? IN : H; }
// FP32 masters (offsets in floats): W_l then b_l, layer after layer
__host__ __device__ constexpr long long off_w(int l) {
  return l == 0 ? 0 : off_w(l - 1) + (long long)out_rows(l - 1) * in_cols(l - 1) + out_rows(l - 1);
}
__host__ __device__ constexpr long long off_b(int l) { return off_w(l) + (long long)out_rows(l) * in_cols(l); }
constexpr long long NPARAM = SCK_MADE_NPARAM;
static_assert(off_b(3) + NSP == NPARAM, "parameter layout");
// bfloat16 masked copies: 8 zero rows of padding after each matrix (the sampler's last n-tiles read them)
constexpr int PAD_ROWS = 8;
__host__ __device__ constexpr long long off_bf(int l) {
  return l == 0 ? 0 : off_bf(l - 1) + (long long)(out_rows(l - 1) + PAD_ROWS) * in_cols(l - 1);
}
constexpr long long NBF = off_bf(3) + (long long)(NSP + PAD_ROWS) * H;

inline long long align256(long long x) { return (x + 255) & ~255ll; }
constexpr long long BF_BASE_BYTES = ((NPARAM * 4) + 255) & ~255ll;

__host__ __device__ inline const __nv_bfloat16* bf_weights(const void* params, int layer) {
  return (const __nv_bfloat16*)((const char*)params + BF_BASE_BYTES) + off_bf(layer);
}

// ------------------------------------------------------------------------------------------ degrees, masks
__host__ __device__ inline int deg_in(int i, int S) { return i < NBD ? 0 : (i - NBD) / S + 1; }
__host__ __device__ inline int deg_hidden(int k, int G) { return k * G / H; }
// connection of output row n to input column k in layer l (0..3)
__host__ __device__ inline bool connected(int l, int n, int k, int G) {
  const int S = NSP / G;
  if (l == 0) return deg_in(k, S) <= deg_hidden(n, G);
  if (l < 3) return deg_hidden(k, G) <= deg_hidden(n, G);
  return deg_hidden(k, G) <= n / S;
}

// ---------------------------------------------------------------------------------------- PTX wrappers
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void ldsm_x4(uint32_t (&r)[4], const void* p) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(smem_u32(p)));
}
__device__ __forceinline__ void ldsm_x4_t(uint32_t (&r)[4], const void* p) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(smem_u32(p)));
}
__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}
// 16-byte global -> shared copy; src_bytes 0 fills zeros
__device__ __forceinline__ void cp_async16(void* dst, const void* src, int src_bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(smem_u32(dst)), "l"(src), "r"(src_bytes));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}
__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<uint32_t*>(&v);
}

// ================================================================================================ GEMM
// C[M x N] = sum_k A(m, k) B(k, n) over k in [z kchunk, (z+1) kchunk) (z = blockIdx.z), with
//   A(m, k) = A[m lda + k] (A_K) or A[k lda + m];   B(k, n) = B[n ldb + k] (B_K) or B[k ldb + n].
// M, the chunk and K are multiples of the tile sizes; N a multiple of 32 (columns past N read as zero and
// are not stored).
enum Epi { EPI_BIAS_RELU_BF16 = 0, EPI_BIAS_F32 = 1, EPI_GATE_BF16 = 2, EPI_F32 = 3 };
constexpr int BM = 64, BN = 64, BK = 32;

struct GemmArgs {
  const __nv_bfloat16* A;
  const __nv_bfloat16* B;
  int M, N, K, kchunk;
  long long lda, ldb, ldc, split_stride;
  void* C;
  const float* bias;
  const __nv_bfloat16* gate;   // EPI_GATE_BF16: C = acc where gate > 0, else 0 (gate laid out like C)
};

template <bool A_K, bool B_K, int EPI>
__global__ void __launch_bounds__(128) gemm_kernel(GemmArgs g) {
  constexpr int A_ROWS = A_K ? BM : BK, A_COLS = (A_K ? BK : BM) + 8;
  constexpr int B_ROWS = B_K ? BN : BK, B_COLS = (B_K ? BK : BN) + 8;
  __shared__ __align__(128) __nv_bfloat16 As[2][A_ROWS * A_COLS];
  __shared__ __align__(128) __nv_bfloat16 Bs[2][B_ROWS * B_COLS];

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
  const int kbeg = blockIdx.z * g.kchunk;
  const int kend = min(g.K, kbeg + g.kchunk);
  const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;

  auto load_tile = [&](int stage, int k0) {
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      const int c = tid + i * 128;
      if (A_K) {
        const int r = c >> 2, c8 = (c & 3) * 8;
        cp_async16(&As[stage][r * A_COLS + c8], g.A + (long long)(m0 + r) * g.lda + k0 + c8, 16);
      } else {
        const int r = c >> 3, c8 = (c & 7) * 8;
        cp_async16(&As[stage][r * A_COLS + c8], g.A + (long long)(k0 + r) * g.lda + m0 + c8, 16);
      }
      if (B_K) {
        const int r = c >> 2, c8 = (c & 3) * 8;
        const bool ok = n0 + r < g.N;
        cp_async16(&Bs[stage][r * B_COLS + c8], g.B + (long long)(ok ? n0 + r : 0) * g.ldb + k0 + c8, ok ? 16 : 0);
      } else {
        const int r = c >> 3, c8 = (c & 7) * 8;
        const bool ok = n0 + c8 < g.N;
        cp_async16(&Bs[stage][r * B_COLS + c8], g.B + (long long)(k0 + r) * g.ldb + (ok ? n0 + c8 : 0), ok ? 16 : 0);
      }
    }
    cp_async_commit();
  };

  float acc[2][4][4];
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int e = 0; e < 4; ++e) acc[i][j][e] = 0.f;

  const int nk = (kend - kbeg) / BK;
  if (nk > 0) load_tile(0, kbeg);
  for (int it = 0; it < nk; ++it) {
    const int st = it & 1;
    if (it + 1 < nk) {
      load_tile(st ^ 1, kbeg + (it + 1) * BK);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < BK; kk += 16) {
      uint32_t a[2][4], b[2][4];
#pragma unroll
      for (int mt = 0; mt < 2; ++mt) {
        const int mb = wm + mt * 16;
        if (A_K) {
          ldsm_x4(a[mt], &As[st][(mb + (lane & 7) + ((lane >> 3) & 1) * 8) * A_COLS + kk + (lane >> 4) * 8]);
        } else {
          ldsm_x4_t(a[mt], &As[st][(kk + (lane >> 4) * 8 + (lane & 7)) * A_COLS + mb + ((lane >> 3) & 1) * 8]);
        }
      }
#pragma unroll
      for (int np = 0; np < 2; ++np) {
        const int nb = wn + np * 16;
        if (B_K) {
          ldsm_x4(b[np], &Bs[st][(nb + (lane >> 4) * 8 + (lane & 7)) * B_COLS + kk + ((lane >> 3) & 1) * 8]);
        } else {
          ldsm_x4_t(b[np], &Bs[st][(kk + ((lane >> 3) & 1) * 8 + (lane & 7)) * B_COLS + nb + (lane >> 4) * 8]);
        }
      }
#pragma unroll
      for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) mma_bf16(acc[mt][nt], a[mt], b[nt >> 1][(nt & 1) * 2], b[nt >> 1][(nt & 1) * 2 + 1]);
    }
    __syncthreads();
  }

  const int gr = lane >> 2, q = lane & 3;
#pragma unroll
  for (int mt = 0; mt < 2; ++mt)
#pragma unroll
    for (int nt = 0; nt < 4; ++nt) {
      const int n = n0 + wn + nt * 8 + 2 * q;
      if (n >= g.N) continue;
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int m = m0 + wm + mt * 16 + gr + 8 * h;
        float v0 = acc[mt][nt][2 * h], v1 = acc[mt][nt][2 * h + 1];
        const long long o = (long long)m * g.ldc + n;
        if (EPI == EPI_BIAS_RELU_BF16) {
          v0 = fmaxf(v0 + g.bias[n], 0.f);
          v1 = fmaxf(v1 + g.bias[n + 1], 0.f);
          *(uint32_t*)((__nv_bfloat16*)g.C + o) = pack_bf16(v0, v1);
        } else if (EPI == EPI_BIAS_F32) {
          *(float2*)((float*)g.C + o) = make_float2(v0 + g.bias[n], v1 + g.bias[n + 1]);
        } else if (EPI == EPI_GATE_BF16) {
          const __nv_bfloat162 gt = *(const __nv_bfloat162*)(g.gate + o);
          v0 = __bfloat162float(gt.x) > 0.f ? v0 : 0.f;
          v1 = __bfloat162float(gt.y) > 0.f ? v1 : 0.f;
          *(uint32_t*)((__nv_bfloat16*)g.C + o) = pack_bf16(v0, v1);
        } else {
          *(float2*)((float*)g.C + (long long)blockIdx.z * g.split_stride + o) = make_float2(v0, v1);
        }
      }
    }
}

// ================================================================================ tcgen05 forward GEMM
// C[M x N] = epilogue(A[M x K] B[N x K]^T) for the forward layers (both operands K-major), on the fifth-generation
// tensor cores: a block of 128 threads owns 128 rows and all N columns; per 32-wide K chunk the threads stage
// A and B in shared memory in the canonical no-swizzle K-major layout (8-row x 16-byte core matrices: 128 bytes
// apart along M or N, 16 x 128 bytes apart along K), one thread issues two tcgen05.mma (M 128, N, K 16, bf16
// in, FP32 accumulating in tensor memory) and commits them to an mbarrier that all threads wait on (bounded)
// before the next chunk overwrites the stage. The epilogue reads the accumulator with tcgen05.ld (warp w reads
// rows 32 w .. 32 w + 31) and applies bias, ReLU and the bfloat16 conversion.
constexpr int UM = 128;     // rows per block (MMA M)
constexpr int UKC = 32;     // K per staged chunk (two K16 MMAs)
constexpr long long kUmmaWaitLimit = 1ll << 22;

static __device__ unsigned long long g_made_wait_timeouts;
// polls of a stage's mbarrier before the forward GEMM gives up (sck_made_set_wait_limit; the drain after a give-up
// always keeps kUmmaWaitLimit, so that no product is in flight when the block frees its tensor memory)
static __device__ long long g_made_wait_limit = kUmmaWaitLimit;

__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;   // descriptor version of sm100; base offset 0, no swizzle
  return d;
}

__device__ __forceinline__ bool umma_try_wait(uint32_t mbar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(mbar), "r"(parity)
      : "memory");
  return ok != 0;
}

template <int N, int EPI>
__global__ void __launch_bounds__(128) umma_gemm_kernel(GemmArgs g) {
  // two stages: the copies of chunk ch + 1 run while the tensor cores multiply chunk ch
  extern __shared__ __align__(1024) unsigned char usm[];
  __nv_bfloat16* As = (__nv_bfloat16*)usm;                                    // [2][UM * UKC]
  __nv_bfloat16* Bs = (__nv_bfloat16*)(usm + 2 * UM * UKC * 2);               // [2][N * UKC]
  uint64_t* mbar = (uint64_t*)(usm + 2 * (UM + N) * UKC * 2);                 // [2]
  uint32_t* tmem_slot = (uint32_t*)(mbar + 2);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.x * UM;
  const uint32_t mb0 = smem_u32(mbar), mb1 = smem_u32(mbar + 1);
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(tmem_slot)),
                 "r"(N < 32 ? 32 : N)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(mb0) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(mb1) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  const uint32_t tmem = *tmem_slot;
  constexpr uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) |
                             ((uint32_t)(UM >> 4) << 24);   // FP32 accumulator, bf16 A and B, K-major
  constexpr uint32_t A_LBO = (UM / 8) * 128, B_LBO = (N / 8) * 128;
  const int nch = g.K / UKC;
  auto stage = [&](int ch) {
    const int k0 = ch * UKC, b = ch & 1;
    __nv_bfloat16* as = As + b * UM * UKC;
    __nv_bfloat16* bs = Bs + b * N * UKC;
    for (int i = tid; i < UM * (UKC / 8); i += 128) {
      const int r = i / (UKC / 8), c = i % (UKC / 8);
      cp_async16(as + ((c * (UM / 8) + (r >> 3)) * 64 + (r & 7) * 8), g.A + (long long)(m0 + r) * g.lda + k0 + 8 * c,
                 16);
    }
    for (int i = tid; i < N * (UKC / 8); i += 128) {
      const int n = i / (UKC / 8), c = i % (UKC / 8);
      cp_async16(bs + ((c * (N / 8) + (n >> 3)) * 64 + (n & 7) * 8), g.B + (long long)n * g.ldb + k0 + 8 * c, 16);
    }
    cp_async_commit();
  };
  // bounded wait of every thread on a stage's mbarrier; false (for the whole block) when it gave up
  uint32_t ph[2] = {0u, 0u};
  auto wait_stage = [&](int b) {
    const uint32_t mb = b ? mb1 : mb0;
    long long polls = 0;
    bool done = false;
    const long long limit = g_made_wait_limit;
    while (polls < limit && !(done = umma_try_wait(mb, ph[b]))) ++polls;
    ph[b] ^= 1u;
    return !__syncthreads_or(!done);
  };
  bool ok = true;
  int pending = -1;   // stage whose products the timeout path must still drain
  stage(0);
  for (int ch = 0; ch < nch && ok; ++ch) {
    const int b = ch & 1;
    if (ch + 1 < nch) {
      if (ch >= 1) {   // chunk ch - 1 used the other stage: its products must be done before it is refilled
        ok = wait_stage(b ^ 1);
        if (!ok) {
          pending = b ^ 1;
          break;
        }
      }
      stage(ch + 1);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");   // the tensor cores read what we wrote
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
      const uint32_t a_s = smem_u32(As + b * UM * UKC), b_s = smem_u32(Bs + b * N * UKC);
#pragma unroll
      for (int s = 0; s < UKC / 16; ++s) {
        const uint64_t ad = umma_desc(a_s + s * 2 * A_LBO, A_LBO, 128);
        const uint64_t bd = umma_desc(b_s + s * 2 * B_LBO, B_LBO, 128);
        const uint32_t acc = (ch > 0 || s > 0) ? 1u : 0u;
        asm volatile(
            "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
            " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n}\n" ::"r"(tmem),
            "l"(ad), "l"(bd), "r"(idesc), "r"(acc), "r"(0u)
            : "memory");
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(b ? mb1 : mb0)
                   : "memory");
    }
  }
  if (ok) {   // the last commit covers every product issued before it
    ok = wait_stage((nch - 1) & 1);
    if (!ok) pending = (nch - 1) & 1;
  }
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  if (ok) {
    const int row = m0 + 32 * warp + lane;
#pragma unroll 1
    for (int col = 0; col < N; col += 8) {
      uint32_t v[8];
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];\n"
          : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
          : "r"(tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)col));
      asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
      float f[8];
#pragma unroll
      for (int e = 0; e < 8; ++e) f[e] = __uint_as_float(v[e]) + g.bias[col + e];
      if (EPI == EPI_BIAS_RELU_BF16) {
        uint4 o;
        o.x = pack_bf16(fmaxf(f[0], 0.f), fmaxf(f[1], 0.f));
        o.y = pack_bf16(fmaxf(f[2], 0.f), fmaxf(f[3], 0.f));
        o.z = pack_bf16(fmaxf(f[4], 0.f), fmaxf(f[5], 0.f));
        o.w = pack_bf16(fmaxf(f[6], 0.f), fmaxf(f[7], 0.f));
        *(uint4*)((__nv_bfloat16*)g.C + (long long)row * g.ldc + col) = o;
      } else {
        float* o = (float*)g.C + (long long)row * g.ldc + col;
        *(float4*)o = make_float4(f[0], f[1], f[2], f[3]);
        *(float4*)(o + 4) = make_float4(f[4], f[5], f[6], f[7]);
      }
    }
  } else {
    if (tid == 0) atomicAdd(&g_made_wait_timeouts, 1ull);
    // products of the stage that timed out may still run: wait for them, bounded, before freeing their memory
    const uint32_t mb = pending ? mb1 : mb0;
    for (long long i = 0; i < kUmmaWaitLimit && !umma_try_wait(mb, ph[pending] ^ 1u); ++i) {
    }
    cp_async_wait<0>();
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(N < 32 ? 32 : N)
                 : "memory");
}

template <int N>
constexpr int umma_smem() { return 2 * (UM + N) * UKC * 2 + 16 + 16; }

}  // namespace made

int made_wait_timeouts(unsigned long long* v) {
  return cuda_status(cudaMemcpyFromSymbol(v, made::g_made_wait_timeouts, sizeof(*v)), "learned wait timeouts");
}

int made_set_wait_limit(long long polls) {
  return cuda_status(cudaMemcpyToSymbol(made::g_made_wait_limit, &polls, sizeof(polls)), "learned wait limit");
}

namespace made {

template <int N, int EPI>
int umma_gemm_n(const GemmArgs& g, cudaStream_t s) {
  const int rc = cuda_status(cudaFuncSetAttribute(umma_gemm_kernel<N, EPI>,
                                                  cudaFuncAttributeMaxDynamicSharedMemorySize, umma_smem<N>()),
                             "made tcgen05 gemm smem");
  if (rc != SCK_OK) return rc;
  umma_gemm_kernel<N, EPI><<<dim3(g.M / UM), 128, umma_smem<N>(), s>>>(g);
  return cuda_status(cudaGetLastError(), "made tcgen05 gemm");
}

template <int EPI>
int umma_gemm(const GemmArgs& g, cudaStream_t s) {
  return g.N == H ? umma_gemm_n<H, EPI>(g, s) : umma_gemm_n<NSP, EPI>(g, s);
}

template <bool A_K, bool B_K, int EPI>
int gemm(const GemmArgs& g, int splits, cudaStream_t s) {
  dim3 grid((g.N + BN - 1) / BN, g.M / BM, splits);
  gemm_kernel<A_K, B_K, EPI><<<grid, 128, 0, s>>>(g);
  return cuda_status(cudaGetLastError(), "made gemm");
}

// ======================================================================================= small kernels
__global__ void prepare_kernel(const float* __restrict__ master, __nv_bfloat16* __restrict__ bf, int G) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= NBF) return;
  int l = 3;
  while (l > 0 && i < off_bf(l)) --l;
  const long long j = i - off_bf(l);
  const int K = in_cols(l);
  const int n = (int)(j / K), k = (int)(j % K);
  float v = 0.f;
  if (n < out_rows(l) && connected(l, n, k, G)) v = master[off_w(l) + (long long)n * K + k];
  bf[i] = __float2bfloat16_rn(v);
}

// loss, log q and the logit gradient -x sigmoid(-x l) / M (bfloat16) of rows of logits
__global__ void loss_kernel(const float* __restrict__ logits, const __nv_bfloat16* __restrict__ x, int M,
                            __nv_bfloat16* __restrict__ grad, float* __restrict__ logq, float* __restrict__ loss) {
  const int row = blockIdx.x * 4 + (threadIdx.x >> 6);
  const int p = threadIdx.x & 63;
  float lq = 0.f;
  if (row < M) {
    const float l = logits[(long long)row * NSP + p];
    const float s = __bfloat162float(x[(long long)row * IN + NBD + p]);
    const float t = s * l;
    // log sigmoid(t) = -(max(-t, 0) + log1p(exp(-|t|)))
    lq = -(fmaxf(-t, 0.f) + log1pf(expf(-fabsf(t))));
    if (grad) grad[(long long)row * NSP + p] = __float2bfloat16_rn(-s / (1.f + expf(t)) / (float)M);
  }
  // 64 lanes of a row: two warps
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) lq += __shfl_xor_sync(0xffffffffu, lq, o);
  __shared__ float part[8];
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = lq;
  __syncthreads();
  if (threadIdx.x < 4) {
    const int r = blockIdx.x * 4 + threadIdx.x;
    const float v = part[2 * threadIdx.x] + part[2 * threadIdx.x + 1];
    if (r < M) {
      if (logq) logq[r] = v;
      if (loss) atomicAdd(loss, -v / (float)M);
    }
  }
}

// column sums of a bfloat16 [M x N] matrix over row chunks: out[z][n]
__global__ void colsum_kernel(const __nv_bfloat16* __restrict__ g, int M, int N, int chunk, float* __restrict__ out) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  const int r0 = blockIdx.y * chunk, r1 = min(M, r0 + chunk);
  float s = 0.f;
  for (int r = r0; r < r1; ++r) s += __bfloat162float(g[(long long)r * N + n]);
  out[(long long)blockIdx.y * N + n] = s;
}

struct FinishArgs {
  const float* wpart[4];   // [splits][rows][cols]
  const float* bpart[4];   // [splits][rows]
  int splits;
  int G;
  int adam;                // 0: write gradients; 1: Adam step on the masters
  float* grads;            // master layout
  float* master;
  float* m1;
  float* m2;
  __nv_bfloat16* bf;
  float lr, beta1, beta2, eps, c1, c2;   // c1 = 1 - beta1^t, c2 = 1 - beta2^t
};

__global__ void finish_kernel(FinishArgs a) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= NPARAM) return;
  int l = 3;
  while (l > 0 && i < off_w(l)) --l;
  const long long j = i - off_w(l);
  const int K = in_cols(l), R = out_rows(l);
  float g = 0.f;
  bool weight = j < (long long)R * K, live = true;
  int n = 0, k = 0;
  if (weight) {
    n = (int)(j / K);
    k = (int)(j % K);
    live = connected(l, n, k, a.G);
    if (live)
      for (int z = 0; z < a.splits; ++z) g += a.wpart[l][((long long)z * R + n) * K + k];
  } else {
    n = (int)(j - (long long)R * K);
    for (int z = 0; z < a.splits; ++z) g += a.bpart[l][(long long)z * R + n];
  }
  if (!a.adam) {
    a.grads[i] = live ? g : 0.f;
    return;
  }
  float w = a.master[i];
  if (live) {
    const float m = a.beta1 * a.m1[i] + (1.f - a.beta1) * g;
    const float v = a.beta2 * a.m2[i] + (1.f - a.beta2) * g * g;
    a.m1[i] = m;
    a.m2[i] = v;
    w -= a.lr * (m / a.c1) / (sqrtf(v / a.c2) + a.eps);
    a.master[i] = w;
  }
  if (weight) a.bf[off_bf(l) + (long long)n * K + k] = __float2bfloat16_rn(live ? w : 0.f);
}

// ================================================================================== block geometry tables
struct Tables {
  int8_t in_off[IN][3];     // local offset (dx, dy, dz) of input column i from the block origin
  int8_t pos_of_raster[NSP];
  int8_t raster_of_pos[NSP];
  int8_t internal[144][2];  // positions
  int8_t face[NBD];         // position of the block spin next to boundary spin q
};
__constant__ Tables c_tab;

static Tables host_tables() {
  Tables t{};
  static const int subs[8][3] = {{0, 0, 0}, {1, 1, 0}, {1, 0, 1}, {0, 1, 1}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {1, 1, 1}};
  int p = 0;
  for (auto& s : subs)
    for (int lz = s[2]; lz < 4; lz += 2)
      for (int ly = s[1]; ly < 4; ly += 2)
        for (int lx = s[0]; lx < 4; lx += 2) {
          const int r = lx + 4 * ly + 16 * lz;
          t.raster_of_pos[p] = (int8_t)r;
          t.pos_of_raster[r] = (int8_t)p;
          ++p;
        }
  int q = 0;
  for (int axis = 0; axis < 3; ++axis)
    for (int side : {-1, 4}) {
      int o0 = axis == 0 ? 1 : 0, o1 = axis == 2 ? 1 : 2;
      for (int b = 0; b < 4; ++b)
        for (int a = 0; a < 4; ++a) {
          int c[3] = {0, 0, 0};
          c[axis] = side;
          c[o0] = a;
          c[o1] = b;
          for (int d = 0; d < 3; ++d) t.in_off[q][d] = (int8_t)c[d];
          int cc[3] = {c[0] < 0 ? 0 : (c[0] > 3 ? 3 : c[0]), c[1] < 0 ? 0 : (c[1] > 3 ? 3 : c[1]),
                       c[2] < 0 ? 0 : (c[2] > 3 ? 3 : c[2])};
          t.face[q] = t.pos_of_raster[cc[0] + 4 * cc[1] + 16 * cc[2]];
          ++q;
        }
    }
  for (int pp = 0; pp < NSP; ++pp) {
    const int r = t.raster_of_pos[pp];
    t.in_off[NBD + pp][0] = (int8_t)(r & 3);
    t.in_off[NBD + pp][1] = (int8_t)((r >> 2) & 3);
    t.in_off[NBD + pp][2] = (int8_t)(r >> 4);
  }
  int n = 0;
  for (int lz = 0; lz < 4; ++lz)
    for (int ly = 0; ly < 4; ++ly)
      for (int lx = 0; lx < 4; ++lx) {
        const int r = lx + 4 * ly + 16 * lz;
        const int d[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
        for (auto& dd : d) {
          const int x2 = lx + dd[0], y2 = ly + dd[1], z2 = lz + dd[2];
          if (x2 < 4 && y2 < 4 && z2 < 4) {
            t.internal[n][0] = t.pos_of_raster[r];
            t.internal[n][1] = t.pos_of_raster[x2 + 4 * y2 + 16 * z2];
            ++n;
          }
        }
      }
  return t;
}

static std::mutex g_tab_lock;
static bool g_tab_ready[256] = {};

static int ensure_tables() {
  int dev = 0;
  int rc = cuda_status(cudaGetDevice(&dev), "made device");
  if (rc) return rc;
  std::lock_guard<std::mutex> lk(g_tab_lock);
  if (dev >= 0 && dev < 256 && g_tab_ready[dev]) return SCK_OK;
  const Tables t = host_tables();
  rc = cuda_status(cudaMemcpyToSymbol(c_tab, &t, sizeof(t)), "made tables");
  if (rc) return rc;
  if (dev >= 0 && dev < 256) g_tab_ready[dev] = true;
  return SCK_OK;
}

// block inputs of every block of R replicas (training data)
__global__ void gather_kernel(const int8_t* __restrict__ spins, int R, int L, __nv_bfloat16* __restrict__ out) {
  const int nb = L >> 2;
  const long long nblk = (long long)R * nb * nb * nb;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nblk * IN) return;
  const long long blk = i / IN;
  const int col = (int)(i % IN);
  const int rep = (int)(blk / ((long long)nb * nb * nb));
  const int b = (int)(blk % ((long long)nb * nb * nb));
  const int x0 = (b % nb) * 4, y0 = (b / nb % nb) * 4, z0 = (b / (nb * nb)) * 4;
  const int x = (x0 + c_tab.in_off[col][0] + L) % L, y = (y0 + c_tab.in_off[col][1] + L) % L,
            z = (z0 + c_tab.in_off[col][2] + L) % L;
  const int8_t s = spins[(((long long)rep * L + z) * L + y) * L + x];
  out[i] = __float2bfloat16_rn((float)s);
}

// ======================================================================================= the colour step
constexpr int XS = IN + 8;     // shared row strides (bfloat16): conflict-free ldmatrix rows
constexpr int HS = H + 8;
constexpr int WARP_SMEM = 16 * XS * 2 + 3 * 16 * HS * 2;   // one 16-row tile: inputs and three layers
constexpr int STEP_WARPS = 5;                                 // 16-row tiles per block of threads

// The weights one autoregressive step reads, staged per block of threads: rows [u0, u0 + 8 NT) of W1 (all 160
// columns) and of W2, W3 (the 16 nkt columns of degree <= g), rows [S g, S g + 8) of W4.
template <int G>
struct Slice {
  static constexpr int U = H / G, S = NSP / G, NT = U >= 8 ? U / 8 : 1, NR = 8 * NT;
  static constexpr int W1 = 0, W2 = NR * XS, W3 = W2 + NR * HS, W4 = W3 + NR * HS, ELEMS = W4 + 8 * HS;
  static constexpr int BYTES = ELEMS * 2;
};

template <int G>
constexpr int step_smem() { return STEP_WARPS * WARP_SMEM + 2 * Slice<G>::BYTES; }

// Warps per 16-row tile: with two n8 tiles of new units per layer and step (G = 16), a pair of warps shares the
// tile, each computing one n8 tile of every layer, so that a step's chain of dependent MMAs is half as long and
// the SM holds twice the warps; the logits, the draws and the acceptance stay with the first warp of the pair.
template <int G>
constexpr int tile_warps() { return Slice<G>::NT >= 2 ? 2 : 1; }
template <int G>
constexpr int step_threads() { return 32 * STEP_WARPS * tile_warps<G>(); }

// the two warps of a tile meet at named barrier 1 + tile (barrier 0 is __syncthreads)
__device__ __forceinline__ void tile_sync(int tile, int warps) {
  if (warps > 1) asm volatile("bar.sync %0, %1;\n" ::"r"(1 + tile), "r"(32 * warps) : "memory");
}

struct StepParams {
  const __nv_bfloat16* W[4];
  const float* bias[4];
  int8_t* spins;
  const float* beta;
  int R, L, nb, nc, colour;
  uint32_t k0, k1;
  int32_t* accepted;
  unsigned char* record;
};

__device__ __forceinline__ float log_sigmoid(float t) { return -(fmaxf(-t, 0.f) + __logf(1.f + __expf(-fabsf(t)))); }

__device__ __forceinline__ void ldsm_x2(uint32_t& r0, uint32_t& r1, const void* p) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x2.shared.b16 {%0,%1}, [%2];\n" : "=r"(r0), "=r"(r1) : "r"(smem_u32(p)));
}

// all threads of the block: copy step g's weight slice into `dst` (cp.async, committed as one group)
template <int G>
__device__ __forceinline__ void load_slice(__nv_bfloat16* dst, const StepParams& p, int g) {
  using SL = Slice<G>;
  const int u0 = g * SL::U;
  const int nkt = (SL::U * (g + 1) + 15) / 16;
  const int c1 = IN / 8, ch = 2 * nkt;
  const int n1 = SL::NR * c1, n2 = SL::NR * ch, n4 = 8 * ch;
  const int total = n1 + 2 * n2 + n4;
  for (int i = threadIdx.x; i < total; i += blockDim.x) {
    const __nv_bfloat16* src;
    __nv_bfloat16* d;
    if (i < n1) {
      const int r = i / c1, c = i - r * c1;
      src = p.W[0] + (long long)(u0 + r) * IN + c * 8;
      d = dst + SL::W1 + r * XS + c * 8;
    } else if (i < n1 + 2 * n2) {
      const int j = i - n1, l = j < n2 ? 1 : 2, jj = j - (l - 1) * n2;
      const int r = jj / ch, c = jj - r * ch;
      src = (l == 1 ? p.W[1] : p.W[2]) + (long long)(u0 + r) * H + c * 8;
      d = dst + (l == 1 ? SL::W2 : SL::W3) + r * HS + c * 8;
    } else {
      const int j = i - n1 - 2 * n2, r = j / ch, c = j - r * ch;
      src = p.W[3] + (long long)(g * SL::S + r) * H + c * 8;
      d = dst + SL::W4 + r * HS + c * 8;
    }
    cp_async16(d, src, 16);
  }
  cp_async_commit();
}

template <int NT>
__device__ __forceinline__ void stage_tile(float (&c)[NT][4], const __nv_bfloat16* arow, const __nv_bfloat16* B,
                                           int ldb, int k, int lane) {
  uint32_t a[4];
  ldsm_x4(a, arow + k * 16);
  if constexpr (NT == 2) {
    uint32_t b[4];
    ldsm_x4(b, B + ((lane >> 4) * 8 + (lane & 7)) * ldb + k * 16 + ((lane >> 3) & 1) * 8);
    mma_bf16(c[0], a, b[0], b[1]);
    mma_bf16(c[1], a, b[2], b[3]);
  } else {
    uint32_t b0, b1;
    ldsm_x2(b0, b1, B + (lane & 7) * ldb + k * 16 + ((lane >> 3) & 1) * 8);
    mma_bf16(c[0], a, b0, b1);
  }
}

// one layer's new units of a 16-row tile: acc = bias + A[16 x 16 nkt] B^T, B rows in shared memory (row-major
// [unit][k])
template <int NT>
__device__ __forceinline__ void stage(float (&acc)[NT][4], const __nv_bfloat16* A, int lda, const __nv_bfloat16* B,
                                      int ldb, const float* __restrict__ bias, int nbias, int u0, int nkt, int lane) {
  const int q = lane & 3;
  float acc2[NT][4], acc3[NT][4], acc4[NT][4];
#pragma unroll
  for (int t = 0; t < NT; ++t) {
    const int n = u0 + t * 8 + 2 * q;   // columns past the layer (last tiles of small U) are computed and dropped
    const float b0 = n < nbias ? bias[n] : 0.f, b1 = n + 1 < nbias ? bias[n + 1] : 0.f;
    acc[t][0] = acc[t][2] = b0;
    acc[t][1] = acc[t][3] = b1;
#pragma unroll
    for (int e = 0; e < 4; ++e) acc2[t][e] = acc3[t][e] = acc4[t][e] = 0.f;
  }
  const __nv_bfloat16* arow = A + ((lane & 7) + ((lane >> 3) & 1) * 8) * lda + (lane >> 4) * 8;
  // k-tiles kt = 0, 1, 2, 3 (mod 4) accumulate in four independent chains: a quarter of the MMA dependency depth
  for (int kt = 0; kt < nkt; kt += 4) {
    stage_tile<NT>(acc, arow, B, ldb, kt, lane);
    if (kt + 1 < nkt) stage_tile<NT>(acc2, arow, B, ldb, kt + 1, lane);
    if (kt + 2 < nkt) stage_tile<NT>(acc3, arow, B, ldb, kt + 2, lane);
    if (kt + 3 < nkt) stage_tile<NT>(acc4, arow, B, ldb, kt + 3, lane);
  }
#pragma unroll
  for (int t = 0; t < NT; ++t)
#pragma unroll
    for (int e = 0; e < 4; ++e) acc[t][e] = (acc[t][e] + acc2[t][e]) + (acc3[t][e] + acc4[t][e]);
}

__device__ __forceinline__ int wrap_block(int v, int L) { return v < 0 ? v + L : (v >= L ? v - L : v); }

template <int G>
__global__ void __launch_bounds__(step_threads<G>()) step_kernel(StepParams p) {
  using SL = Slice<G>;
  constexpr int U = SL::U, S = SL::S, TW = tile_warps<G>(), NT = SL::NT / TW;
  extern __shared__ __align__(16) unsigned char smem[];
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31, gr = lane >> 2, q = lane & 3;
  const int warp = wid / TW, sub = wid - warp * TW;   // the tile, and this warp's n8 tile within a layer step
  __nv_bfloat16* X = (__nv_bfloat16*)(smem + warp * WARP_SMEM);
  __nv_bfloat16* const H0 = X + 16 * XS;       // layer l's activations at H0 + l * 16 * HS
  __nv_bfloat16* const slices = (__nv_bfloat16*)(smem + STEP_WARPS * WARP_SMEM);   // two buffers of ELEMS
  for (int i = lane + 32 * sub; i < WARP_SMEM / 16; i += 32 * TW) ((uint4*)X)[i] = make_uint4(0, 0, 0, 0);
  tile_sync(warp, TW);

  const long long tasks = (long long)p.R * p.nc;
  const long long ctasks = (tasks + 8 * STEP_WARPS - 1) / (8 * STEP_WARPS);   // 8 blocks per warp
  const int half = p.nb >> 1, L = p.L;
  if ((long long)blockIdx.x < ctasks) load_slice<G>(slices, p, 0);
  for (long long ct = blockIdx.x; ct < ctasks; ct += gridDim.x) {
    tile_sync(warp, TW);   // the tile's first warp is done with the previous blocks' rows
    // ---- block r = gr of this warp (lanes 4r..4r+3): rows r (proposal) and r + 8 (current spins)
    const long long task = (ct * STEP_WARPS + warp) * 8 + gr;
    const bool valid = task < tasks;
    const int rep = valid ? (int)(task / p.nc) : 0;
    const int k = valid ? (int)(task % p.nc) : 0;
    const int bx = 2 * (k % half) + (p.colour & 1), by = 2 * (k / half % half) + ((p.colour >> 1) & 1),
              bz = 2 * (k / (half * half)) + (p.colour >> 2);
    const int x0 = 4 * bx, y0 = 4 * by, z0 = 4 * bz;
    const long long uid = (long long)rep * p.nb * p.nb * p.nb + (bx + p.nb * (by + p.nb * bz));
    const int8_t* base = p.spins + (long long)rep * L * L * L;
    for (int col = q + 4 * sub; col < IN; col += 4 * TW) {
      float s = 0.f;
      if (valid) {
        const int x = wrap_block(x0 + c_tab.in_off[col][0], L), y = wrap_block(y0 + c_tab.in_off[col][1], L),
                  z = wrap_block(z0 + c_tab.in_off[col][2], L);
        s = (float)base[((long long)z * L + y) * L + x];
      }
      const __nv_bfloat16 v = __float2bfloat16_rn(s);
      X[(gr + 8) * XS + col] = v;
      X[gr * XS + col] = col < NBD ? v : __float2bfloat16_rn(0.f);
    }
    __syncwarp();
    tile_sync(warp, TW);

    float lq_new = 0.f, lq_old = 0.f;
    Philox4 rnd{0, 0, 0, 0};
    int rnd_w = -1;
    for (int g = 0; g < G; ++g) {
      cp_async_wait<0>();
      __syncthreads();   // slice g has landed; every warp is done with the other buffer
      const bool more = ct + gridDim.x < ctasks;
      __nv_bfloat16* const next = slices + ((g + 1) & 1) * SL::ELEMS;
      if (g + 1 < G) load_slice<G>(next, p, g + 1);
      else if (more) load_slice<G>(next, p, 0);
      const __nv_bfloat16* sl = slices + (g & 1) * SL::ELEMS;
      const int nkt = (U * (g + 1) + 15) / 16;    // hidden units of degree <= g
      // layer 1: inputs of degree <= g are the boundary and the spins of groups < g
      {
        float acc[NT][4];
        stage<NT>(acc, X, XS, sl + SL::W1 + sub * 8 * XS, XS, p.bias[0], H, g * U + sub * 8,
                  (NBD + S * g + 15) / 16, lane);
#pragma unroll
        for (int t = 0; t < NT; ++t) {
          const int c = g * U + sub * 8 + t * 8 + 2 * q;
          if (2 * q < U) {
            *(uint32_t*)(H0 + gr * HS + c) = pack_bf16(fmaxf(acc[t][0], 0.f), fmaxf(acc[t][1], 0.f));
            *(uint32_t*)(H0 + (gr + 8) * HS + c) = pack_bf16(fmaxf(acc[t][2], 0.f), fmaxf(acc[t][3], 0.f));
          }
        }
      }
      __syncwarp();
      tile_sync(warp, TW);
#pragma unroll
      for (int l = 1; l < 3; ++l) {
        float acc[NT][4];
        stage<NT>(acc, H0 + (l - 1) * 16 * HS, HS, sl + (l == 1 ? SL::W2 : SL::W3) + sub * 8 * HS, HS, p.bias[l], H,
                  g * U + sub * 8, nkt, lane);
#pragma unroll
        for (int t = 0; t < NT; ++t) {
          const int c = g * U + sub * 8 + t * 8 + 2 * q;
          if (2 * q < U) {
            *(uint32_t*)(H0 + l * 16 * HS + gr * HS + c) = pack_bf16(fmaxf(acc[t][0], 0.f), fmaxf(acc[t][1], 0.f));
            *(uint32_t*)(H0 + l * 16 * HS + (gr + 8) * HS + c) =
                pack_bf16(fmaxf(acc[t][2], 0.f), fmaxf(acc[t][3], 0.f));
          }
        }
        __syncwarp();
        tile_sync(warp, TW);
      }
      if (sub != 0) continue;   // the logits and draws of the tile: its first warp
      // logits of group g (positions S g .. S g + S - 1 in the first columns of one n8 tile)
      float lo[1][4];
      stage<1>(lo, H0 + 2 * 16 * HS, HS, sl + SL::W4, HS, p.bias[3], NSP, g * S, nkt, lane);
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int j = 2 * q + e;
        if (j < S) {
          const int pos = g * S + j;
          const int w = pos >> 2;
          if (w != rnd_w) {
            rnd = philox4x32_10((uint32_t)(int32_t)(17 * uid + w), 0u, p.k0, p.k1);
            rnd_w = w;
          }
          const int o = pos & 3;
          const uint32_t bits = o == 0 ? rnd.x0 : (o == 1 ? rnd.x1 : (o == 2 ? rnd.x2 : rnd.x3));
          const float u = to_uniform(bits);
          const float ln = lo[0][e], lc = lo[0][2 + e];
          const float xn = u < 1.f / (1.f + __expf(-ln)) ? 1.f : -1.f;
          const float xc = __bfloat162float(X[(gr + 8) * XS + NBD + pos]);
          lq_new += log_sigmoid(xn * ln);
          lq_old += log_sigmoid(xc * lc);
          X[gr * XS + NBD + pos] = __float2bfloat16_rn(xn);
        }
      }
      __syncwarp();
    }
    if (sub != 0) continue;   // energy change, acceptance and write-back: the tile's first warp
    lq_new += __shfl_xor_sync(0xffffffffu, lq_new, 1);
    lq_new += __shfl_xor_sync(0xffffffffu, lq_new, 2);
    lq_old += __shfl_xor_sync(0xffffffffu, lq_old, 1);
    lq_old += __shfl_xor_sync(0xffffffffu, lq_old, 2);

    // ---- energy change, integer: -(sum_internal (x'x' - xx) + sum_face (x' - x) b)
    const __nv_bfloat16* xn_row = X + gr * XS + NBD;
    const __nv_bfloat16* xc_row = X + (gr + 8) * XS + NBD;
    int de = 0;
    for (int i = q; i < 144; i += 4) {
      const int a = c_tab.internal[i][0], b = c_tab.internal[i][1];
      const int sn = (int)__bfloat162float(xn_row[a]) * (int)__bfloat162float(xn_row[b]);
      const int sc = (int)__bfloat162float(xc_row[a]) * (int)__bfloat162float(xc_row[b]);
      de -= sn - sc;
    }
    for (int i = q; i < NBD; i += 4) {
      const int a = c_tab.face[i];
      const int bd = (int)__bfloat162float(X[gr * XS + i]);
      de -= ((int)__bfloat162float(xn_row[a]) - (int)__bfloat162float(xc_row[a])) * bd;
    }
    de += __shfl_xor_sync(0xffffffffu, de, 1);
    de += __shfl_xor_sync(0xffffffffu, de, 2);

    int acc_flag = 0;
    if (q == 0 && valid) {
      const Philox4 ra = philox4x32_10((uint32_t)(int32_t)(17 * uid + 16), 0u, p.k0, p.k1);
      const float ua = to_uniform(ra.x0);
      const float logr = -p.beta[rep] * (float)de + lq_old - lq_new;
      acc_flag = ua < __expf(fminf(logr, 0.f)) ? 1 : 0;
      if (acc_flag && p.accepted) atomicAdd(p.accepted + rep, 1);
    }
    acc_flag = __shfl_sync(0xffffffffu, acc_flag, lane & ~3);
    if (valid && acc_flag) {
      // lane q writes the four x-rows of layer lz = q
      int8_t* dst = p.spins + (long long)rep * L * L * L;
      for (int ly = 0; ly < 4; ++ly) {
        uint32_t word = 0;
#pragma unroll
        for (int lx = 0; lx < 4; ++lx) {
          const int pos = c_tab.pos_of_raster[lx + 4 * ly + 16 * q];
          const int8_t s = (int8_t)(int)__bfloat162float(xn_row[pos]);
          word |= (uint32_t)(uint8_t)s << (8 * lx);
        }
        *(uint32_t*)(dst + ((long long)(z0 + q) * L + (y0 + ly)) * L + x0) = word;
      }
    }
    if (valid && p.record) {
      unsigned char* rec = p.record + 80 * task;
      for (int pos = q; pos < NSP; pos += 4) rec[pos] = (unsigned char)(int8_t)(int)__bfloat162float(xn_row[pos]);
      if (q == 0) {
        float* f = (float*)(rec + NSP);
        f[0] = lq_new;
        f[1] = lq_old;
        f[2] = (float)de;
        f[3] = (float)acc_flag;
      }
    }
    __syncwarp();
  }
  cp_async_wait<0>();
}

// ================================================================= the colour step, 16 proposals per tile (G = 16)
// The kernel above carries the current spins of a tile's 8 blocks through the autoregressive chain in rows
// 8..15 of its MMA tiles. This one fills all 16 rows with proposals (16 blocks per tile, two blocks per lane
// group) and evaluates the current spins' density afterwards in one dense pass: the network's masks make every
// logit of x a function of x alone, so the 16 x 4 layer steps need no chaining there — layer by layer, 32 units at
// a time, the weights streamed through the same double buffer. Every unit is computed with the same k-tiles and
// summation order as in the chain (the extra k-tiles of a chunk meet masked zero weights and add exact zeros), and
// log q(x) sums its 64 terms in the chain's order, so that the density of a configuration is the same number
// whether it is drawn or current: the Metropolis-Hastings ratio stays exact to the last bit.
constexpr int PAIR_TILE_SMEM = WARP_SMEM + 2 * 16 * NSP + 16 * 4;   // + current and proposed spins, log q(x')
constexpr int DENSE_CHUNKS = 26;      // 8 per hidden layer (32 units each), 2 for the output layer
// the dense pass splits the two slice buffers into three chunk buffers, so that two chunks load while one is used
constexpr int DENSE_BUF_ELEMS = 2 * 13248 / 3;
static_assert(3 * DENSE_BUF_ELEMS == 2 * Slice<16>::ELEMS, "three chunk buffers fill the two slice buffers");
static_assert(32 * HS <= DENSE_BUF_ELEMS && 32 * XS <= DENSE_BUF_ELEMS, "a chunk fits its buffer");

constexpr int pair_smem() { return STEP_WARPS * PAIR_TILE_SMEM + 2 * Slice<16>::BYTES; }

struct DenseChunk {
  int layer, u0, nkt, ld;
};

// chunk i: rows [u0, u0 + 32) of W_{layer + 1} with the k-tiles of degree <= the chunk's highest unit degree
__device__ __forceinline__ DenseChunk dense_chunk(int i) {
  DenseChunk d;
  if (i < 24) {
    const int c = i & 7;
    d.layer = i >> 3;
    d.u0 = 32 * c;
    d.nkt = d.layer == 0 ? (NBD + 4 * (2 * c + 1) + 15) / 16 : 2 * c + 2;
    d.ld = d.layer == 0 ? XS : HS;
  } else {
    const int c = i - 24;
    d.layer = 3;
    d.u0 = 32 * c;
    d.nkt = 8 * c + 8;
    d.ld = HS;
  }
  return d;
}

// all threads of the block: copy dense chunk i into `dst` (cp.async, one commit group)
__device__ __forceinline__ void load_dense_chunk(__nv_bfloat16* dst, const StepParams& p, int i) {
  const DenseChunk d = dense_chunk(i);
  const int K = d.layer == 0 ? IN : H;
  const int ch = 2 * d.nkt;                       // 16-byte pieces per row
  const __nv_bfloat16* W = p.W[d.layer];
  for (int j = threadIdx.x; j < 32 * ch; j += blockDim.x) {
    const int r = j / ch, c = j - r * ch;
    cp_async16(dst + r * d.ld + c * 8, W + (long long)(d.u0 + r) * K + c * 8, 16);
  }
  cp_async_commit();
}

// Grid of persistent blocks of 5 tiles x 2 warps; tile rows r = 0..15 are the proposals of blocks 16 t + r, lanes
// (gr, q) of the tile's first warp own blocks gr and gr + 8 for the draws, densities, energy and write-back.
__global__ void __launch_bounds__(32 * STEP_WARPS * 2) step_pair_kernel(StepParams p) {
  using SL = Slice<16>;
  constexpr int U = SL::U, S = SL::S;
  extern __shared__ __align__(16) unsigned char smem[];
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31, gr = lane >> 2, q = lane & 3;
  const int warp = wid >> 1, sub = wid & 1;
  unsigned char* tbase = smem + warp * PAIR_TILE_SMEM;
  __nv_bfloat16* X = (__nv_bfloat16*)tbase;
  __nv_bfloat16* const H0 = X + 16 * XS;
  int8_t* const CUR = (int8_t*)(tbase + WARP_SMEM);           // [16][64] current spins of the tile's blocks
  int8_t* const PROP = CUR + 16 * NSP;                        // [16][64] proposed spins
  float* const LS = (float*)H0;   // [16][64] log-sigmoid terms of x, over layer 1's activations once they are spent
  float* const LQN = (float*)(PROP + 16 * NSP);               // [16] log q(x') of the rows the second warp drew
  __nv_bfloat16* const slices = (__nv_bfloat16*)(smem + STEP_WARPS * PAIR_TILE_SMEM);
  for (int i = lane + 32 * sub; i < WARP_SMEM / 16; i += 64) ((uint4*)X)[i] = make_uint4(0, 0, 0, 0);
  tile_sync(warp, 2);

  const long long tasks = (long long)p.R * p.nc;
  const long long ctasks = (tasks + 16 * STEP_WARPS - 1) / (16 * STEP_WARPS);   // 16 blocks per tile
  const int half = p.nb >> 1, L = p.L;
  if ((long long)blockIdx.x < ctasks) load_slice<16>(slices, p, 0);
  for (long long ct = blockIdx.x; ct < ctasks; ct += gridDim.x) {
    tile_sync(warp, 2);   // the first warp is done with the previous blocks' rows
    const bool more = ct + gridDim.x < ctasks;
    // ---- gather: row r = block 16 (ct * tiles + tile) + r; both warps, rows split by lane group and warp
    for (int rr = 0; rr < 2; ++rr) {
      const int r = gr + 8 * rr;
      const long long task = (ct * STEP_WARPS + warp) * 16 + r;
      const bool valid = task < tasks;
      const int rep = valid ? (int)(task / p.nc) : 0;
      const int k = valid ? (int)(task % p.nc) : 0;
      const int bx = 2 * (k % half) + (p.colour & 1), by = 2 * (k / half % half) + ((p.colour >> 1) & 1),
                bz = 2 * (k / (half * half)) + (p.colour >> 2);
      const int8_t* base = p.spins + (long long)rep * L * L * L;
      for (int col = q + 4 * sub; col < IN; col += 8) {
        float s = 0.f;
        if (valid) {
          const int x = wrap_block(4 * bx + c_tab.in_off[col][0], L), y = wrap_block(4 * by + c_tab.in_off[col][1], L),
                    z = wrap_block(4 * bz + c_tab.in_off[col][2], L);
          s = (float)base[((long long)z * L + y) * L + x];
        }
        X[r * XS + col] = col < NBD ? __float2bfloat16_rn(s) : __float2bfloat16_rn(0.f);
        if (col >= NBD) CUR[r * NSP + col - NBD] = (int8_t)(int)s;
      }
    }
    __syncwarp();
    tile_sync(warp, 2);

    // ---- the first warp's two blocks
    long long task2[2];
    bool valid2[2];
    int rep2[2], b3[2][3];
    long long uid2[2];
#pragma unroll
    for (int rr = 0; rr < 2; ++rr) {
      task2[rr] = (ct * STEP_WARPS + warp) * 16 + gr + 8 * rr;
      valid2[rr] = task2[rr] < tasks;
      rep2[rr] = valid2[rr] ? (int)(task2[rr] / p.nc) : 0;
      const int k = valid2[rr] ? (int)(task2[rr] % p.nc) : 0;
      b3[rr][0] = 2 * (k % half) + (p.colour & 1);
      b3[rr][1] = 2 * (k / half % half) + ((p.colour >> 1) & 1);
      b3[rr][2] = 2 * (k / (half * half)) + (p.colour >> 2);
      uid2[rr] = (long long)rep2[rr] * p.nb * p.nb * p.nb + (b3[rr][0] + p.nb * (b3[rr][1] + p.nb * b3[rr][2]));
    }
    // warp `sub` draws the spins of rows gr + 8 sub (block uid_mine)
    const long long uid_mine = sub ? uid2[1] : uid2[0];
    float lq_mine = 0.f;
    // ---- the autoregressive chain: 16 steps of 4 spins
    for (int g = 0; g < 16; ++g) {
      // this step's uniforms first: their Philox rounds overlap the layers' MMA chains
      const Philox4 rnd = philox4x32_10((uint32_t)(int32_t)(17 * uid_mine + g), 0u, p.k0, p.k1);
      cp_async_wait<0>();
      __syncthreads();   // slice g has landed; every warp is done with the other buffer
      __nv_bfloat16* const next = slices + ((g + 1) & 1) * SL::ELEMS;
      if (g + 1 < 16) load_slice<16>(next, p, g + 1);
      else load_dense_chunk(slices, p, 0);   // chunk buffer 0 lies in slice buffer 0, unused by step 15
      const __nv_bfloat16* sl = slices + (g & 1) * SL::ELEMS;
      const int nkt = (U * (g + 1) + 15) / 16;
      {
        float acc[1][4];
        stage<1>(acc, X, XS, sl + SL::W1 + sub * 8 * XS, XS, p.bias[0], H, g * U + sub * 8, (NBD + S * g + 15) / 16,
                 lane);
        const int c = g * U + sub * 8 + 2 * q;
        *(uint32_t*)(H0 + gr * HS + c) = pack_bf16(fmaxf(acc[0][0], 0.f), fmaxf(acc[0][1], 0.f));
        *(uint32_t*)(H0 + (gr + 8) * HS + c) = pack_bf16(fmaxf(acc[0][2], 0.f), fmaxf(acc[0][3], 0.f));
      }
      __syncwarp();
      tile_sync(warp, 2);
#pragma unroll
      for (int l = 1; l < 3; ++l) {
        float acc[1][4];
        stage<1>(acc, H0 + (l - 1) * 16 * HS, HS, sl + (l == 1 ? SL::W2 : SL::W3) + sub * 8 * HS, HS, p.bias[l], H,
                 g * U + sub * 8, nkt, lane);
        const int c = g * U + sub * 8 + 2 * q;
        *(uint32_t*)(H0 + l * 16 * HS + gr * HS + c) = pack_bf16(fmaxf(acc[0][0], 0.f), fmaxf(acc[0][1], 0.f));
        *(uint32_t*)(H0 + l * 16 * HS + (gr + 8) * HS + c) = pack_bf16(fmaxf(acc[0][2], 0.f), fmaxf(acc[0][3], 0.f));
        __syncwarp();
        tile_sync(warp, 2);
      }
      {
        // logits of group g in both warps (the same MMAs), each warp drawing the spins of its own rows
        float lo[1][4];
        stage<1>(lo, H0 + 2 * 16 * HS, HS, sl + SL::W4, HS, p.bias[3], NSP, g * S, nkt, lane);
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int j = 2 * q + e;
          if (j < S) {
            const int pos = g * S + j;
            const int o = pos & 3;
            const uint32_t bits = o == 0 ? rnd.x0 : (o == 1 ? rnd.x1 : (o == 2 ? rnd.x2 : rnd.x3));
            const float u = to_uniform(bits);
            const float ln = sub ? lo[0][2 + e] : lo[0][e];
            const float xn = u < 1.f / (1.f + __expf(-ln)) ? 1.f : -1.f;
            lq_mine += log_sigmoid(xn * ln);
            X[(gr + 8 * sub) * XS + NBD + pos] = __float2bfloat16_rn(xn);
          }
        }
      }
      __syncwarp();
    }
    lq_mine += __shfl_xor_sync(0xffffffffu, lq_mine, 1);
    lq_mine += __shfl_xor_sync(0xffffffffu, lq_mine, 2);
    if (sub == 1 && q == 0) LQN[gr + 8] = lq_mine;
    tile_sync(warp, 2);   // the last draws are in X, the second warp's densities in LQN
    // ---- keep the proposals, put the current spins in their place
    for (int i = lane + 32 * sub; i < 16 * NSP; i += 64) {
      const int r = i / NSP, j = i - r * NSP;
      PROP[i] = (int8_t)(int)__bfloat162float(X[r * XS + NBD + j]);
      X[r * XS + NBD + j] = __float2bfloat16_rn((float)CUR[i]);
    }
    // ---- the dense pass over the current spins: the terms of log q(x) of the 16 blocks
    for (int i = 0; i < DENSE_CHUNKS; ++i) {
      // chunk i has landed (chunk i + 1, issued a step earlier, may still be in flight); after the barrier every
      // warp is done with chunk i - 1, whose buffer takes chunk i + 2, and with the previous layer's activations
      if (i == 0 || i + 1 == DENSE_CHUNKS) cp_async_wait<0>();
      else cp_async_wait<1>();
      __syncthreads();
      if (i == 0) load_dense_chunk(slices + DENSE_BUF_ELEMS, p, 1);
      if (i + 2 < DENSE_CHUNKS) load_dense_chunk(slices + ((i + 2) % 3) * DENSE_BUF_ELEMS, p, i + 2);
      const __nv_bfloat16* wc = slices + (i % 3) * DENSE_BUF_ELEMS;
      const DenseChunk d = dense_chunk(i);
      float acc[2][4];
      const int u0 = d.u0 + 16 * sub;
      if (d.layer == 0) {
        stage<2>(acc, X, XS, wc + 16 * sub * XS, XS, p.bias[0], H, u0, d.nkt, lane);
      } else {
        stage<2>(acc, H0 + (d.layer - 1) * 16 * HS, HS, wc + 16 * sub * HS, HS, p.bias[d.layer],
                 d.layer == 3 ? NSP : H, u0, d.nkt, lane);
      }
#pragma unroll
      for (int tt = 0; tt < 2; ++tt) {
        const int c = u0 + tt * 8 + 2 * q;
        if (d.layer < 3) {
          *(uint32_t*)(H0 + d.layer * 16 * HS + gr * HS + c) =
              pack_bf16(fmaxf(acc[tt][0], 0.f), fmaxf(acc[tt][1], 0.f));
          *(uint32_t*)(H0 + d.layer * 16 * HS + (gr + 8) * HS + c) =
              pack_bf16(fmaxf(acc[tt][2], 0.f), fmaxf(acc[tt][3], 0.f));
        } else {
#pragma unroll
          for (int rr = 0; rr < 2; ++rr)
#pragma unroll
            for (int e = 0; e < 2; ++e) {
              const int o = (gr + 8 * rr) * NSP + c + e;
              LS[o] = log_sigmoid((float)CUR[o] * acc[tt][2 * rr + e]);
            }
        }
      }
    }
    __syncthreads();   // every warp is done with the chunk buffers and the terms of log q(x) are in place
    if (more) load_slice<16>(slices, p, 0);
    if (sub != 0) continue;   // densities, energy change, acceptance and write-back: the tile's first warp
    // log q(x) in the chain's order: lane q < 2 adds positions 4 g + 2 q, 4 g + 2 q + 1 for g = 0 .. 15
    float lq_old[2] = {0.f, 0.f};
#pragma unroll
    for (int rr = 0; rr < 2; ++rr) {
      if (q < 2)
        for (int g = 0; g < 16; ++g) {
          lq_old[rr] += LS[(gr + 8 * rr) * NSP + 4 * g + 2 * q];
          lq_old[rr] += LS[(gr + 8 * rr) * NSP + 4 * g + 2 * q + 1];
        }
      lq_old[rr] += __shfl_xor_sync(0xffffffffu, lq_old[rr], 1);
      lq_old[rr] += __shfl_xor_sync(0xffffffffu, lq_old[rr], 2);
    }
#pragma unroll
    for (int rr = 0; rr < 2; ++rr) {
      const int r = gr + 8 * rr;
      const float lqn = rr ? LQN[r] : lq_mine;
      const float lqo = lq_old[rr];
      // energy change, integer: -(sum_internal (x'x' - xx) + sum_face (x' - x) b)
      const int8_t* xn_row = PROP + r * NSP;
      const int8_t* xc_row = CUR + r * NSP;
      int de = 0;
      for (int i = q; i < 144; i += 4) {
        const int a = c_tab.internal[i][0], b = c_tab.internal[i][1];
        de -= (int)xn_row[a] * (int)xn_row[b] - (int)xc_row[a] * (int)xc_row[b];
      }
      for (int i = q; i < NBD; i += 4) {
        const int a = c_tab.face[i];
        const int bd = (int)__bfloat162float(X[r * XS + i]);
        de -= ((int)xn_row[a] - (int)xc_row[a]) * bd;
      }
      de += __shfl_xor_sync(0xffffffffu, de, 1);
      de += __shfl_xor_sync(0xffffffffu, de, 2);
      const bool valid = valid2[rr];
      const int rep = rep2[rr];
      int acc_flag = 0;
      if (q == 0 && valid) {
        const Philox4 ra = philox4x32_10((uint32_t)(int32_t)(17 * uid2[rr] + 16), 0u, p.k0, p.k1);
        const float ua = to_uniform(ra.x0);
        const float logr = -p.beta[rep] * (float)de + lqo - lqn;
        acc_flag = ua < __expf(fminf(logr, 0.f)) ? 1 : 0;
        if (acc_flag && p.accepted) atomicAdd(p.accepted + rep, 1);
      }
      acc_flag = __shfl_sync(0xffffffffu, acc_flag, lane & ~3);
      if (valid && acc_flag) {
        // lane q writes the four x-rows of layer lz = q
        int8_t* dst = p.spins + (long long)rep * L * L * L;
        const int x0 = 4 * b3[rr][0], y0 = 4 * b3[rr][1], z0 = 4 * b3[rr][2];
        for (int ly = 0; ly < 4; ++ly) {
          uint32_t word = 0;
#pragma unroll
          for (int lx = 0; lx < 4; ++lx) {
            const int pos = c_tab.pos_of_raster[lx + 4 * ly + 16 * q];
            word |= (uint32_t)(uint8_t)xn_row[pos] << (8 * lx);
          }
          *(uint32_t*)(dst + ((long long)(z0 + q) * L + (y0 + ly)) * L + x0) = word;
        }
      }
      if (valid && p.record) {
        unsigned char* rec = p.record + 80 * task2[rr];
        for (int pos = q; pos < NSP; pos += 4) rec[pos] = (unsigned char)xn_row[pos];
        if (q == 0) {
          float* f = (float*)(rec + NSP);
          f[0] = lqn;
          f[1] = lqo;
          f[2] = (float)de;
          f[3] = (float)acc_flag;
        }
      }
    }
    __syncwarp();
  }
  cp_async_wait<0>();
}

// ======================================================================================= workspace layout
struct TrainLayout {
  long long h[3], logits, g4, gh[3], wpart[4], bpart[4], grads, total;
  int splits, chunk;   // the weight gradients reduce the batch in `splits` chunks of `chunk` rows (multiple of 64)
};

inline TrainLayout train_layout(int M) {
  TrainLayout t{};
  long long o = 0;
  auto take = [&](long long bytes) {
    const long long at = o;
    o = align256(o + bytes);
    return at;
  };
  int s = M / 1024;
  s = s < 1 ? 1 : (s > 16 ? 16 : s);
  t.chunk = ((M + s - 1) / s + 63) / 64 * 64;
  t.splits = (M + t.chunk - 1) / t.chunk;
  for (int l = 0; l < 3; ++l) t.h[l] = take((long long)M * H * 2);
  t.logits = take((long long)M * NSP * 4);
  t.g4 = take((long long)M * NSP * 2);
  for (int l = 0; l < 3; ++l) t.gh[l] = take((long long)M * H * 2);
  for (int l = 0; l < 4; ++l) t.wpart[l] = take((long long)t.splits * out_rows(l) * in_cols(l) * 4);
  for (int l = 0; l < 4; ++l) t.bpart[l] = take((long long)t.splits * out_rows(l) * 4);
  t.grads = take(NPARAM * 4);
  t.total = o;
  return t;
}

int forward_layers(const void* params, const __nv_bfloat16* x, int M, char* ws, const TrainLayout& t, cudaStream_t s) {
  const float* master = (const float*)params;
  const __nv_bfloat16* in = x;
  long long ld = IN;
  for (int l = 0; l < 4; ++l) {
    GemmArgs g{};
    g.A = in;
    g.lda = ld;
    g.B = bf_weights(params, l);
    g.ldb = in_cols(l);
    g.M = M;
    g.N = out_rows(l);
    g.K = in_cols(l);
    g.kchunk = in_cols(l);
    g.bias = master + off_b(l);
    int rc;
    // batches of whole 128-row tiles run on tcgen05; others on the mma.sync kernel
    const bool umma = M % UM == 0;
    if (l < 3) {
      g.C = ws + t.h[l];
      g.ldc = H;
      rc = umma ? umma_gemm<EPI_BIAS_RELU_BF16>(g, s) : gemm<true, true, EPI_BIAS_RELU_BF16>(g, 1, s);
      in = (const __nv_bfloat16*)(ws + t.h[l]);
      ld = H;
    } else {
      g.C = ws + t.logits;
      g.ldc = NSP;
      rc = umma ? umma_gemm<EPI_BIAS_F32>(g, s) : gemm<true, true, EPI_BIAS_F32>(g, 1, s);
    }
    if (rc) return rc;
  }
  return SCK_OK;
}

int backward(const void* params, const __nv_bfloat16* x, int M, char* ws, const TrainLayout& t, cudaStream_t s) {
  const int chunk = t.chunk;
  // gradients of the preactivations, top down: G4 (logits), G3, G2, G1
  const __nv_bfloat16* gcur = (const __nv_bfloat16*)(ws + t.g4);
  int gN = NSP;
  for (int l = 3; l >= 0; --l) {
    const __nv_bfloat16* act = l == 0 ? x : (const __nv_bfloat16*)(ws + t.h[l - 1]);
    const int K = in_cols(l);
    // dW_l[n][k] = sum_m G[m][n] act[m][k]
    GemmArgs g{};
    g.A = gcur;
    g.lda = gN;
    g.B = act;
    g.ldb = K;
    g.M = gN;
    g.N = K;
    g.K = M;
    g.kchunk = chunk;
    g.C = ws + t.wpart[l];
    g.ldc = K;
    g.split_stride = (long long)gN * K;
    int rc = gemm<false, false, EPI_F32>(g, t.splits, s);
    if (rc) return rc;
    dim3 cg((gN + 255) / 256, t.splits);
    colsum_kernel<<<cg, 256, 0, s>>>(gcur, M, gN, chunk, (float*)(ws + t.bpart[l]));
    rc = cuda_status(cudaGetLastError(), "made colsum");
    if (rc) return rc;
    if (l == 0) break;
    // G_{l-1} = (G_l W_l) where act > 0
    GemmArgs d{};
    d.A = gcur;
    d.lda = gN;
    d.B = bf_weights(params, l);
    d.ldb = K;
    d.M = M;
    d.N = K;
    d.K = gN;
    d.kchunk = gN;
    d.C = ws + t.gh[l - 1];
    d.ldc = K;
    d.gate = act;
    rc = gemm<true, false, EPI_GATE_BF16>(d, 1, s);
    if (rc) return rc;
    gcur = (const __nv_bfloat16*)(ws + t.gh[l - 1]);
    gN = K;
  }
  return SCK_OK;
}

}  // namespace made
}  // namespace sck

using namespace sck;
using namespace sck::made;

static int made_fail(int code, const char* msg) {
  set_error(msg);
  return code;
}

static bool groups_ok(int G) { return G == 16 || G == 64; }

extern "C" {

int sck_made_set_wait_limit(int64_t polls) {
  if (polls < 0) return made_fail(SCK_ERR_INVALID, "polls must not be negative");
  return made_set_wait_limit((long long)polls);
}

int sck_made_wait_status(void* stream) {
  // give-ups counted on the current device since its last status read
  static unsigned long long seen[64];
  int dev = 0;
  int rc = cuda_status(cudaGetDevice(&dev), "learned wait status");
  if (rc != SCK_OK) return rc;
  rc = cuda_status(cudaStreamSynchronize((cudaStream_t)stream), "learned wait status");
  if (rc != SCK_OK) return rc;
  unsigned long long now = 0;
  rc = made_wait_timeouts(&now);
  if (rc != SCK_OK) return rc;
  if (dev < 0 || dev >= 64) return SCK_OK;
  if (now != seen[dev]) {
    seen[dev] = now;
    return made_fail(SCK_ERR_TIMEOUT, "a bounded wait of the learned proposal's tensor-core GEMM gave up: its "
                                      "output rows were left unwritten");
  }
  return SCK_OK;
}

int sck_made_sizes(int32_t groups, int32_t batch, int64_t* param_bytes, int64_t* adam_bytes, int64_t* train_bytes) {
  if (!groups_ok(groups)) return made_fail(SCK_ERR_INVALID, "groups must be 16 or 64");
  if (train_bytes && (batch <= 0 || batch % 64 != 0))
    return made_fail(SCK_ERR_INVALID, "batch must be a positive multiple of 64");
  if (param_bytes) *param_bytes = align256(BF_BASE_BYTES + NBF * 2);
  if (adam_bytes) *adam_bytes = 2 * NPARAM * 4;
  if (train_bytes) *train_bytes = train_layout(batch).total;
  return SCK_OK;
}

int sck_made_prepare(void* params, int32_t groups, void* stream) {
  if (params == nullptr) return made_fail(SCK_ERR_INVALID, "null parameters");
  if (!groups_ok(groups)) return made_fail(SCK_ERR_INVALID, "groups must be 16 or 64");
  cudaStream_t s = (cudaStream_t)stream;
  __nv_bfloat16* bf = (__nv_bfloat16*)((char*)params + BF_BASE_BYTES);
  prepare_kernel<<<(unsigned)((NBF + 255) / 256), 256, 0, s>>>((const float*)params, bf, groups);
  return cuda_status(cudaGetLastError(), "made prepare");
}

int sck_made_gather(const int8_t* spins, int32_t R, int32_t L, uint16_t* out, void* stream) {
  if (spins == nullptr || out == nullptr) return made_fail(SCK_ERR_INVALID, "null spins or output");
  if (R < 1 || L < 8 || L % 8 != 0) return made_fail(SCK_ERR_INVALID, "need R >= 1 and L a multiple of 8");
  int rc = ensure_tables();
  if (rc) return rc;
  const long long n = (long long)R * (L / 4) * (L / 4) * (L / 4) * IN;
  gather_kernel<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(spins, R, L, (__nv_bfloat16*)out);
  return cuda_status(cudaGetLastError(), "made gather");
}

int sck_made_forward(const void* params, int32_t groups, const uint16_t* x, int32_t batch, float* logits, float* logq,
                     void* workspace, void* stream) {
  if (params == nullptr || x == nullptr || workspace == nullptr || logits == nullptr)
    return made_fail(SCK_ERR_INVALID, "null parameters, inputs, logits or workspace");
  if (!groups_ok(groups)) return made_fail(SCK_ERR_INVALID, "groups must be 16 or 64");
  if (batch <= 0 || batch % 64 != 0) return made_fail(SCK_ERR_INVALID, "batch must be a positive multiple of 64");
  cudaStream_t s = (cudaStream_t)stream;
  const TrainLayout t = train_layout(batch);
  char* ws = (char*)workspace;
  int rc = forward_layers(params, (const __nv_bfloat16*)x, batch, ws, t, s);
  if (rc) return rc;
  rc = cuda_status(cudaMemcpyAsync(logits, ws + t.logits, (size_t)batch * NSP * 4, cudaMemcpyDeviceToDevice, s),
                   "made logits");
  if (rc) return rc;
  if (logq) {
    loss_kernel<<<(batch + 3) / 4, 256, 0, s>>>(logits, (const __nv_bfloat16*)x, batch, nullptr, logq, nullptr);
    rc = cuda_status(cudaGetLastError(), "made density");
  }
  return rc;
}

static int grads_common(const void* params, int groups, const uint16_t* x, int batch, float* loss, char* ws,
                        const TrainLayout& t, cudaStream_t s) {
  int rc = forward_layers(params, (const __nv_bfloat16*)x, batch, ws, t, s);
  if (rc) return rc;
  if (loss) {
    rc = cuda_status(cudaMemsetAsync(loss, 0, 4, s), "made loss");
    if (rc) return rc;
  }
  loss_kernel<<<(batch + 3) / 4, 256, 0, s>>>((const float*)(ws + t.logits), (const __nv_bfloat16*)x, batch,
                                               (__nv_bfloat16*)(ws + t.g4), nullptr, loss);
  rc = cuda_status(cudaGetLastError(), "made loss");
  if (rc) return rc;
  return backward(params, (const __nv_bfloat16*)x, batch, ws, t, s);
}

static FinishArgs finish_args(char* ws, const TrainLayout& t, int groups) {
  FinishArgs a{};
  for (int l = 0; l < 4; ++l) {
    a.wpart[l] = (const float*)(ws + t.wpart[l]);
    a.bpart[l] = (const float*)(ws + t.bpart[l]);
  }
  a.splits = t.splits;
  a.G = groups;
  return a;
}

int sck_made_grads(const void* params, int32_t groups, const uint16_t* x, int32_t batch, float* grads, float* loss,
                   void* workspace, void* stream) {
  if (params == nullptr || x == nullptr || workspace == nullptr || grads == nullptr)
    return made_fail(SCK_ERR_INVALID, "null parameters, inputs, gradients or workspace");
  if (!groups_ok(groups)) return made_fail(SCK_ERR_INVALID, "groups must be 16 or 64");
  if (batch <= 0 || batch % 64 != 0) return made_fail(SCK_ERR_INVALID, "batch must be a positive multiple of 64");
  cudaStream_t s = (cudaStream_t)stream;
  const TrainLayout t = train_layout(batch);
  char* ws = (char*)workspace;
  int rc = grads_common(params, groups, x, batch, loss, ws, t, s);
  if (rc) return rc;
  FinishArgs a = finish_args(ws, t, groups);
  a.adam = 0;
  a.grads = grads;
  finish_kernel<<<(unsigned)((NPARAM + 255) / 256), 256, 0, s>>>(a);
  return cuda_status(cudaGetLastError(), "made gradients");
}

int sck_made_train_step(void* params, float* adam, int32_t groups, const uint16_t* x, int32_t batch, float lr,
                        float beta1, float beta2, float eps, int32_t t_step, float* loss, void* workspace,
                        void* stream) {
  if (params == nullptr || adam == nullptr || x == nullptr || workspace == nullptr)
    return made_fail(SCK_ERR_INVALID, "null parameters, moments, inputs or workspace");
  if (!groups_ok(groups)) return made_fail(SCK_ERR_INVALID, "groups must be 16 or 64");
  if (batch <= 0 || batch % 64 != 0) return made_fail(SCK_ERR_INVALID, "batch must be a positive multiple of 64");
  if (t_step < 1) return made_fail(SCK_ERR_INVALID, "Adam step t must be >= 1");
  cudaStream_t s = (cudaStream_t)stream;
  const TrainLayout t = train_layout(batch);
  char* ws = (char*)workspace;
  int rc = grads_common(params, groups, x, batch, loss, ws, t, s);
  if (rc) return rc;
  FinishArgs a = finish_args(ws, t, groups);
  a.adam = 1;
  a.master = (float*)params;
  a.m1 = adam;
  a.m2 = adam + NPARAM;
  a.bf = (__nv_bfloat16*)((char*)params + BF_BASE_BYTES);
  a.lr = lr;
  a.beta1 = beta1;
  a.beta2 = beta2;
  a.eps = eps;
  a.c1 = 1.f - powf(beta1, (float)t_step);
  a.c2 = 1.f - powf(beta2, (float)t_step);
  finish_kernel<<<(unsigned)((NPARAM + 255) / 256), 256, 0, s>>>(a);
  return cuda_status(cudaGetLastError(), "made Adam");
}

int sck_made_colour_step(const void* params, int32_t groups, int8_t* spins, int32_t R, int32_t L, const float* beta,
                         int32_t colour, int64_t seed, int32_t round, int32_t* accepted, void* record, void* stream) {
  if (params == nullptr || spins == nullptr || beta == nullptr)
    return made_fail(SCK_ERR_INVALID, "null parameters, spins or beta");
  if (!groups_ok(groups)) return made_fail(SCK_ERR_INVALID, "groups must be 16 or 64");
  if (R < 1 || L < 8 || L % 8 != 0) return made_fail(SCK_ERR_INVALID, "need R >= 1 and L a multiple of 8");
  if (colour < 0 || colour > 7) return made_fail(SCK_ERR_INVALID, "colour must be 0..7");
  const long long nb = L / 4;
  if ((long long)R * nb * nb * nb * 17 + 17 > 2147483647ll)
    return made_fail(SCK_ERR_COUNTER, "17 x replicas x blocks exceeds the int32 Philox counter");
  int rc = ensure_tables();
  if (rc) return rc;
  StepParams p{};
  for (int l = 0; l < 4; ++l) {
    p.W[l] = bf_weights(params, l);
    p.bias[l] = (const float*)params + off_b(l);
  }
  p.spins = spins;
  p.beta = beta;
  p.R = R;
  p.L = L;
  p.nb = (int)nb;
  p.nc = (int)(nb * nb * nb / 8);
  p.colour = colour;
  const long long v = seed * 1000003ll + (8ll * round + colour) * 7919ll + 24680ll;
  const int32_t key = (int32_t)(v % 2147483629ll);
  p.k0 = (uint32_t)key;
  p.k1 = key < 0 ? 0xFFFFFFFFu : 0u;
  p.accepted = accepted;
  p.record = (unsigned char*)record;
  cudaStream_t s = (cudaStream_t)stream;
  const long long ctasks = ((long long)R * p.nc + 8 * STEP_WARPS - 1) / (8 * STEP_WARPS);
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const long long grid = ctasks < sms ? ctasks : sms;
  if (groups == 16) {
    // 16 proposals per tile, the current spins' densities in a dense pass
    const long long ctasks2 = ((long long)R * p.nc + 16 * STEP_WARPS - 1) / (16 * STEP_WARPS);
    const long long grid2 = ctasks2 < sms ? ctasks2 : sms;
    rc = cuda_status(cudaFuncSetAttribute(step_pair_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, pair_smem()),
                     "made step smem");
    if (rc) return rc;
    step_pair_kernel<<<(unsigned)grid2, 32 * STEP_WARPS * 2, pair_smem(), s>>>(p);
  } else {
    rc = cuda_status(cudaFuncSetAttribute(step_kernel<64>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          step_smem<64>()), "made step smem");
    if (rc) return rc;
    step_kernel<64><<<(unsigned)grid, step_threads<64>(), step_smem<64>(), s>>>(p);
  }
  return cuda_status(cudaGetLastError(), "made colour step");
}

}  // extern "C"
