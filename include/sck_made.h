/* Learned block proposal for 3D Ising (simple cubic, periodic): C ABI of libsckb200.so.
 *
 * No counterpart in the reference, which has no learned part. A masked autoregressive MLP (MADE) proposes a joint
 * update of a 4x4x4 block of spins conditioned on its 96 boundary spins; the proposal's exact density enters a
 * Metropolis-Hastings ratio, so the Boltzmann distribution is kept. A colour step updates every block of one
 * parity class of the block coordinates (code px + 2 py + 4 pz) in every replica at once; the host orders these
 * classes by the block colouring it finds with the site colouring's search (8 colours: blocks touching at a
 * face, an edge or a corner differ).
 *
 * Conventions as in sck.h: caller-owned device buffers, every call asynchronous on the stream passed as void*,
 * no allocation and no synchronisation inside a call, 0 or a negative SCK_ERR_* status with sck_last_error().
 *
 * Spins: int8 +-1, [R, L, L, L] with x fastest (the int8 storage of sck.h for a one-site basis), L a multiple of 8.
 * Block inputs: bfloat16 +-1 rows of 160 = 96 boundary spins (faces -x, +x, -y, +y, -z, +z; 16 each, raster over
 * the two other local coordinates, lower axis fastest) then the 64 block spins in autoregressive order (the
 * block's even sites, then its odd sites, each parity sublattice (x%2, y%2, z%2) in raster order, sublattices in
 * the order 000, 110, 101, 011, 100, 010, 001, 111).
 * Network: 160 -> 256 -> 256 -> 256 -> 64 logits, ReLU; `groups` G = 16 or 64 autoregressive steps of 64 / G
 * spins; degrees boundary 0, position p: p / (64 / G) + 1, hidden unit k: k G / 256; masks as in MADE.
 * Parameters (one device buffer of sck_made_sizes' param_bytes, 256-byte aligned): FP32 masters
 * W1[256][160] b1[256] W2[256][256] b2[256] W3[256][256] b3[256] W4[64][256] b4[64] at the start (SCK_MADE_NPARAM
 * floats, in that order; the caller initialises them), then derived bfloat16 copies of the masked weights that
 * sck_made_prepare writes. */
#ifndef SCK_MADE_H
#define SCK_MADE_H

#include <stdint.h>

#include "sck.h"

#ifdef __cplusplus
extern "C" {
#endif

#define SCK_MADE_IN 160
#define SCK_MADE_HIDDEN 256
#define SCK_MADE_SPINS 64
#define SCK_MADE_BOUNDARY 96
#define SCK_MADE_NPARAM (256 * 160 + 256 + 2 * (256 * 256 + 256) + 64 * 256 + 64)

/* Sizes: param_bytes of the parameter buffer; adam_bytes of the Adam moments (2 x SCK_MADE_NPARAM floats);
 * train_bytes of the workspace of sck_made_grads / sck_made_train_step / sck_made_forward for `batch` rows
 * (batch a positive multiple of 64). Any output pointer may be null. */
int sck_made_sizes(int32_t groups, int32_t batch, int64_t* param_bytes, int64_t* adam_bytes, int64_t* train_bytes);

/* Write the masked bfloat16 weight copies from the FP32 masters (after initialising or changing them). */
int sck_made_prepare(void* params, int32_t groups, void* stream);

/* Block inputs of every block (all colours) of R replicas: out[(r * nb^3 + block) * 160 + i], bfloat16, block
 * = bx + nb by + nb^2 bz, nb = L / 4. */
int sck_made_gather(const int8_t* spins, int32_t R, int32_t L, uint16_t* out, void* stream);

/* Logits (FP32 [batch][64]) and log q (FP32 [batch], may be null) of `batch` block-input rows. */
int sck_made_forward(const void* params, int32_t groups, const uint16_t* x, int32_t batch, float* logits,
                     float* logq, void* workspace, void* stream);

/* Mean negative log-density over `batch` rows (written to *loss, device FP32, may be null) and its gradients
 * (masked), FP32 in the master layout (SCK_MADE_NPARAM floats). Backward GEMMs take bfloat16 gradients. */
int sck_made_grads(const void* params, int32_t groups, const uint16_t* x, int32_t batch, float* grads,
                   float* loss, void* workspace, void* stream);

/* One Adam step on the masters (moments in `adam`, step t >= 1 for the bias corrections), then
 * sck_made_prepare. */
int sck_made_train_step(void* params, float* adam, int32_t groups, const uint16_t* x, int32_t batch, float lr,
                        float beta1, float beta2, float eps, int32_t t, float* loss, void* workspace,
                        void* stream);

/* One colour step: every block of colour `colour` (0..7) in every replica proposes x' ~ q(. | boundary) and
 * accepts it with probability min(1, exp(-beta_r (E(x') - E(x))) q(x | b) / q(x' | b)) (J = 1, h = 0).
 * Philox4x32-10 key (seed * 1000003 + (8 round + colour) * 7919 + 24680) mod 2147483629, counter 17 uid + w
 * (uid = replica * nb^3 + block): call w < 16 gives the uniforms of positions 4w..4w+3, call 16 output 0 the
 * acceptance uniform; x'_p = +1 iff u_p < sigmoid(logit_p). `accepted` (int32 per replica, may be null) is
 * incremented by the number of accepted blocks. `record` (may be null) receives per block task
 * (replica r, k-th block of the colour in raster order) 64 int8 proposed spins at record + 80 (r nc + k) and
 * 4 FP32 (log q(x'), log q(x), E(x') - E(x), accepted) after them (nc = nb^3 / 8). */
int sck_made_colour_step(const void* params, int32_t groups, int8_t* spins, int32_t R, int32_t L, const float* beta,
                         int32_t colour, int64_t seed, int32_t round, int32_t* accepted, void* record,
                         void* stream);

/* Bounded waits. The tensor-core forward GEMM (training and sck_made_forward, 128-row batches) waits on its
 * stages' mbarriers with an iteration limit (default 2^22 polls; sck_made_set_wait_limit sets it on the current
 * device, synchronously; 0 makes every stage wait give up at once, for failure-detection tests). A block whose
 * wait gives up waits for its products in flight, leaves its output rows unwritten and counts itself;
 * sck_made_wait_status synchronises `stream` and returns SCK_ERR_TIMEOUT when a wait on the current device gave
 * up since its last status read. */
int sck_made_set_wait_limit(int64_t polls);
int sck_made_wait_status(void* stream);

#ifdef __cplusplus
}
#endif

#endif
