/*
 * sck.h — C ABI of libsckb200.so: the colour-class Metropolis sweep of spin-colour-kernel on B200 (sm_100a).
 *
 * The reference crosses from host to device in exactly one place on this path: the launch of its generated
 * Triton class kernel,
 *     kernel[grid](src_ptr, dst_ptr, mask_ptr, k1_ptr, beta_ptr | p_ptr, state_ptr, x_only, row0[, nword],
 *                  ALPHA=, COLOUR=, BLOCK=, SYNC=, STRIDE=, BX=, R=[, G=])
 * (Spin_Colour_Kernel/generator.py:191-194, bitwise.py:278-281), issued only by Sampler._launch
 * (sampler.py:191-232). This header replaces that launch and the Sampler methods built on it.
 *
 * Conventions (as in the reference):
 *   - Device buffers are caller-owned and updated in place. `state` = {base_seed, sweep} (int64) lives on the
 *     device; a sweep advances state[1] on the device, so a captured CUDA graph keeps the random stream.
 *   - Every call is asynchronous on the given stream (a cudaStream_t passed as void*, NULL = default stream),
 *     allocates nothing, synchronises nothing, and may be captured into a CUDA graph (the set-up calls excepted:
 *     sck_plan_tune allocates the group pipeline's counters when it enables the pipeline; the counter queries
 *     such as sck_wait_timeouts synchronise).
 *   - Every function returns 0 (SCK_OK) or a negative SCK_ERR_* code; sck_last_error() explains the last
 *     failure of the calling thread. Kernels never trap.
 *   - Layout: S[B, n, b, L3, L2, L1] (x fastest; L3 = 1 in 2D) in the plan's storage type; packed and bitwise
 *     storage hold W = ceil(B / 32) int32 words per site, bit j of word w = replica 32 w + j (1 = spin +1).
 *   - Interleaved storage (SCK_MODE_QUAD, vector models) holds Q = ceil(B / 4) quads of n * sites float4
 *     elements; lane j of an element is replica 4 q + j (lanes past B are padding: swept, never observed). Within
 *     a quad, element (((alpha L3 + z) L2 + y) n + k) L1 + (x mod P) (L1 / P) + x / P holds component k of site
 *     (alpha, z, y, x), P being the colouring's x-period (1 or 2): the rows of one class are contiguous. It is
 *     the sampler's resident state, converted from and to S by sck_quad_pack / sck_quad_unpack, as the
 *     reference converts its packed Ising words (Sampler.pack / unpack). Spins and beta must be 16-byte aligned.
 */
#ifndef SCK_H
#define SCK_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SCK_ABI_VERSION 1

/* status codes */
#define SCK_OK 0
#define SCK_ERR_INVALID (-1)      /* bad descriptor or argument (ValueError in the reference) */
#define SCK_ERR_COUNTER (-2)      /* replicas x sites >= 2^31 - 1: the int32 Philox counter would wrap */
#define SCK_ERR_UNSUPPORTED (-3)  /* mode not available for this system (e.g. bitwise on a vector model) */
#define SCK_ERR_CUDA (-4)         /* a CUDA runtime call failed */
#define SCK_ERR_TIMEOUT (-5)      /* a bounded device-side wait gave up */

/* storage / update modes (Sampler(packed=, bitwise=, independent=) in the reference) */
#define SCK_MODE_INT8 0           /* Ising, int8 spins, per-replica Philox (generator.py, unpacked) */
#define SCK_MODE_F32 1            /* any n, float32 components (XY, Heisenberg; Ising with spin_dtype=float32) */
#define SCK_MODE_PACKED 2         /* Ising, 32 replicas per int32 word, per-replica Philox == SCK_MODE_INT8 */
#define SCK_MODE_BITWISE 3        /* Ising multi-spin coding, one uniform per (word, site, sweep) */
#define SCK_MODE_BITWISE_INDEP 4  /* Ising multi-spin coding, one 32-bit draw per (replica, site, sweep) */
#define SCK_MODE_QUAD 5           /* XY / Heisenberg, float32 components of four replicas interleaved (below) */

#define SCK_METROPOLIS 0
#define SCK_BARKER 1

#define SCK_MAX_BASIS 4
#define SCK_MAX_BONDS 64          /* bonds leaving one sublattice */
#define SCK_MAX_GROUPS 8          /* coupling groups (distinct J) per sublattice */
#define SCK_MAX_EXTRA 8           /* bonds with an extra n x n matrix per sublattice */
#define SCK_MAX_FACTORS 4         /* cyclic factors of the colouring group */

/* One bond leaving sublattice `alpha`: (c, alpha) -> (c + d, alpha2). */
typedef struct sck_bond {
  int32_t alpha2;
  int32_t d[3];                   /* cell offset along x, y, z (z = 0 in 2D) */
  int32_t group;                  /* coupling group; bonds are listed group by group */
  int32_t extra;                  /* slot of this bond's extra matrix, -1 if none */
  double J64;                     /* isotropic coupling of the bond's shell (FP64, for observables) */
} sck_bond;

/* The bonds of one sublattice in local-field accumulation order: coupling groups in first-appearance
 * order of their float J over the bond table, members in table order (generator.py:219-224). */
typedef struct sck_sublattice {
  int32_t n_bonds;
  int32_t n_groups;
  int32_t group_end[SCK_MAX_GROUPS];   /* bonds [group_end[g-1], group_end[g]) belong to group g */
  float group_J[SCK_MAX_GROUPS];       /* float32 J of the group */
  int32_t group_apply[SCK_MAX_GROUPS]; /* 0: J == 0, the group is loaded only for its extra matrices */
  int32_t n_extra;                     /* extra slots, in bond-table order */
  float extra[SCK_MAX_EXTRA][9];       /* float32 n x n matrix, row-major in a 3 x 3 block */
  double extra64[SCK_MAX_EXTRA][9];    /* FP64 copy for observables */
  sck_bond bonds[SCK_MAX_BONDS];
} sck_sublattice;

/* A validated system (Spin_Colour_Kernel/system.py:19-98) with its linear colouring
 * gamma(c, alpha) = K c + o_alpha (mod m), colour index mixed-radix over the factors (colouring.py:30-36). */
typedef struct sck_system_desc {
  int32_t abi_version;            /* SCK_ABI_VERSION */
  int32_t n;                      /* spin components: 1, 2 or 3 */
  int32_t dim;                    /* lattice dimension: 2 or 3 */
  int32_t b;                      /* basis sites */
  int32_t L[3];                   /* L1, L2, L3 cells (L3 = 1 in 2D) */
  int32_t periodic[3];
  int32_t acceptance;             /* SCK_METROPOLIS or SCK_BARKER */
  int32_t has_mask;               /* a site mask is passed with every call */
  int32_t has_cubic;              /* per-site k1 is passed with every call (n = 3 only) */
  float h[3];                     /* float32 field; components equal to 0 are skipped */
  double h64[3];
  float k2;                       /* (sx sy sz)^2 coefficient */
  double k2_64;
  int32_t n_factors;              /* colouring factors r (0 = one colour) */
  int32_t m[SCK_MAX_FACTORS];
  int32_t K[SCK_MAX_FACTORS][3];
  int32_t o[SCK_MAX_BASIS][SCK_MAX_FACTORS];
  int32_t n_classes;              /* sweep order: (colour, alpha) pairs, colour-major, empty classes skipped */
  int32_t classes[128][2];
  sck_sublattice sub[SCK_MAX_BASIS];
} sck_system_desc;

/* Device buffers of one sampler (caller-owned). */
typedef struct sck_buffers {
  void* spins;                    /* S in the plan's storage type, updated in place */
  const int8_t* mask;             /* b*L3*L2*L1 bytes, nonzero = spin present; NULL without a mask */
  const float* k1;                /* b*L3*L2*L1 floats; NULL without cubic anisotropy */
  const float* beta;              /* one float32 inverse temperature per computed replica */
  const void* table;              /* acceptance table: see sck_plan_table_size */
  int64_t* state;                 /* {base_seed, sweep} */
} sck_buffers;

typedef struct sck_plan sck_plan;

/* Build a plan (host-only; no device memory) for `batch` replicas in `mode`. Errors: SCK_ERR_INVALID for a
 * malformed descriptor, SCK_ERR_COUNTER when ceil(batch) * sites >= 2^31 - 1 (sampler.py:73-74),
 * SCK_ERR_UNSUPPORTED for a mode the system cannot run (bitwise.py:59-71, sampler.py:62-63). */
int sck_plan_create(const sck_system_desc* desc, int32_t batch, int32_t mode, sck_plan** out);
int sck_plan_destroy(sck_plan* plan);

/* Size in elements of the acceptance table the plan reads, and its element size in bytes:
 *   INT8 / F32 Ising / PACKED: float32 e[Bp][b][keys] with e = exp(-beta dE) (Metropolis) or exp(beta dE)
 *       (Barker) for every reachable Ising energy change, built by the host with the same float32 arithmetic
 *       and exp as the reference's CPU path; keys per sublattice via *keys (may be NULL).
 *   F32 vector models: no table (0).
 *   BITWISE: float32 p[W][2][Z+1][Z+1] (bitwise.py:79-84).  BITWISE_INDEP: int64 P[W][2][Z+1][Z+1] (:87-93). */
int sck_plan_table_size(const sck_plan* plan, int64_t* elements, int32_t* element_bytes, int32_t* keys);

/* Replicas the kernels compute (B, or 32 W for packed storage) and the number of storage rows (B or W). */
int sck_plan_shape(const sck_plan* plan, int32_t* computed_replicas, int32_t* rows);

/* Execution choices of sck_sweep (set by the autotuner; the chain does not depend on them):
 *   specialised           3: compile-time lattice kernels and, where eligible, the tile kernels (vector
 *                         models, periodic box, L1 of 32, 64 or 128, rows a multiple of 8: neighbours
 *                         read from shared memory);
 *                         2: lattice kernels and, where eligible, the segment kernels (vector models,
 *                         periodic box, classes alternating along x);
 *                         1: compile-time lattice kernels only (default); 0: generic kernels;
 *   l2_budget_bytes       L2 bytes the group pipeline may fill; 0 disables it (the default: the class kernels
 *                         are issue-bound, and the pipeline's ordering costs more than the saved HBM traffic).
 *                         Enabling it allocates the pipeline's completion counters (4 bytes per replica group
 *                         and class) on the current device, which then runs this plan's sweeps; freed by
 *                         sck_plan_destroy. Call it outside stream capture;
 *   resident_limit_bytes  replicas up to this size (int8 / float32 storage) run all sweeps of a call in shared
 *                         memory, one block per replica; 0 disables it (default 200 KiB, at most 220 KiB).
 * sck_plan_path reports the chosen path: specialised = 100 * kernel kind (1 lattice, 2 segment, 3 tile) + table
 * id (0 = generic), budget, pipeline group (replicas per group; 0 = class by class over all replicas) and whether
 * sweeps run resident. No counterpart in the
 * reference, whose Triton launch geometry plays this role (Sampler.__init__,
 * sampler.py:84-115). */
int sck_plan_tune(sck_plan* plan, int32_t specialised, int64_t l2_budget_bytes, int64_t resident_limit_bytes);
int sck_plan_path(const sck_plan* plan, int32_t* specialised, int64_t* l2_budget_bytes, int32_t* group,
                  int32_t* resident);

/* The class-skewed L2 pipeline of interleaved storage (SCK_MODE_QUAD plans; no counterpart in the reference,
 * whose sweeps launch class by class). Class-by-class launches read the whole state once per class; the pipeline
 * cuts the quads into groups of group_replicas / 4 quads and runs the classes of a group back to back, so that
 * its later classes find the group in L2. Class c of unit u (sweep-major groups) runs at position skew u + c:
 * skew = the class count runs the groups one after another, skew 1 overlaps the most groups (and needs the
 * largest L2 working set, about classes / skew + 1 groups). One launch carries a whole sck_sweep call; the
 * chain is identical to class-by-class launches. group_replicas = 0 returns to class-by-class launches. Set-up
 * (not capturable): allocates the ticket and completion counters on the current device and a host-mapped flag.
 * Errors: SCK_ERR_UNSUPPORTED for other plans; SCK_ERR_INVALID for a group that is not whole quads, a skew that
 * does not divide the class count, or too few groups for the skew (skew x groups must reach the class count).
 *
 * Bounded waits. Every device-side wait of a plan's kernels has an iteration limit (sck_plan_set_wait_limit,
 * default 2^20 polls, about a second; 0 makes every wait that is not already satisfied give up at once, which
 * failure-detection tests use): the pipelines' blocks waiting for the class they follow (this call and the
 * L2 budget of sck_plan_tune) and the tile kernels waiting for their bulk copies (sck_plan_tune level 3). A block
 * whose wait gives up leaves its sites unchanged and raises the plan's host-mapped flag (allocated when such a
 * path is chosen). sck_plan_wait_status synchronises `stream` and returns SCK_ERR_TIMEOUT (clearing the flag)
 * when a wait of this plan gave up since the last status read; until then sck_sweep and sck_sweep_measure of the
 * plan refuse with SCK_ERR_TIMEOUT. */
int sck_plan_pipeline(sck_plan* plan, int32_t group_replicas, int32_t skew);
/* Site blocks (256 class sites of a quad) that one pipeline ticket covers, 1 .. 64 (default 4): more per ticket
 * means fewer ticket, wait and completion operations, a coarser overlap between the classes. The chain does not
 * depend on it. No counterpart in the reference (its classes are separate launches). */
int sck_plan_pipeline_chunks(sck_plan* plan, int32_t site_blocks);
int sck_plan_set_wait_limit(sck_plan* plan, int64_t polls);
int sck_plan_wait_status(sck_plan* plan, void* stream);

/* One class launch: every site of class (colour, alpha) of every replica, read from `src`, written to
 * `buf->spins` (src may equal buf->spins). colour < 0 with sync != 0 is the synchronous control (every site of
 * the sublattice from `src`). Replaces kernel[grid](...) of generator.py:191 / bitwise.py:278. */
int sck_class_update(const sck_plan* plan, const sck_buffers* buf, const void* src, int32_t colour,
                     int32_t alpha, int32_t sync, void* stream);

/* n_sweeps sweeps in place (Sampler.sweep, sampler.py:234-240): all classes in order, then state[1] += 1. */
int sck_sweep(const sck_plan* plan, const sck_buffers* buf, int32_t n_sweeps, void* stream);

/* Synchronous control (Sampler.sync_sweep, sampler.py:271-279): every site from the previous state;
 * `scratch` is a caller buffer the size of the spins. */
int sck_sync_sweep(const sck_plan* plan, const sck_buffers* buf, void* scratch, int32_t n_sweeps, void* stream);

/* Sequential reference chain (Sampler.reference_sweep, sampler.py:281-293): class by class, sites one at a
 * time in raster order (z, y, x), same counters. One thread (or warp of 32 replicas) per replica; for small
 * systems and checks only. */
int sck_reference_sweep(const sck_plan* plan, const sck_buffers* buf, int32_t n_sweeps, void* stream);

/* FP64 observables (Sampler.energy / magnetization, sampler.py:296-345) of the first `batch` replicas (1 .. the
 * plan's batch) stored as `storage` (SCK_MODE_INT8: int8 spins, SCK_MODE_F32: float32 components,
 * SCK_MODE_PACKED: int32 words, SCK_MODE_QUAD: interleaved quads of a SCK_MODE_QUAD plan):
 *   E[r]            = -1/2 sum_i s_i . v_i - sum_i h . s_i + sum_i a(s_i)   (r < batch)
 *   M[r][alpha][k]  = sum over sublattice alpha of s_k                       (batch x b x n doubles)
 * `workspace` holds per-block partial sums; its size in bytes comes from sck_observables_workspace_size.
 * Either output may be NULL. Deterministic: the partials are summed in a fixed order. */
int sck_observables_workspace_size(const sck_plan* plan, int32_t batch, int64_t* bytes);
int sck_observables(const sck_plan* plan, const sck_buffers* buf, const void* spins, int32_t storage,
                    int32_t batch, double* E, double* M, void* workspace, void* stream);

/* A measure step: n_sweeps sweeps in place (as sck_sweep), then the FP64 observables of the configuration they
 * leave, E[batch] and M[batch][b][n] for the plan's batch (Sampler.sweep followed by Sampler.energy /
 * magnetization, sampler.py:234-345, fused). With interleaved storage (SCK_MODE_QUAD) on a colouring whose
 * coupling groups never mix neighbours of earlier and later classes (every lattice-table system the
 * interleaved plans take), the last sweep's class launches accumulate them as they go: each bond is counted
 * once, by its later endpoint, when both its spins are final, so no pass re-reads the state. Each site's energy
 * share is formed in float32 from the float32 local fields of the sweep and summed in FP64 (energies agree with
 * sck_observables to float32 rounding of the shares, magnetizations to FP64 rounding); other plans run the
 * sweeps and then the sck_observables pass (FP64 throughout). `workspace` holds
 * sck_sweep_measure_workspace_size bytes; deterministic, fixed-order sums. No counterpart in the reference. */
int sck_sweep_measure_workspace_size(const sck_plan* plan, int64_t* bytes);
int sck_sweep_measure(const sck_plan* plan, const sck_buffers* buf, int32_t n_sweeps, double* E, double* M,
                      void* workspace, void* stream);

/* One observation of a measure step folded into FP64 accumulators: the reference's ladder runner
 * (simulate_state, simulate.py:338-353) observes every `every` sweeps and accumulates, per replica r,
 *   acc[0*batch + r] += E - E_ref[r],  acc[1*batch + r] += (E - E_ref[r])^2,
 *   acc[2*batch + r] += |m|,           acc[3*batch + r] += |m|^2,            accv[r*n + k] += m_k,
 * with E the total FP64 energy and m = (sum over sublattices of M) / n_active the mean magnetization vector.
 * This entry point runs the sck_observables pass (E [batch], M [batch][b][n] receive the observation) and folds
 * it in on the device, each quantity rounded in the reference's operation order; no host work, so a measure
 * step of sweeps and this call can be captured in one CUDA graph. `workspace` as for sck_observables. */
int sck_observables_accumulate(const sck_plan* plan, const sck_buffers* buf, const void* spins, int32_t storage,
                               int32_t batch, double n_active, const double* E_ref, double* E, double* M,
                               double* acc, double* accv, void* workspace, void* stream);

/* Berg-Luscher topological charge per replica of z-layer `layer` of sublattice 0 (the nanodisk anneal's middle
 * layer, anneal.py:69-80 and Observer.__call__ :125-146): over every plaquette of the layer whose four corners
 * are active, the solid angles of its two spherical triangles, Q = sum / 4 pi, in FP64. Float32 Heisenberg
 * storage; Q holds `batch` doubles. No workspace; one block per replica. */
int sck_topological_charge(const sck_plan* plan, const sck_buffers* buf, const float* spins, int32_t batch,
                           int32_t layer, double* Q, void* stream);

/* sck_observables without a caller workspace — no counterpart in the reference (added for callers that cannot
 * allocate device memory: a host whose device memory all belongs to its own pool or caching allocator, a loop
 * that cannot afford the synchronisation an allocation may bring, an FFI binding that cannot own a device
 * buffer). The partial sums go to a fixed 2 MiB array compiled into the library, which every GPU that loads the
 * library keeps until the process exits; a request needing more (batch x blocks per replica x 16 doubles) fails
 * with SCK_ERR_INVALID — use sck_observables then. The entry point allocates nothing. Every call looks up the
 * array's device address in the current context; the first call on a device may load the library's kernels into
 * that context, so make that first call before any stream capture. Every call shares the
 * one array and leaves its partial sums there; no part needs clearing, since each slot the final sum reads is
 * written earlier in the same call, but calls that overlap on the GPU (other streams, other threads) race on it:
 * keep them ordered. */
int sck_observables_noalloc(const sck_plan* plan, const sck_buffers* buf, const void* spins, int32_t storage,
                            int32_t batch, double* E, double* M, void* stream);

/* Bounded device-side waits that gave up since the library was loaded (0 in normal operation). The tile
 * kernels wait on the shared-memory fill of a brick, the group pipeline's blocks on the completion of the class
 * task they follow, and the learned proposal's tcgen05 GEMMs on their tensor-core products, with an iteration
 * limit; a brick whose fill timed out and a pipeline block whose wait timed out leave their sites unchanged, a
 * GEMM tile whose products timed out leaves its output unwritten, and each adds one here. Reads the count from the current
 * device (synchronising it). No counterpart in the reference. */
int sck_wait_timeouts(int64_t* count);

/* Interleaved storage (SCK_MODE_QUAD plans): pack float32 S[B, n, b, L3, L2, L1] into quads (padding lanes 0),
 * unpack quads into S (padding lanes dropped). No counterpart in the reference, whose vector models keep S; the
 * analogue of its packed-word conversion (Sampler.pack / unpack, sampler.py:169-188). The plan accepts a
 * vector-model system with a compile-time lattice table (square, triangular, sc, bcc, bcc J1-J2, fcc; no extra
 * bond matrices), every axis periodic, no mask and a colouring of x-period 1 or 2 dividing L1; otherwise
 * sck_plan_create returns SCK_ERR_UNSUPPORTED. sck_sweep, sck_class_update (src = spins), sck_observables*
 * (storage SCK_MODE_QUAD) read the quads directly; the synchronous control, the sequential reference and the
 * topological charge take S (unpack first). */
int sck_quad_pack(const sck_plan* plan, const float* spins, void* quads, void* stream);
int sck_quad_unpack(const sck_plan* plan, const void* quads, float* spins, void* stream);

/* Storage conversion (Sampler.pack / unpack, sampler.py:169-188). pack: int8 spins [B, 1, b, L3, L2, L1]
 * (+-1, 0 masked) -> int32 words [W, 1, b, L3, L2, L1] (padding replicas 0). unpack: words -> int8 spins,
 * masked sites 0. */
int sck_pack(const sck_plan* plan, const int8_t* spins, int32_t* words, void* stream);
int sck_unpack(const sck_plan* plan, const int32_t* words, const int8_t* mask, int8_t* spins, void* stream);

/* Ragged batches (no counterpart in the reference, which runs one Sampler per system): several plans with one
 * storage mode (int8 or float32) and one spin dimension, of different crystal, size, mask, colouring and
 * temperatures, swept together. A call is one persistent launch driven by the per-system descriptors: blocks take
 * work items in ticket order; systems whose replica takes at most resident_limit_bytes of shared memory are one
 * item per replica that runs every sweep of the call on-chip, the others one item per (sweep, class, replica
 * slot, 2,048-site chunk), each waiting (bounded) for the class it follows in its own system to finish.
 *   sck_batch_workspace_size  device bytes of the per-system descriptors and the call's counters (caller-owned
 *                             workspace; one call at a time per workspace);
 *   sck_batch_bind            write the descriptors for these per-system buffers (a host-to-device copy on
 *                             `stream`: call it outside stream capture, again when a buffer moves); sizes the
 *                             persistent grid for the current device and allocates a host-mapped give-up flag;
 *   sck_batch_sweep           n sweeps of every system, kernel launches and a counter reset only (capturable);
 *                             each system's state[1] advances by n; refuses with SCK_ERR_TIMEOUT while a wait
 *                             that gave up is unread;
 *   sck_batch_set_wait_limit  polls of a wait before it gives up (default 2^20; 0 for failure-detection tests);
 *   sck_batch_wait_status     synchronise `stream`; SCK_ERR_TIMEOUT (clearing it) when a wait gave up;
 *   sck_batch_info            resident systems and items, streaming items per sweep. */
typedef struct sck_batch sck_batch;
int sck_batch_create(const sck_plan* const* plans, int32_t n_plans, int64_t resident_limit_bytes, sck_batch** out);
int sck_batch_destroy(sck_batch* batch);
int sck_batch_workspace_size(const sck_batch* batch, int64_t* bytes);
int sck_batch_bind(sck_batch* batch, const sck_buffers* buffers, void* workspace, void* stream);
int sck_batch_sweep(sck_batch* batch, void* workspace, int32_t n_sweeps, void* stream);
int sck_batch_info(const sck_batch* batch, int32_t* resident_systems, int32_t* resident_blocks, int64_t* step_blocks);
int sck_batch_set_wait_limit(sck_batch* batch, int64_t polls);
int sck_batch_wait_status(sck_batch* batch, void* stream);

/* Advance state[1] by `n` on the device (what a sweep does after its class launches). */
int sck_advance(int64_t* state, int32_t n, void* stream);

const char* sck_last_error(void);
int sck_abi_version(void);

/* sizeof of the ABI structs as compiled into the library, for FFI bindings to check their mirrors. */
int sck_struct_sizes(int64_t* system_desc, int64_t* sublattice, int64_t* bond, int64_t* buffers);

#ifdef __cplusplus
}
#endif

#endif /* SCK_H */
