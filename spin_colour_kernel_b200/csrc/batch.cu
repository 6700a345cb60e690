// Ragged batches: many systems of different size, crystal, mask and temperature swept together.
//
// A batch holds several plans with one storage mode. Per-system descriptors (geometry, colouring, bonds,
// device buffers) live in a caller-owned workspace on the device, written by sck_batch_bind, together with the
// call's ticket and completion counters. A call of n sweeps is ONE persistent launch: a grid sized to the
// resident capacity of the GPU whose blocks take work items in ticket order from a counter:
//   - resident items (system, replica), for systems whose replica fits shared memory: the block loads the
//     replica once and runs every class of every sweep of the call on-chip;
//   - streaming items (sweep, colour step k, system, replica slot, 2,048-site chunk) for the others, found by
//     binary searches over per-step item offsets. Before touching spins, a block waits (bounded) until every item of the
//     class its item follows is done: class k - 1 of the same system and sweep, or the system's last class of the
//     previous sweep; per-(system, class) completion counters count finished items. That class holds smaller
//     tickets, taken by blocks that are running or done, so every wait ends, and each system's classes are
//     serialised exactly as separate launches would serialise them, while different systems overlap freely.
// Both kinds read each system's descriptor from the workspace, so one kernel serves every crystal.
#include <string.h>

#include <algorithm>
#include <vector>

#include "site.cuh"
#include "spec_site.cuh"

namespace sck {

// In-place site update of replica `rep` whose block starts at `spins` (global or shared memory).
template <int N, typename ST>
__device__ __forceinline__ void batch_site(const Common& c, const SubDev& sub, int alpha, int rep, int x, int y,
                                           int z, int32_t key, ST* spins) {
  if constexpr (N == 1)
    ising_site<ST>(c, sub, alpha, rep, x, y, z, key, spins, spins);
  else
    vec_site<N>(c, sub, alpha, rep, x, y, z, key, (const float*)spins, (float*)spins);
}

constexpr int kBatchMaxSystems = 256;
constexpr int kBatchItemPasses = 8;   // a streaming item: 8 x 256 class sites of one replica slot and class
constexpr int kBatchMaxClasses = 32;

struct SysDev {
  Common c;
  SubDev sub[SCK_MAX_BASIS];
  int n_classes;
  int classes[kBatchMaxClasses][2];
  int resident;
  int chunks;          // streaming items of one class and replica slot (kBatchItemPasses x 256 class sites each)
  int rpi;             // replicas per streaming item: 2 for vector models (a pair in packed float32x2), 1 Ising
  int spec, per;       // compile-time lattice table of the system (0: generic site update), periodic wrap
  float J[SCK_MAX_BASIS][SCK_MAX_GROUPS];
};

struct BatchLayout {   // offsets into the workspace
  size_t sys;          // SysDev[n]
  size_t step_off;     // int[max_classes][n + 1]: first item of system s in colour step k (streaming)
  size_t res_off;      // int[n + 1]: first resident item of system s
  size_t k_off;        // long long[max_classes + 1]: first item of colour step k within a sweep
  size_t counters;     // unsigned[1 + n max_classes]: ticket, then finished items per (system, class)
};

struct BatchDevParams {
  const SysDev* sys;
  const int* step_off;
  const int* res_off;
  const long long* k_off;
  int n, max_classes;
  int res_items;                // resident items of a launch
  long long step_items;         // streaming items of one sweep
  int n_sweeps, sweep_base;     // sweeps of this launch, offset of its first sweep within the call
  unsigned* ticket;
  unsigned* done;
  unsigned wait_limit;
  int* giveup;
};

}  // namespace sck

struct sck_batch {
  std::vector<const sck_plan*> plans;
  int n, mode, ncomp;
  int max_classes;
  std::vector<int> resident;      // per system
  size_t resident_smem;
  long long resident_limit;
  sck::BatchLayout layout;
  size_t bytes;
  std::vector<unsigned char> staging;   // host image of the workspace
  std::vector<int> step_blocks;   // total items per colour step
  int resident_blocks;
  long long step_items;           // streaming items per sweep
  int grid;                       // persistent blocks of a launch (resident capacity of the device)
  int device;                     // the device bind sized the grid for
  unsigned wait_limit;
  int* giveup_host;               // host-mapped flag a block raises when a wait gives up
  int* giveup_dev;
  bool bound;
};

namespace sck {

__device__ __forceinline__ int find_system(const int* off, int n, int block) {
  int lo = 0, hi = n;   // off[lo] <= block < off[hi]
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (off[mid] <= block) lo = mid;
    else hi = mid;
  }
  return lo;
}

__device__ __forceinline__ int find_step(const long long* k_off, int K, long long item) {
  int k = 0;
  while (k + 1 < K && k_off[k + 1] <= item) ++k;
  return k;
}

__device__ __forceinline__ unsigned batch_ld_acquire(const unsigned* a) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(a) : "memory");
  return v;
}

// The site update of a streaming item: the specialised lattice update (the lattice kernels' arithmetic, a
// replica pair per thread for vector models) for systems on the square, triangular or simple cubic table, else
// the generic update of each replica of the slot.
template <class Lat, int N, typename ST>
__device__ __forceinline__ void batch_spec_site(const SysDev& d, int rep0, int x, int y, int z, int32_t key) {
  auto run = [&](auto per_c) {
    constexpr bool PER = decltype(per_c)::value;
    if constexpr (N == 1)
      ising_spec_site<Lat, 0, ST, PER>(d.c, rep0, x, y, z, key);
    else
      vec_spec_pair<Lat, 0, N, PER, 0>(d.c, d.J[0], rep0, rep0 + 1 < d.c.B, x, y, z, key);
  };
  if (d.per) run(std::true_type{});
  else run(std::false_type{});
}

template <int N, typename ST>
__device__ __forceinline__ void batch_stream_site(const SysDev& d, int alpha, int rep0, int x, int y, int z,
                                                  int32_t key) {
  if (d.spec == Lat_square_1::id) return batch_spec_site<Lat_square_1, N, ST>(d, rep0, x, y, z, key);
  if (d.spec == Lat_triangular_1::id) return batch_spec_site<Lat_triangular_1, N, ST>(d, rep0, x, y, z, key);
  if (d.spec == Lat_sc_1::id) return batch_spec_site<Lat_sc_1, N, ST>(d, rep0, x, y, z, key);
  ST* base = (ST*)d.c.dst;
  for (int r = rep0; r < rep0 + d.rpi && r < d.c.B; ++r)
    batch_site<N, ST>(d.c, d.sub[alpha], alpha, r, x, y, z, key, base + (size_t)r * N * d.c.g.nsite);
}

struct BatchItem {
  int kind;      // 0: no more work, 1: resident, 2: streaming, 3: streaming item whose wait gave up
  int s, rep, chunk, k, sw;
};

// The persistent batch kernel: 256 threads per block (at most 64 registers: four blocks per SM when the
// resident replicas allow), dynamic shared memory for the largest resident replica.
template <int N, typename ST>
__global__ void __launch_bounds__(256, 4) batch_persistent_kernel(const BatchDevParams p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ BatchItem it;
  const long long total = (long long)p.res_items + (long long)p.n_sweeps * p.step_items;
  for (;;) {
    if (threadIdx.x == 0) {
      const long long tk = (long long)atomicAdd(p.ticket, 1u);
      it.kind = 0;
      if (tk < p.res_items) {
        const int s = find_system(p.res_off, p.n, (int)tk);
        it.kind = 1;
        it.s = s;
        it.rep = (int)tk - p.res_off[s];
      } else if (tk < total) {
        const long long u = tk - p.res_items;
        const int sw = (int)(u / p.step_items);
        const long long r = u - (long long)sw * p.step_items;
        const int k = find_step(p.k_off, p.max_classes, r);
        const int local = (int)(r - p.k_off[k]);
        const int* off = p.step_off + (size_t)k * (p.n + 1);
        const int s = find_system(off, p.n, local);
        const SysDev& d = p.sys[s];
        const int j = local - off[s];
        it.kind = 2;
        it.s = s;
        it.k = k;
        it.sw = sw;
        it.rep = j / d.chunks;
        it.chunk = j - it.rep * d.chunks;
        // the class this item follows: k - 1 of this sweep, or the last class of the previous sweep
        const unsigned per = (unsigned)d.chunks * (unsigned)((d.c.B + d.rpi - 1) / d.rpi);
        const unsigned* dep = nullptr;
        unsigned need = 0;
        if (k > 0) {
          dep = p.done + (size_t)s * p.max_classes + (k - 1);
          need = (unsigned)(sw + 1) * per;
        } else if (sw > 0) {
          dep = p.done + (size_t)s * p.max_classes + (d.n_classes - 1);
          need = (unsigned)sw * per;
        }
        if (dep != nullptr) {
          unsigned polls = 0;
          while (batch_ld_acquire(dep) < need) {
            if (++polls > p.wait_limit) {
              it.kind = 3;
              if (p.giveup != nullptr) atomicExch_system(p.giveup, 1);
              break;
            }
            __nanosleep(64);
          }
        }
      }
    }
    __syncthreads();
    const int kind = it.kind;
    if (kind == 0) return;
    const SysDev& d = p.sys[it.s];
    if (kind == 1) {
      ST* S = reinterpret_cast<ST*>(smem_raw);
      const int n = N * d.c.g.nsite;
      ST* home = (ST*)d.c.dst + (size_t)it.rep * n;
      for (int i = threadIdx.x; i < n; i += blockDim.x) S[i] = home[i];
      __syncthreads();
      const uint32_t per = (uint32_t)d.c.rows * (uint32_t)d.c.bx;
      for (int sw = 0; sw < p.n_sweeps; ++sw) {
        const int32_t key = sweep_key_at(d.c.state, p.sweep_base + sw);
        for (int ci = 0; ci < d.n_classes; ++ci) {
          const int colour = d.classes[ci][0], alpha = d.classes[ci][1];
          for (uint32_t t = threadIdx.x; t < per; t += blockDim.x) {
            int x, y, z;
            if (class_site(d.c, colour, alpha, t, x, y, z))
              batch_site<N, ST>(d.c, d.sub[alpha], alpha, it.rep, x, y, z, key, S);
          }
          __syncthreads();
        }
      }
      for (int i = threadIdx.x; i < n; i += blockDim.x) home[i] = S[i];
    } else {
      if (kind == 2) {
        const uint32_t per = (uint32_t)d.c.rows * (uint32_t)d.c.bx;
        const int colour = d.classes[it.k][0], alpha = d.classes[it.k][1];
        const int32_t key = sweep_key_at(d.c.state, p.sweep_base + it.sw);
        const int rep0 = it.rep * d.rpi;
#pragma unroll 1
        for (int pass = 0; pass < kBatchItemPasses; ++pass) {
          const uint32_t t = ((uint32_t)it.chunk * kBatchItemPasses + pass) * 256u + threadIdx.x;
          int x, y, z;
          if (t < per && class_site(d.c, colour, alpha, t, x, y, z))
            batch_stream_site<N, ST>(d, alpha, rep0, x, y, z, key);
        }
      }
      __syncthreads();
      // done (or given up): the class's next items may start; the barrier orders the block's stores before it
      if (threadIdx.x == 0)
        asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(p.done + (size_t)it.s * p.max_classes + it.k)
                     : "memory");
    }
    __syncthreads();   // `it` is rewritten by the next ticket
  }
}

// state[1] += inc for every system.
__global__ void batch_advance_kernel(const SysDev* sys, int n, int inc) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < n) const_cast<int64_t*>(sys[s].c.state)[1] += inc;
}

template <int N, typename ST>
static int batch_prepare(sck_batch* b) {
  cudaError_t e = cudaFuncSetAttribute(batch_persistent_kernel<N, ST>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)b->resident_smem);
  if (e != cudaSuccess) return cuda_status(e, "batch shared memory");
  int dev = 0, sms = 0, per_sm = 0;
  e = cudaGetDevice(&dev);
  b->device = dev;
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e == cudaSuccess)
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batch_persistent_kernel<N, ST>, 256, b->resident_smem);
  if (e != cudaSuccess) return cuda_status(e, "batch occupancy");
  b->grid = sms * (per_sm > 0 ? per_sm : 1);
  return SCK_OK;
}

template <int N, typename ST>
static int run_batch(const sck_batch* b, unsigned char* ws, int n_sweeps, cudaStream_t st) {
  BatchDevParams p;
  memset(&p, 0, sizeof(p));
  p.sys = (const SysDev*)(ws + b->layout.sys);
  p.step_off = (const int*)(ws + b->layout.step_off);
  p.res_off = (const int*)(ws + b->layout.res_off);
  p.k_off = (const long long*)(ws + b->layout.k_off);
  p.n = b->n;
  p.max_classes = b->max_classes;
  p.res_items = b->resident_blocks;
  p.step_items = b->step_items;
  p.ticket = (unsigned*)(ws + b->layout.counters);
  p.done = p.ticket + 1;
  p.wait_limit = b->wait_limit;
  p.giveup = b->giveup_dev;
  const size_t counter_bytes = sizeof(unsigned) * (1 + (size_t)b->n * b->max_classes);
  // sweeps per launch: tickets and per-class completion counts stay below 2^31
  long long per_launch = b->step_items > 0 ? ((1ll << 31) - 1 - b->resident_blocks) / b->step_items : n_sweeps;
  if (per_launch < 1) return cuda_status(cudaErrorInvalidConfiguration, "batch too large for one launch");
  for (int sw0 = 0; sw0 < n_sweeps; sw0 += (int)per_launch) {
    p.sweep_base = sw0;
    p.n_sweeps = (int)std::min<long long>(per_launch, n_sweeps - sw0);
    int rc = cuda_status(cudaMemsetAsync(p.ticket, 0, counter_bytes, st), "batch counters");
    if (rc != SCK_OK) return rc;
    const long long items = (long long)p.res_items + (long long)p.n_sweeps * p.step_items;
    const int grid = (int)std::min<long long>(b->grid, items);
    if (grid > 0) {
      batch_persistent_kernel<N, ST><<<grid, 256, b->resident_smem, st>>>(p);
      rc = cuda_status(cudaGetLastError(), "batch launch");
      if (rc != SCK_OK) return rc;
    }
  }
  batch_advance_kernel<<<(b->n + 127) / 128, 128, 0, st>>>(p.sys, b->n, n_sweeps);
  return cuda_status(cudaGetLastError(), "batch advance");
}

int batch_sweep_dispatch(const sck_batch* b, unsigned char* ws, int n_sweeps, cudaStream_t st) {
  if (b->mode == SCK_MODE_INT8) return run_batch<1, int8_t>(b, ws, n_sweeps, st);
  switch (b->ncomp) {
    case 1: return run_batch<1, float>(b, ws, n_sweeps, st);
    case 2: return run_batch<2, float>(b, ws, n_sweeps, st);
    default: return run_batch<3, float>(b, ws, n_sweeps, st);
  }
}

int batch_prepare_dispatch(sck_batch* b) {
  if (b->mode == SCK_MODE_INT8) return batch_prepare<1, int8_t>(b);
  switch (b->ncomp) {
    case 1: return batch_prepare<1, float>(b);
    case 2: return batch_prepare<2, float>(b);
    default: return batch_prepare<3, float>(b);
  }
}

Common make_common_public(const sck_plan* plan, const sck_buffers* buf);

}  // namespace sck

using namespace sck;

static size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

static int batch_fail(int code, const char* msg) {
  set_error(msg);
  return code;
}

extern "C" {

int sck_batch_create(const sck_plan* const* plans, int32_t n_plans, int64_t resident_limit_bytes, sck_batch** out) {
  if (plans == nullptr || out == nullptr || n_plans < 1 || n_plans > kBatchMaxSystems)
    return batch_fail(SCK_ERR_INVALID, "a batch holds 1 to 256 plans");
  if (resident_limit_bytes < 0 || resident_limit_bytes > (220ll << 10))
    return batch_fail(SCK_ERR_INVALID, "resident limit must be within 0 .. 220 KiB");
  *out = nullptr;
  const int mode = plans[0]->mode, ncomp = plans[0]->geom.n;
  if (mode != SCK_MODE_INT8 && mode != SCK_MODE_F32)
    return batch_fail(SCK_ERR_UNSUPPORTED, "batches hold int8 or float32 storage");
  for (int i = 0; i < n_plans; ++i) {
    if (plans[i] == nullptr) return batch_fail(SCK_ERR_INVALID, "null plan in batch");
    if (plans[i]->mode != mode || plans[i]->geom.n != ncomp)
      return batch_fail(SCK_ERR_INVALID, "every plan of a batch needs the same storage mode and spin components");
    if (plans[i]->desc.n_classes > kBatchMaxClasses)
      return batch_fail(SCK_ERR_UNSUPPORTED, "batched systems have at most 32 colour classes");
  }
  sck_batch* b = new sck_batch();
  b->plans.assign(plans, plans + n_plans);
  b->n = n_plans;
  b->mode = mode;
  b->ncomp = ncomp;
  b->resident_limit = resident_limit_bytes;
  b->max_classes = 0;
  b->resident_smem = 0;
  b->resident.resize(n_plans);
  for (int i = 0; i < n_plans; ++i) {
    const size_t bytes = resident_bytes(plans[i]);
    b->resident[i] = (long long)bytes <= resident_limit_bytes ? 1 : 0;
    if (b->resident[i]) b->resident_smem = std::max(b->resident_smem, align_up(bytes, 16));
    b->max_classes = std::max(b->max_classes, plans[i]->desc.n_classes);
  }
  b->layout.sys = 0;
  b->layout.step_off = align_up(sizeof(SysDev) * n_plans, 256);
  b->layout.res_off = align_up(b->layout.step_off + sizeof(int) * (size_t)b->max_classes * (n_plans + 1), 256);
  b->layout.k_off = align_up(b->layout.res_off + sizeof(int) * (size_t)(n_plans + 1), 256);
  b->layout.counters = align_up(b->layout.k_off + sizeof(long long) * (size_t)(b->max_classes + 1), 256);
  b->bytes = align_up(b->layout.counters + sizeof(unsigned) * (1 + (size_t)n_plans * b->max_classes), 256);
  b->staging.assign(b->bytes, 0);
  b->step_blocks.assign(b->max_classes, 0);
  b->resident_blocks = 0;
  b->step_items = 0;
  b->grid = 0;
  b->device = -1;
  b->wait_limit = 1u << 20;
  b->giveup_host = nullptr;
  b->giveup_dev = nullptr;
  b->bound = false;
  *out = b;
  return SCK_OK;
}

int sck_batch_destroy(sck_batch* batch) {
  if (batch != nullptr && batch->giveup_host != nullptr) cudaFreeHost(batch->giveup_host);
  delete batch;
  return SCK_OK;
}

int sck_batch_set_wait_limit(sck_batch* batch, int64_t polls) {
  if (batch == nullptr || polls < 0 || polls > 0xFFFFFFFFll)
    return batch_fail(SCK_ERR_INVALID, "polls must be 0 .. 2^32-1");
  batch->wait_limit = (unsigned)polls;
  return SCK_OK;
}

int sck_batch_wait_status(sck_batch* batch, void* stream) {
  if (batch == nullptr) return batch_fail(SCK_ERR_INVALID, "null batch");
  if (batch->giveup_host == nullptr) return SCK_OK;
  const int rc = cuda_status(cudaStreamSynchronize((cudaStream_t)stream), "batch wait status");
  if (rc != SCK_OK) return rc;
  if (*(volatile int*)batch->giveup_host) {
    *(volatile int*)batch->giveup_host = 0;
    return batch_fail(SCK_ERR_TIMEOUT, "a bounded wait of the batch kernel gave up: the affected sites were left "
                                       "unchanged");
  }
  return SCK_OK;
}

int sck_batch_workspace_size(const sck_batch* batch, int64_t* bytes) {
  if (batch == nullptr || bytes == nullptr) return batch_fail(SCK_ERR_INVALID, "null batch or output");
  *bytes = (int64_t)batch->bytes;
  return SCK_OK;
}

int sck_batch_bind(sck_batch* b, const sck_buffers* buffers, void* workspace, void* stream) {
  if (b == nullptr || buffers == nullptr || workspace == nullptr)
    return batch_fail(SCK_ERR_INVALID, "null batch, buffers or workspace");
  unsigned char* img = b->staging.data();
  SysDev* sys = (SysDev*)(img + b->layout.sys);
  int* step_off = (int*)(img + b->layout.step_off);
  int* res_off = (int*)(img + b->layout.res_off);
  long long res_total = 0;
  std::vector<long long> step_total(b->max_classes, 0);
  for (int s = 0; s < b->n; ++s) {
    const sck_plan* plan = b->plans[s];
    const sck_buffers& bu = buffers[s];
    if (bu.spins == nullptr || bu.state == nullptr) return batch_fail(SCK_ERR_INVALID, "null spins or state in batch");
    if (plan->geom.has_mask && bu.mask == nullptr) return batch_fail(SCK_ERR_INVALID, "a batched system needs its mask");
    if (plan->geom.has_cubic && bu.k1 == nullptr) return batch_fail(SCK_ERR_INVALID, "a batched system needs k1");
    if (plan->ising_lut ? bu.table == nullptr : bu.beta == nullptr)
      return batch_fail(SCK_ERR_INVALID, "a batched system needs its beta / acceptance table");
    SysDev& d = sys[s];
    memset(&d, 0, sizeof(d));
    d.c = make_common_public(plan, &bu);
    for (int a = 0; a < SCK_MAX_BASIS; ++a) d.sub[a] = plan->sub[a];
    d.n_classes = plan->desc.n_classes;
    for (int i = 0; i < d.n_classes; ++i) {
      d.classes[i][0] = plan->desc.classes[i][0];
      d.classes[i][1] = plan->desc.classes[i][1];
    }
    d.resident = b->resident[s];
    const long long per = (long long)d.c.rows * d.c.bx;
    d.chunks = (int)((per + 256 * kBatchItemPasses - 1) / (256 * kBatchItemPasses));
    d.rpi = plan->geom.n == 1 ? 1 : 2;
    const bool table = plan->spec == Lat_square_1::id || plan->spec == Lat_triangular_1::id ||
                       plan->spec == Lat_sc_1::id;
    d.spec = table ? plan->spec : 0;
    d.per = table ? spec_periodic_box(plan) : 0;
    for (int a = 0; a < SCK_MAX_BASIS; ++a)
      for (int gi = 0; gi < SCK_MAX_GROUPS; ++gi) d.J[a][gi] = plan->sub[a].J[gi];
    res_off[s] = (int)res_total;
    if (d.resident) res_total += plan->Bp;
    const long long slots = (plan->Bp + d.rpi - 1) / d.rpi;
    for (int k = 0; k < b->max_classes; ++k) {
      step_off[k * (b->n + 1) + s] = (int)step_total[k];
      if (!d.resident && k < d.n_classes) step_total[k] += (long long)d.chunks * slots;
    }
  }
  res_off[b->n] = (int)res_total;
  long long* k_off = (long long*)(img + b->layout.k_off);
  long long items = 0;
  for (int k = 0; k < b->max_classes; ++k) {
    if (step_total[k] >= (1ll << 31)) return batch_fail(SCK_ERR_UNSUPPORTED, "batch too large for one launch");
    step_off[k * (b->n + 1) + b->n] = (int)step_total[k];
    b->step_blocks[k] = (int)step_total[k];
    k_off[k] = items;
    items += step_total[k];
  }
  k_off[b->max_classes] = items;
  if (items + res_total >= (1ll << 31)) return batch_fail(SCK_ERR_UNSUPPORTED, "batch too large for one launch");
  b->step_items = items;
  b->resident_blocks = (int)res_total;
  // set-up outside any sweep: the kernel's shared-memory limit and grid, the give-up flag
  int rc0 = batch_prepare_dispatch(b);
  if (rc0 != SCK_OK) return rc0;
  if (b->giveup_host == nullptr) {
    rc0 = cuda_status(cudaHostAlloc((void**)&b->giveup_host, sizeof(int), cudaHostAllocMapped | cudaHostAllocPortable),
                      "batch give-up flag");
    if (rc0 != SCK_OK) {
      b->giveup_host = nullptr;
      return rc0;
    }
    *b->giveup_host = 0;
    rc0 = cuda_status(cudaHostGetDevicePointer((void**)&b->giveup_dev, b->giveup_host, 0), "batch give-up flag");
    if (rc0 != SCK_OK) return rc0;
  }
  const int rc = cuda_status(cudaMemcpyAsync(workspace, img, b->bytes, cudaMemcpyHostToDevice, (cudaStream_t)stream),
                             "batch descriptors");
  if (rc != SCK_OK) return rc;
  b->bound = true;
  return SCK_OK;
}

int sck_batch_sweep(sck_batch* b, void* workspace, int32_t n_sweeps, void* stream) {
  if (b == nullptr || workspace == nullptr || n_sweeps < 0) return batch_fail(SCK_ERR_INVALID, "bad batch sweep call");
  if (!b->bound) return batch_fail(SCK_ERR_INVALID, "bind the batch's buffers first (sck_batch_bind)");
  if (n_sweeps == 0) return SCK_OK;
  if (b->giveup_host != nullptr && *(volatile int*)b->giveup_host)
    return batch_fail(SCK_ERR_TIMEOUT, "an earlier bounded wait of this batch gave up (read sck_batch_wait_status)");
  int dev = -1;
  const int rc = cuda_status(cudaGetDevice(&dev), "batch sweep");
  if (rc != SCK_OK) return rc;
  if (dev != b->device) return batch_fail(SCK_ERR_INVALID, "the batch was bound on another device: bind it here");
  return batch_sweep_dispatch(b, (unsigned char*)workspace, n_sweeps, (cudaStream_t)stream);
}

int sck_batch_info(const sck_batch* b, int32_t* resident_systems, int32_t* resident_blocks, int64_t* step_blocks) {
  if (b == nullptr) return batch_fail(SCK_ERR_INVALID, "null batch");
  int r = 0;
  for (int v : b->resident) r += v;
  if (resident_systems) *resident_systems = r;
  if (resident_blocks) *resident_blocks = b->resident_blocks;
  if (step_blocks) {
    long long t = 0;
    for (int v : b->step_blocks) t += v;
    *step_blocks = t;
  }
  return SCK_OK;
}

}  // extern "C"
