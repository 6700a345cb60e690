// Ragged batches: many systems of different size, crystal, mask and temperature swept together.
//
// A batch holds several plans with one storage mode. Per-system descriptors (geometry, colouring, bonds,
// device buffers) live in a caller-owned workspace on the device, written by sck_batch_bind. A sweep of the
// batch then needs no host work:
//   - systems whose replica fits in shared memory run one resident launch for all of them: block (system,
//     replica) loads the replica once and runs every class of every sweep of the call on-chip;
//   - the other systems run one launch per colour step: step k updates class k of every system that has one,
//     every (system, replica, 256-site chunk) a block, found by a binary search over per-step block offsets.
// Both launch kinds read each system's descriptor from the workspace, so one kernel serves every crystal.
#include <string.h>

#include <algorithm>
#include <vector>

#include "site.cuh"

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
constexpr int kBatchMaxClasses = 32;

struct SysDev {
  Common c;
  SubDev sub[SCK_MAX_BASIS];
  int n_classes;
  int classes[kBatchMaxClasses][2];
  int resident;
  int chunks;          // 256-site chunks of one class (streaming systems)
};

struct BatchLayout {   // offsets into the workspace
  size_t sys;          // SysDev[n]
  size_t step_off;     // int[max_classes][n + 1]: first block of system s in colour step k (streaming)
  size_t res_off;      // int[n + 1]: first block of system s in the resident launch
};

struct BatchDevParams {
  const SysDev* sys;
  const int* offsets;  // n + 1 block offsets of this launch
  int n;
  int step;            // colour step (streaming) or number of sweeps (resident)
  int sweep_offset;
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
  std::vector<int> step_blocks;   // total blocks per colour step
  int resident_blocks;
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

template <int N, typename ST>
__global__ void __launch_bounds__(256) batch_step_kernel(const BatchDevParams p) {
  const int s = find_system(p.offsets, p.n, blockIdx.x);
  const SysDev& d = p.sys[s];
  if (d.resident || p.step >= d.n_classes) return;
  const int local = blockIdx.x - p.offsets[s];
  const int rep = local / d.chunks;
  const int chunk = local - rep * d.chunks;
  const uint32_t t = (uint32_t)chunk * 256u + threadIdx.x;
  if (t >= (uint32_t)d.c.rows * (uint32_t)d.c.bx) return;
  const int colour = d.classes[p.step][0], alpha = d.classes[p.step][1];
  int x, y, z;
  if (!class_site(d.c, colour, alpha, t, x, y, z)) return;
  const int32_t key = sweep_key(d.c.state);
  ST* spins = (ST*)d.c.dst + (size_t)rep * N * d.c.g.nsite;
  batch_site<N, ST>(d.c, d.sub[alpha], alpha, rep, x, y, z, key, spins);
}

template <int N, typename ST>
__global__ void __launch_bounds__(1024) batch_resident_kernel(const BatchDevParams p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  ST* S = reinterpret_cast<ST*>(smem_raw);
  const int s = find_system(p.offsets, p.n, blockIdx.x);
  const SysDev& d = p.sys[s];
  if (!d.resident) return;
  const int rep = blockIdx.x - p.offsets[s];
  const int n = N * d.c.g.nsite;
  ST* home = (ST*)d.c.dst + (size_t)rep * n;
  for (int i = threadIdx.x; i < n; i += blockDim.x) S[i] = home[i];
  __syncthreads();
  const uint32_t per = (uint32_t)d.c.rows * (uint32_t)d.c.bx;
  for (int sw = 0; sw < p.step; ++sw) {
    const int32_t key = sweep_key_at(d.c.state, sw);
    for (int ci = 0; ci < d.n_classes; ++ci) {
      const int colour = d.classes[ci][0], alpha = d.classes[ci][1];
      for (uint32_t t = threadIdx.x; t < per; t += blockDim.x) {
        int x, y, z;
        if (class_site(d.c, colour, alpha, t, x, y, z)) batch_site<N, ST>(d.c, d.sub[alpha], alpha, rep, x, y, z, key, S);
      }
      __syncthreads();
    }
  }
  for (int i = threadIdx.x; i < n; i += blockDim.x) home[i] = S[i];
}

// state[1] += inc for every system of the given kind (resident or streaming).
__global__ void batch_advance_kernel(const SysDev* sys, int n, int resident, int inc) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < n && sys[s].resident == resident) const_cast<int64_t*>(sys[s].c.state)[1] += inc;
}

template <int N, typename ST>
static int run_batch(const sck_batch* b, const unsigned char* ws, int n_sweeps, cudaStream_t st) {
  BatchDevParams p;
  p.sys = (const SysDev*)(ws + b->layout.sys);
  p.n = b->n;
  p.sweep_offset = 0;
  if (b->resident_blocks > 0) {
    p.offsets = (const int*)(ws + b->layout.res_off);
    p.step = n_sweeps;
    cudaError_t e = cudaFuncSetAttribute(batch_resident_kernel<N, ST>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)b->resident_smem);
    if (e != cudaSuccess) return cuda_status(e, "batch resident shared memory");
    batch_resident_kernel<N, ST><<<b->resident_blocks, 512, b->resident_smem, st>>>(p);
    int rc = cuda_status(cudaGetLastError(), "batch resident launch");
    if (rc != SCK_OK) return rc;
    batch_advance_kernel<<<(b->n + 127) / 128, 128, 0, st>>>(p.sys, b->n, 1, n_sweeps);
    rc = cuda_status(cudaGetLastError(), "batch advance");
    if (rc != SCK_OK) return rc;
  }
  for (int sw = 0; sw < n_sweeps; ++sw) {
    bool any = false;
    for (int k = 0; k < b->max_classes; ++k) {
      if (b->step_blocks[k] == 0) continue;
      any = true;
      p.offsets = (const int*)(ws + b->layout.step_off) + (size_t)k * (b->n + 1);
      p.step = k;
      batch_step_kernel<N, ST><<<b->step_blocks[k], 256, 0, st>>>(p);
      const int rc = cuda_status(cudaGetLastError(), "batch step launch");
      if (rc != SCK_OK) return rc;
    }
    if (!any) break;
    batch_advance_kernel<<<(b->n + 127) / 128, 128, 0, st>>>(p.sys, b->n, 0, 1);
    const int rc = cuda_status(cudaGetLastError(), "batch advance");
    if (rc != SCK_OK) return rc;
  }
  return SCK_OK;
}

int batch_sweep_dispatch(const sck_batch* b, const unsigned char* ws, int n_sweeps, cudaStream_t st) {
  if (b->mode == SCK_MODE_INT8) return run_batch<1, int8_t>(b, ws, n_sweeps, st);
  switch (b->ncomp) {
    case 1: return run_batch<1, float>(b, ws, n_sweeps, st);
    case 2: return run_batch<2, float>(b, ws, n_sweeps, st);
    default: return run_batch<3, float>(b, ws, n_sweeps, st);
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
  b->bytes = align_up(b->layout.res_off + sizeof(int) * (size_t)(n_plans + 1), 256);
  b->staging.assign(b->bytes, 0);
  b->step_blocks.assign(b->max_classes, 0);
  b->resident_blocks = 0;
  b->bound = false;
  *out = b;
  return SCK_OK;
}

int sck_batch_destroy(sck_batch* batch) {
  delete batch;
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
    d.chunks = (int)((per + 255) / 256);
    res_off[s] = (int)res_total;
    if (d.resident) res_total += plan->Bp;
    for (int k = 0; k < b->max_classes; ++k) {
      step_off[k * (b->n + 1) + s] = (int)step_total[k];
      if (!d.resident && k < d.n_classes) step_total[k] += (long long)d.chunks * plan->Bp;
    }
  }
  res_off[b->n] = (int)res_total;
  for (int k = 0; k < b->max_classes; ++k) {
    if (step_total[k] >= (1ll << 31)) return batch_fail(SCK_ERR_UNSUPPORTED, "batch too large for one launch");
    step_off[k * (b->n + 1) + b->n] = (int)step_total[k];
    b->step_blocks[k] = (int)step_total[k];
  }
  b->resident_blocks = (int)res_total;
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
  return batch_sweep_dispatch(b, (const unsigned char*)workspace, n_sweeps, (cudaStream_t)stream);
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
