// The C ABI of libsckb200.so (include/sck.h): plan validation, derived launch geometry and the entry points.
#include <string.h>

#include <numeric>
#include <string>

#include "internal.h"
#include "spec.cuh"

namespace sck {

static thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }

int cuda_status(cudaError_t e, const char* where) {
  if (e == cudaSuccess) return SCK_OK;
  set_error(std::string(where) + ": " + cudaGetErrorString(e));
  return SCK_ERR_CUDA;
}

static int fail(int code, const std::string& msg) {
  set_error(msg);
  return code;
}

static int x_period(const Colouring& c) {
  int P = 1;
  for (int r = 0; r < c.r; ++r) {
    const int mr = c.m[r];
    int k = c.K[r][0] % mr;
    if (k == 0) k = mr;
    P = std::lcm(P, mr / std::gcd(k, mr));
  }
  return P;
}

static Common make_common(const sck_plan* plan, const sck_buffers* buf, const void* src) {
  Common c;
  memset(&c, 0, sizeof(c));
  c.g = plan->geom;
  c.col = plan->col;
  c.B = plan->Bp;
  c.W = plan->W;
  c.P = plan->P;
  c.bx = plan->bx;
  c.rows = plan->geom.L3 * plan->geom.L2;
  for (int k = 0; k < 3; ++k) {
    c.h[k] = plan->desc.h[k];
    c.hnz[k] = (k < plan->geom.n && plan->desc.h[k] != 0.0f) ? 1 : 0;
  }
  c.k2 = plan->desc.k2;
  c.keys = plan->keys;
  c.lut_rep_stride = plan->geom.b * plan->keys;
  c.Z1 = plan->Z1;
  c.NT = 2 * plan->Z1 * plan->Z1;
  c.field = plan->field;
  c.src = src;
  c.dst = buf->spins;
  c.mask = buf->mask;
  c.k1 = buf->k1;
  c.beta = buf->beta;
  c.table = buf->table;
  c.state = buf->state;
  c.giveup = plan->giveup_dev;
  c.wait_limit = plan->wait_limit;
  c.fd_bx = make_fastdiv((uint32_t)c.bx);
  c.fd_L1 = make_fastdiv((uint32_t)c.g.L1);
  c.fd_L2 = make_fastdiv((uint32_t)c.g.L2);
  for (int r = 0; r < SCK_MAX_FACTORS; ++r) c.fd_m[r] = make_fastdiv((uint32_t)c.col.m[r]);
  return c;
}

Common make_common_public(const sck_plan* plan, const sck_buffers* buf) { return make_common(plan, buf, buf->spins); }

static bool is_bitwise(int mode) { return mode == SCK_MODE_BITWISE || mode == SCK_MODE_BITWISE_INDEP; }

static bool is_aligned16(const void* p) { return ((uintptr_t)p & 15u) == 0; }

constexpr long long kResidentDefault = 200ll << 10;
constexpr long long kResidentMax = 220ll << 10;

// Whole sweeps in shared memory: int8 / float32 storage and a replica within the resident limit.
static bool use_resident(const sck_plan* p) {
  if (p->mode != SCK_MODE_INT8 && p->mode != SCK_MODE_F32) return false;
  return p->resident_limit > 0 && (long long)resident_bytes(p) <= p->resident_limit;
}

// Replicas per group of the L2 pipeline, or 0 when the sweep runs class by class over all replicas: the
// specialised kernels only, a state larger than the budget, at least as many groups as classes.
static int pipeline_group(const sck_plan* p) {
  if (!p->spec || p->l2_budget <= 0 || p->mode == SCK_MODE_QUAD) return 0;
  const int C = p->desc.n_classes;
  if (C < 2 || C > 8) return 0;
  const long long per_rep = (long long)p->geom.nsite * p->geom.n * (p->mode == SCK_MODE_INT8 ? 1 : 4);
  if (per_rep * p->Bp <= p->l2_budget) return 0;
  long long group = p->l2_budget / ((long long)C * per_rep);
  if (p->geom.n > 1) group &= ~1ll;
  if (group < 1) return 0;
  if ((p->Bp + group - 1) / group < C) return 0;
  return (int)group;
}

static int check_buffers(const sck_plan* plan, const sck_buffers* buf, bool need_spins) {
  if (plan == nullptr || buf == nullptr) return fail(SCK_ERR_INVALID, "null plan or buffers");
  if (need_spins && buf->spins == nullptr) return fail(SCK_ERR_INVALID, "null spins");
  if (buf->state == nullptr) return fail(SCK_ERR_INVALID, "null state");
  if (plan->geom.has_mask && buf->mask == nullptr) return fail(SCK_ERR_INVALID, "the system has a mask: pass it");
  if (plan->geom.has_cubic && buf->k1 == nullptr) return fail(SCK_ERR_INVALID, "the system has cubic anisotropy: pass k1");
  if ((plan->ising_lut || is_bitwise(plan->mode)) && buf->table == nullptr)
    return fail(SCK_ERR_INVALID, "this mode needs its acceptance table");
  if (!plan->ising_lut && !is_bitwise(plan->mode) && buf->beta == nullptr)
    return fail(SCK_ERR_INVALID, "null beta");
  if (plan->mode == SCK_MODE_QUAD && !(is_aligned16(buf->spins) && is_aligned16(buf->beta)))
    return fail(SCK_ERR_INVALID, "interleaved storage needs 16-byte aligned spins and beta");
  return SCK_OK;
}

}  // namespace sck

using namespace sck;

extern "C" {

int sck_abi_version(void) { return SCK_ABI_VERSION; }

const char* sck_last_error(void) { return g_last_error.c_str(); }

int sck_struct_sizes(int64_t* system_desc, int64_t* sublattice, int64_t* bond, int64_t* buffers) {
  if (system_desc) *system_desc = (int64_t)sizeof(sck_system_desc);
  if (sublattice) *sublattice = (int64_t)sizeof(sck_sublattice);
  if (bond) *bond = (int64_t)sizeof(sck_bond);
  if (buffers) *buffers = (int64_t)sizeof(sck_buffers);
  return SCK_OK;
}

int sck_plan_create(const sck_system_desc* d, int32_t batch, int32_t mode, sck_plan** out) {
  if (d == nullptr || out == nullptr) return fail(SCK_ERR_INVALID, "null descriptor or output");
  *out = nullptr;
  if (d->abi_version != SCK_ABI_VERSION) return fail(SCK_ERR_INVALID, "descriptor ABI version mismatch");
  if (d->n < 1 || d->n > 3) return fail(SCK_ERR_INVALID, "n must be 1, 2 or 3");
  if (d->dim != 2 && d->dim != 3) return fail(SCK_ERR_INVALID, "dim must be 2 or 3");
  if (d->b < 1 || d->b > SCK_MAX_BASIS) return fail(SCK_ERR_INVALID, "basis size out of range");
  for (int k = 0; k < 3; ++k)
    if (d->L[k] < 1) return fail(SCK_ERR_INVALID, "box extents must be positive");
  if (d->dim == 2 && d->L[2] != 1) return fail(SCK_ERR_INVALID, "2D systems have L3 = 1");
  if (d->acceptance != SCK_METROPOLIS && d->acceptance != SCK_BARKER)
    return fail(SCK_ERR_INVALID, "acceptance must be Metropolis or Barker");
  if (d->has_cubic && d->n != 3) return fail(SCK_ERR_INVALID, "cubic anisotropy needs n = 3");
  if (batch < 1) return fail(SCK_ERR_INVALID, "batch must be positive");
  if (d->n_factors < 0 || d->n_factors > SCK_MAX_FACTORS) return fail(SCK_ERR_INVALID, "colouring factors out of range");
  for (int r = 0; r < d->n_factors; ++r)
    if (d->m[r] < 1) return fail(SCK_ERR_INVALID, "colouring group orders must be positive");
  if (d->n_classes < 1 || d->n_classes > 128) return fail(SCK_ERR_INVALID, "class list out of range");
  if (mode < SCK_MODE_INT8 || mode > SCK_MODE_QUAD) return fail(SCK_ERR_INVALID, "unknown mode");
  if (mode != SCK_MODE_F32 && mode != SCK_MODE_QUAD && d->n != 1)
    return fail(SCK_ERR_UNSUPPORTED, "int8, packed and bitwise storage are for Ising (n = 1) only");
  if (mode == SCK_MODE_QUAD && d->n == 1)
    return fail(SCK_ERR_UNSUPPORTED, "interleaved storage is for vector models (n = 2 or 3)");

  sck_plan* p = new sck_plan();
  memset(p, 0, sizeof(*p));
  p->desc = *d;
  p->mode = mode;
  p->batch = batch;
  Geometry& g = p->geom;
  g.n = d->n;
  g.b = d->b;
  g.dim = d->dim;
  g.L1 = d->L[0];
  g.L2 = d->L[1];
  g.L3 = d->L[2];
  for (int k = 0; k < 3; ++k) g.per[k] = d->periodic[k] ? 1 : 0;
  g.plane = g.L3 * g.L2 * g.L1;
  g.nsite = g.b * g.plane;
  g.has_mask = d->has_mask ? 1 : 0;
  g.has_cubic = d->has_cubic ? 1 : 0;
  g.acceptance = d->acceptance;
  Colouring& col = p->col;
  col.r = d->n_factors;
  for (int r = 0; r < SCK_MAX_FACTORS; ++r) {
    col.m[r] = d->m[r] > 0 ? d->m[r] : 1;
    for (int k = 0; k < 3; ++k) col.K[r][k] = d->K[r][k];
    for (int a = 0; a < SCK_MAX_BASIS; ++a) col.o[a][r] = d->o[a][r];
  }
  for (int r = 0; r < col.r; ++r)
    for (int k = 0; k < 3; ++k)
      if (col.K[r][k] < 0) {
        delete p;
        return fail(SCK_ERR_INVALID, "colouring coefficients must be non-negative group elements");
      }
  for (int i = 0; i < d->n_classes; ++i) {
    const int c = d->classes[i][0], a = d->classes[i][1];
    int nc = 1;
    for (int r = 0; r < col.r; ++r) nc *= col.m[r];
    if (c < 0 || c >= nc || a < 0 || a >= g.b) {
      delete p;
      return fail(SCK_ERR_INVALID, "class out of range");
    }
  }
  const bool packed = mode == SCK_MODE_PACKED || is_bitwise(mode);
  p->W = (batch + 31) / 32;
  p->Bp = packed ? p->W * 32 : (mode == SCK_MODE_QUAD ? 4 * ((batch + 3) / 4) : batch);
  p->rows_storage = packed ? p->W : (mode == SCK_MODE_QUAD ? p->Bp / 4 : batch);
  if ((long long)p->Bp * (long long)g.nsite >= 2147483647LL) {
    delete p;
    return fail(SCK_ERR_COUNTER, "replica batch too large for the int32 Philox counter");
  }
  p->P = x_period(col);
  p->bx = (g.L1 + p->P - 1) / p->P;
  p->ising_lut = (d->n == 1 && !is_bitwise(mode)) ? 1 : 0;

  // sublattice descriptors
  int keys_max = 1;
  int Zmax = 0;
  float Jbw = 0.0f;
  bool Jbw_set = false;
  for (int a = 0; a < g.b; ++a) {
    const sck_sublattice& s = d->sub[a];
    SubDev& sd = p->sub[a];
    SubObs& so = p->obs[a];
    if (s.n_bonds < 0 || s.n_bonds > SCK_MAX_BONDS || s.n_groups < 0 || s.n_groups > SCK_MAX_GROUPS ||
        s.n_extra < 0 || s.n_extra > SCK_MAX_EXTRA) {
      delete p;
      return fail(SCK_ERR_INVALID, "sublattice bond, group or extra count out of range");
    }
    sd.n_bonds = s.n_bonds;
    sd.n_groups = s.n_groups;
    sd.n_extra = s.n_extra;
    so.n_bonds = s.n_bonds;
    int prev = 0;
    for (int gi = 0; gi < s.n_groups; ++gi) {
      if (s.group_end[gi] < prev || s.group_end[gi] > s.n_bonds) {
        delete p;
        return fail(SCK_ERR_INVALID, "group ends must be non-decreasing and within the bond list");
      }
      sd.group_end[gi] = s.group_end[gi];
      sd.group_z[gi] = s.group_end[gi] - prev;
      sd.J[gi] = s.group_J[gi];
      sd.apply[gi] = s.group_apply[gi] ? 1 : 0;
      prev = s.group_end[gi];
    }
    if (s.n_groups > 0 && prev != s.n_bonds) {
      delete p;
      return fail(SCK_ERR_INVALID, "the last group must end at the last bond");
    }
    for (int e = 0; e < s.n_extra; ++e) {
      int nz = 0;
      for (int k = 0; k < 3; ++k)
        for (int l = 0; l < 3; ++l) {
          sd.E[e][3 * k + l] = s.extra[e][3 * k + l];
          so.E[e][3 * k + l] = s.extra64[e][3 * k + l];
          if (k < d->n && l < d->n && s.extra[e][3 * k + l] != 0.0f) nz |= 1 << (3 * k + l);
        }
      sd.Enz[e] = nz;
    }
    for (int bi = 0; bi < s.n_bonds; ++bi) {
      const sck_bond& bd = s.bonds[bi];
      if (bd.alpha2 < 0 || bd.alpha2 >= g.b || bd.extra < -1 || bd.extra >= s.n_extra) {
        delete p;
        return fail(SCK_ERR_INVALID, "bond target sublattice or extra slot out of range");
      }
      for (int k = 0; k < 3; ++k)
        if (bd.d[k] < -64 || bd.d[k] > 64) {
          delete p;
          return fail(SCK_ERR_INVALID, "bond offset out of range");
        }
      if (d->dim == 2 && bd.d[2] != 0) {
        delete p;
        return fail(SCK_ERR_INVALID, "2D bonds have dz = 0");
      }
      BondDev b8;
      memset(&b8, 0, sizeof(b8));
      b8.a2 = (int8_t)bd.alpha2;
      b8.dx = (int8_t)bd.d[0];
      b8.dy = (int8_t)bd.d[1];
      b8.dz = (int8_t)bd.d[2];
      b8.extra = (int8_t)bd.extra;
      sd.bonds[bi] = b8;
      so.J[bi] = bd.J64;
    }
    // Ising key: own spin (2) x applied groups (2 z_g + 1) x extra bonds with a non-zero coupling (3)
    long long stride = 2;
    for (int gi = 0; gi < s.n_groups; ++gi) {
      if (sd.apply[gi]) {
        sd.key_stride[gi] = (int)stride;
        stride *= 2 * sd.group_z[gi] + 1;
      } else {
        sd.key_stride[gi] = 0;
      }
    }
    for (int e = 0; e < s.n_extra; ++e) {
      if (d->n == 1 && s.extra[e][0] != 0.0f) {
        sd.extra_stride[e] = (int)stride;
        stride *= 3;
      } else {
        sd.extra_stride[e] = 0;
      }
      if (stride > (1LL << 22)) break;
    }
    if (p->ising_lut && stride > (1LL << 22)) {
      delete p;
      return fail(SCK_ERR_UNSUPPORTED, "Ising acceptance table exceeds 2^22 keys per sublattice");
    }
    if (stride > keys_max) keys_max = (int)stride;
    int zb = 0;
    for (int gi = 0; gi < s.n_groups; ++gi) {
      if (!sd.apply[gi]) continue;
      zb += sd.group_z[gi];
      if (!Jbw_set) {
        Jbw = sd.J[gi];
        Jbw_set = true;
      } else if (sd.J[gi] != Jbw && is_bitwise(mode)) {
        delete p;
        return fail(SCK_ERR_UNSUPPORTED, "bitwise multi-spin coding needs one uniform coupling J on every bond");
      }
    }
    if (is_bitwise(mode)) {
      for (int gi = 0; gi < s.n_groups; ++gi)
        if (!sd.apply[gi]) {
          delete p;
          return fail(SCK_ERR_UNSUPPORTED, "bitwise multi-spin coding needs isotropic exchange only");
        }
    }
    if (zb > Zmax) Zmax = zb;
  }
  if (is_bitwise(mode)) {
    for (int a = 0; a < g.b; ++a)
      if (d->sub[a].n_extra > 0) {
        delete p;
        return fail(SCK_ERR_UNSUPPORTED,
                    "bitwise multi-spin coding needs isotropic exchange only (no extra bond matrices)");
      }
    if (d->has_cubic) {
      delete p;
      return fail(SCK_ERR_UNSUPPORTED, "bitwise multi-spin coding does not support anisotropy");
    }
    if (Zmax > 64) {
      delete p;
      return fail(SCK_ERR_UNSUPPORTED, "bitwise kernels support coordination up to 64");
    }
  }
  p->keys = keys_max;
  p->Z = Zmax;
  p->Z1 = Zmax + 1;
  int np = 0;
  while ((1 << np) <= Zmax) ++np;
  p->NP = np < 1 ? 1 : np;
  p->field = (d->n == 1 && d->h64[0] != 0.0) ? 1 : 0;
  p->spec = find_spec(p);
  if (mode == SCK_MODE_QUAD) {
    std::string why;
    if (!quad_ok(p, &why)) {
      delete p;
      return fail(SCK_ERR_UNSUPPORTED, why);
    }
  }
  p->kernel_kind = 1;
  p->wait_limit = 1u << 20;
  p->quad_cpt = 4;
  p->l2_budget = 0;
  p->resident_limit = kResidentDefault;
  *out = p;
  return SCK_OK;
}

// The plan's give-up flag: 4 bytes of mapped, portable pinned host memory that kernels with bounded waits (the
// tile kernels' bulk-copy waits, the group pipelines' completion-counter waits) raise when a wait gives up.
// Allocated once, on the first choice of such a path, never inside a sweep.
static int ensure_giveup_flag(sck_plan* plan) {
  if (plan->giveup_host != nullptr) return SCK_OK;
  int rc = cuda_status(cudaHostAlloc((void**)&plan->giveup_host, sizeof(int),
                                     cudaHostAllocMapped | cudaHostAllocPortable), "give-up flag");
  if (rc != SCK_OK) {
    plan->giveup_host = nullptr;
    return rc;
  }
  *plan->giveup_host = 0;
  rc = cuda_status(cudaHostGetDevicePointer((void**)&plan->giveup_dev, plan->giveup_host, 0), "give-up flag");
  if (rc != SCK_OK) {
    cudaFreeHost(plan->giveup_host);
    plan->giveup_host = nullptr;
    plan->giveup_dev = nullptr;
  }
  return rc;
}

int sck_plan_tune(sck_plan* plan, int32_t specialised, int64_t l2_budget_bytes, int64_t resident_limit_bytes) {
  if (plan == nullptr || l2_budget_bytes < 0 || resident_limit_bytes < 0)
    return fail(SCK_ERR_INVALID, "null plan or negative budget");
  if (resident_limit_bytes > kResidentMax) return fail(SCK_ERR_INVALID, "resident limit above 220 KiB of shared memory");
  plan->spec = (specialised || plan->mode == SCK_MODE_QUAD) ? find_spec(plan) : 0;   // interleaved: always
  plan->kernel_kind = specialised >= 3 ? 3 : (specialised >= 2 ? 2 : 1);
  plan->l2_budget = l2_budget_bytes;
  plan->resident_limit = resident_limit_bytes;
  if (plan->kernel_kind == 3 || pipeline_group(plan) > 0) {
    const int rc = ensure_giveup_flag(plan);
    if (rc != SCK_OK) return rc;
  }
  // the group pipeline's counters live on the current device, allocated here (never inside a sweep)
  const int group = pipeline_group(plan);
  if (group > 0 && !use_resident(plan)) {
    const size_t need = stream_counter_bytes(plan, group);
    int dev = 0;
    int rc = cuda_status(cudaGetDevice(&dev), "group pipeline counters");
    if (rc != SCK_OK) return rc;
    if (plan->pipe_counters == nullptr || plan->pipe_bytes < need || plan->pipe_device != dev) {
      if (plan->pipe_counters != nullptr) cudaFree(plan->pipe_counters);
      plan->pipe_counters = nullptr;
      plan->pipe_bytes = 0;
      rc = cuda_status(cudaMalloc(&plan->pipe_counters, need), "group pipeline counters");
      if (rc != SCK_OK) {
        plan->pipe_counters = nullptr;
        return rc;
      }
      plan->pipe_bytes = need;
      plan->pipe_device = dev;
    }
  }
  return SCK_OK;
}

int sck_plan_path(const sck_plan* plan, int32_t* specialised, int64_t* l2_budget_bytes, int32_t* group,
                  int32_t* resident) {
  if (plan == nullptr) return fail(SCK_ERR_INVALID, "null plan");
  if (specialised) {
    int kind = pipeline_group(plan) > 0 ? 1 : (tile_kernel_ok(plan) ? 3 : (seg_kernel_ok(plan) ? 2 : 1));
    if (plan->mode == SCK_MODE_QUAD) kind = 4;
    *specialised = plan->spec ? kind * 100 + plan->spec : 0;
  }
  if (l2_budget_bytes) *l2_budget_bytes = plan->l2_budget;
  if (group) *group = plan->mode == SCK_MODE_QUAD ? 4 * plan->quad_group : pipeline_group(plan);
  if (resident) *resident = use_resident(plan) ? 1 : 0;
  return SCK_OK;
}

int sck_plan_pipeline(sck_plan* plan, int32_t group_replicas, int32_t skew) {
  if (plan == nullptr) return fail(SCK_ERR_INVALID, "null plan");
  if (plan->mode != SCK_MODE_QUAD)
    return fail(SCK_ERR_UNSUPPORTED, "the class-skewed pipeline runs interleaved storage (SCK_MODE_QUAD); "
                                     "other plans take an L2 budget in sck_plan_tune");
  if (group_replicas == 0) {
    plan->quad_group = 0;
    return SCK_OK;
  }
  const int C = plan->desc.n_classes;
  if (group_replicas < 0 || group_replicas % 4 != 0)
    return fail(SCK_ERR_INVALID, "pipeline groups hold whole quads: a positive multiple of 4 replicas");
  if (skew < 1 || skew > C || C % skew != 0 || C > 8)
    return fail(SCK_ERR_INVALID, "the skew must divide the class count (" + std::to_string(C) + ", at most 8)");
  const int Q = plan->Bp / 4;
  const int group = group_replicas / 4 < Q ? group_replicas / 4 : Q;
  const int ngroups = (Q + group - 1) / group;
  if ((long long)skew * ngroups <= C - 1)
    return fail(SCK_ERR_INVALID, "too few replica groups for this skew: a group's next sweep would follow its own "
                                 "last class too closely (need skew x groups >= classes)");
  int dev = 0;
  int rc = cuda_status(cudaGetDevice(&dev), "pipeline set-up");
  if (rc != SCK_OK) return rc;
  plan->quad_group = group;
  const size_t need = quad_pipe_counter_bytes(plan);
  if (plan->pipe_counters == nullptr || plan->pipe_bytes < need || plan->pipe_device != dev) {
    if (plan->pipe_counters != nullptr) cudaFree(plan->pipe_counters);
    plan->pipe_counters = nullptr;
    plan->pipe_bytes = 0;
    rc = cuda_status(cudaMalloc(&plan->pipe_counters, need), "pipeline counters");
    if (rc != SCK_OK) {
      plan->quad_group = 0;
      return rc;
    }
    plan->pipe_bytes = need;
    plan->pipe_device = dev;
  }
  rc = ensure_giveup_flag(plan);
  if (rc != SCK_OK) {
    plan->quad_group = 0;
    return rc;
  }
  plan->quad_skew = skew;
  return SCK_OK;
}

int sck_plan_pipeline_chunks(sck_plan* plan, int32_t site_blocks) {
  if (plan == nullptr || site_blocks < 1 || site_blocks > 64)
    return fail(SCK_ERR_INVALID, "site blocks per pipeline ticket must be 1 .. 64");
  plan->quad_cpt = site_blocks;
  return SCK_OK;
}

int sck_plan_set_wait_limit(sck_plan* plan, int64_t polls) {
  if (plan == nullptr || polls < 0 || polls > 0xFFFFFFFFll) return fail(SCK_ERR_INVALID, "polls must be 0 .. 2^32-1");
  plan->wait_limit = (unsigned)polls;
  return SCK_OK;
}

int sck_plan_wait_status(sck_plan* plan, void* stream) {
  if (plan == nullptr) return fail(SCK_ERR_INVALID, "null plan");
  if (plan->giveup_host == nullptr) return SCK_OK;
  const int rc = cuda_status(cudaStreamSynchronize((cudaStream_t)stream), "wait status");
  if (rc != SCK_OK) return rc;
  if (*(volatile int*)plan->giveup_host) {
    *(volatile int*)plan->giveup_host = 0;
    return fail(SCK_ERR_TIMEOUT, "a bounded wait of this plan's kernels gave up: the affected sites were left "
                                 "unchanged");
  }
  return SCK_OK;
}

int sck_plan_destroy(sck_plan* plan) {
  if (plan != nullptr && plan->giveup_host != nullptr) cudaFreeHost(plan->giveup_host);
  if (plan != nullptr && plan->pipe_counters != nullptr) cudaFree(plan->pipe_counters);
  delete plan;
  return SCK_OK;
}

int sck_plan_table_size(const sck_plan* p, int64_t* elements, int32_t* element_bytes, int32_t* keys) {
  if (p == nullptr) return fail(SCK_ERR_INVALID, "null plan");
  int64_t n = 0;
  int32_t eb = 4;
  if (p->ising_lut) {
    n = (int64_t)p->Bp * p->geom.b * p->keys;
  } else if (p->mode == SCK_MODE_BITWISE) {
    n = (int64_t)p->W * 2 * p->Z1 * p->Z1;
  } else if (p->mode == SCK_MODE_BITWISE_INDEP) {
    n = (int64_t)p->W * 2 * p->Z1 * p->Z1;
    eb = 8;
  }
  if (elements) *elements = n;
  if (element_bytes) *element_bytes = eb;
  if (keys) *keys = p->keys;
  return SCK_OK;
}

int sck_plan_shape(const sck_plan* p, int32_t* computed, int32_t* rows) {
  if (p == nullptr) return fail(SCK_ERR_INVALID, "null plan");
  if (computed) *computed = p->Bp;
  if (rows) *rows = p->rows_storage;
  return SCK_OK;
}

static int class_launch(const sck_plan* plan, const sck_buffers* buf, const void* src, int colour, int alpha,
                        cudaStream_t s) {
  if (plan->mode == SCK_MODE_QUAD) {
    if (src != buf->spins || colour < 0)
      return fail(SCK_ERR_UNSUPPORTED, "interleaved storage updates in place (src = spins, no synchronous control)");
    return launch_quad_class(plan, buf, colour, alpha, s);
  }
  Common c = make_common(plan, buf, src);
  if (is_bitwise(plan->mode)) return launch_bitwise_class(plan, c, colour, alpha, s);
  return launch_class(plan, c, colour, alpha, s);
}

int sck_class_update(const sck_plan* plan, const sck_buffers* buf, const void* src, int32_t colour, int32_t alpha,
                     int32_t sync, void* stream) {
  int rc = check_buffers(plan, buf, true);
  if (rc != SCK_OK) return rc;
  if (alpha < 0 || alpha >= plan->geom.b) return fail(SCK_ERR_INVALID, "sublattice out of range");
  if (colour < 0 && !sync) return fail(SCK_ERR_INVALID, "colour < 0 is the synchronous control: pass sync = 1");
  return class_launch(plan, buf, src ? src : buf->spins, sync ? -1 : colour, alpha, (cudaStream_t)stream);
}

int sck_sweep(const sck_plan* plan, const sck_buffers* buf, int32_t n_sweeps, void* stream) {
  int rc = check_buffers(plan, buf, true);
  if (rc != SCK_OK) return rc;
  if (n_sweeps < 0) return fail(SCK_ERR_INVALID, "negative sweep count");
  cudaStream_t s = (cudaStream_t)stream;
  if (n_sweeps == 0) return SCK_OK;
  if (plan->giveup_host != nullptr && *(volatile int*)plan->giveup_host)
    return fail(SCK_ERR_TIMEOUT, "an earlier bounded wait of this plan gave up (read sck_plan_wait_status)");
  if (plan->mode == SCK_MODE_QUAD) {
    if (plan->quad_group > 0) {
      int dev = -1;
      rc = cuda_status(cudaGetDevice(&dev), "interleaved pipeline");
      if (rc != SCK_OK) return rc;
      if (plan->pipe_device != dev)
        return fail(SCK_ERR_INVALID, "the pipeline's counters belong to another device: call sck_plan_pipeline here");
      rc = launch_quad_pipeline(plan, buf, n_sweeps, s, nullptr);
      if (rc != SCK_OK) return rc;
      return launch_advance(buf->state, n_sweeps, s);
    }
    for (int k = 0; k < n_sweeps; ++k) {
      for (int i = 0; i < plan->desc.n_classes; ++i) {
        rc = launch_quad_class(plan, buf, plan->desc.classes[i][0], plan->desc.classes[i][1], s);
        if (rc != SCK_OK) return rc;
      }
      rc = launch_advance(buf->state, 1, s);
      if (rc != SCK_OK) return rc;
    }
    return SCK_OK;
  }
  if (use_resident(plan)) {
    const Common c = make_common(plan, buf, buf->spins);
    rc = launch_resident(plan, c, n_sweeps, s);
    if (rc != SCK_OK) return rc;
    return launch_advance(buf->state, n_sweeps, s);
  }
  if (plan->spec) {
    const Common c = make_common(plan, buf, buf->spins);
    const int group = pipeline_group(plan);
    if (group > 0) {
      int dev = -1;
      rc = cuda_status(cudaGetDevice(&dev), "group pipeline");
      if (rc != SCK_OK) return rc;
      if (plan->pipe_counters == nullptr || plan->pipe_device != dev || plan->pipe_bytes < stream_counter_bytes(plan, group))
        return fail(SCK_ERR_INVALID, "the group pipeline's counters belong to another device: call sck_plan_tune on this one");
      rc = launch_spec_pipeline(plan, c, n_sweeps, group, plan->pipe_counters, s);
      if (rc != SCK_OK) return rc;
      return launch_advance(buf->state, n_sweeps, s);
    }
    for (int k = 0; k < n_sweeps; ++k) {
      for (int i = 0; i < plan->desc.n_classes; ++i) {
        rc = launch_spec_class(plan, c, plan->desc.classes[i][0], plan->desc.classes[i][1], s);
        if (rc != SCK_OK) return rc;
      }
      rc = launch_advance(buf->state, 1, s);
      if (rc != SCK_OK) return rc;
    }
    return SCK_OK;
  }
  for (int k = 0; k < n_sweeps; ++k) {
    for (int i = 0; i < plan->desc.n_classes; ++i) {
      rc = class_launch(plan, buf, buf->spins, plan->desc.classes[i][0], plan->desc.classes[i][1], s);
      if (rc != SCK_OK) return rc;
    }
    rc = launch_advance(buf->state, 1, s);
    if (rc != SCK_OK) return rc;
  }
  return SCK_OK;
}

int sck_sync_sweep(const sck_plan* plan, const sck_buffers* buf, void* scratch, int32_t n_sweeps, void* stream) {
  int rc = check_buffers(plan, buf, true);
  if (rc != SCK_OK) return rc;
  if (scratch == nullptr) return fail(SCK_ERR_INVALID, "the synchronous control needs a scratch copy of the spins");
  if (plan->mode == SCK_MODE_QUAD)
    return fail(SCK_ERR_UNSUPPORTED, "the synchronous control reads S: unpack interleaved storage first");
  cudaStream_t s = (cudaStream_t)stream;
  size_t elem = plan->mode == SCK_MODE_INT8 ? 1 : 4;
  size_t bytes = (size_t)plan->rows_storage * (plan->mode == SCK_MODE_F32 ? plan->geom.n : 1) * plan->geom.nsite * elem;
  for (int k = 0; k < n_sweeps; ++k) {
    rc = cuda_status(cudaMemcpyAsync(scratch, buf->spins, bytes, cudaMemcpyDeviceToDevice, s), "sync copy");
    if (rc != SCK_OK) return rc;
    sck_buffers b2 = *buf;
    b2.spins = scratch;
    for (int a = 0; a < plan->geom.b; ++a) {
      rc = class_launch(plan, &b2, buf->spins, -1, a, s);
      if (rc != SCK_OK) return rc;
    }
    rc = cuda_status(cudaMemcpyAsync(buf->spins, scratch, bytes, cudaMemcpyDeviceToDevice, s), "sync copy back");
    if (rc != SCK_OK) return rc;
    rc = launch_advance(buf->state, 1, s);
    if (rc != SCK_OK) return rc;
  }
  return SCK_OK;
}

int sck_reference_sweep(const sck_plan* plan, const sck_buffers* buf, int32_t n_sweeps, void* stream) {
  int rc = check_buffers(plan, buf, true);
  if (rc != SCK_OK) return rc;
  if (plan->mode == SCK_MODE_QUAD)
    return fail(SCK_ERR_UNSUPPORTED, "the sequential reference reads S: unpack interleaved storage first");
  cudaStream_t s = (cudaStream_t)stream;
  for (int k = 0; k < n_sweeps; ++k) {
    Common c = make_common(plan, buf, buf->spins);
    rc = is_bitwise(plan->mode) ? launch_bitwise_sequential(plan, c, s) : launch_sequential(plan, c, s);
    if (rc != SCK_OK) return rc;
    rc = launch_advance(buf->state, 1, s);
    if (rc != SCK_OK) return rc;
  }
  return SCK_OK;
}

int sck_observables_workspace_size(const sck_plan* plan, int32_t batch, int64_t* bytes) {
  if (plan == nullptr || bytes == nullptr || batch < 1) return fail(SCK_ERR_INVALID, "null plan or output, or batch < 1");
  *bytes = (int64_t)batch * obs_blocks_per_rep(plan, batch) * OBS_VALUES * (int64_t)sizeof(double);
  return SCK_OK;
}

}  // extern "C"

namespace sck {
// The checks every observables entry point shares: a storage the plan can hold, and a batch within the plan's
// (the spins buffer behind a plan holds at most that many replicas, so larger requests would read past it).
int check_observables_request(const sck_plan* plan, int storage, int batch) {
  if (batch < 1 || batch > plan->batch)
    return fail(SCK_ERR_INVALID, "batch must be within 1 .. the plan's batch (" + std::to_string(plan->batch) + ")");
  if (batch > 65535) return fail(SCK_ERR_INVALID, "observables: batch above 65535");
  if (storage != SCK_MODE_INT8 && storage != SCK_MODE_F32 && storage != SCK_MODE_PACKED && storage != SCK_MODE_QUAD)
    return fail(SCK_ERR_INVALID, "observables read int8, float32, packed or interleaved storage");
  if (storage == SCK_MODE_QUAD && plan->mode != SCK_MODE_QUAD)
    return fail(SCK_ERR_INVALID, "interleaved storage needs a plan of SCK_MODE_QUAD");
  if (storage != SCK_MODE_F32 && storage != SCK_MODE_QUAD && plan->geom.n != 1)
    return fail(SCK_ERR_INVALID, "vector models use float32 or interleaved storage");
  if (storage == SCK_MODE_PACKED && plan->mode != SCK_MODE_PACKED && !is_bitwise(plan->mode))
    return fail(SCK_ERR_INVALID, "packed storage needs a packed or bitwise plan");
  return SCK_OK;
}
}  // namespace sck

extern "C" {

int sck_observables(const sck_plan* plan, const sck_buffers* buf, const void* spins, int32_t storage,
                    int32_t batch, double* E, double* M, void* workspace, void* stream) {
  if (plan == nullptr || buf == nullptr || spins == nullptr) return fail(SCK_ERR_INVALID, "null plan, buffers or spins");
  if (workspace == nullptr) return fail(SCK_ERR_INVALID, "null workspace (see sck_observables_workspace_size)");
  int rc = check_observables_request(plan, storage, batch);
  if (rc != SCK_OK) return rc;
  if (storage == SCK_MODE_QUAD && !is_aligned16(spins))
    return fail(SCK_ERR_INVALID, "interleaved storage needs 16-byte aligned spins");
  if (plan->geom.has_mask && buf->mask == nullptr) return fail(SCK_ERR_INVALID, "the system has a mask: pass it");
  if (plan->geom.has_cubic && buf->k1 == nullptr) return fail(SCK_ERR_INVALID, "the system has cubic anisotropy: pass k1");
  return launch_observables(plan, spins, storage, batch, buf->mask, buf->k1, E, M, workspace, (cudaStream_t)stream);
}

int sck_sweep_measure_workspace_size(const sck_plan* plan, int64_t* bytes) {
  if (plan == nullptr || bytes == nullptr) return fail(SCK_ERR_INVALID, "null plan or output");
  const int64_t obs = (int64_t)plan->batch * obs_blocks_per_rep(plan, plan->batch) * OBS_VALUES * (int64_t)sizeof(double);
  const int64_t fused = plan->mode == SCK_MODE_QUAD ? (int64_t)quad_measure_workspace(plan) : 0;
  *bytes = obs > fused ? obs : fused;
  return SCK_OK;
}

int sck_sweep_measure(const sck_plan* plan, const sck_buffers* buf, int32_t n_sweeps, double* E, double* M,
                      void* workspace, void* stream) {
  int rc = check_buffers(plan, buf, true);
  if (rc != SCK_OK) return rc;
  if (n_sweeps < 1) return fail(SCK_ERR_INVALID, "a measure step needs at least one sweep");
  if (workspace == nullptr) return fail(SCK_ERR_INVALID, "null workspace (see sck_sweep_measure_workspace_size)");
  if (plan->batch > 65535) return fail(SCK_ERR_INVALID, "measure step: batch above 65535");
  cudaStream_t s = (cudaStream_t)stream;
  if (plan->giveup_host != nullptr && *(volatile int*)plan->giveup_host)
    return fail(SCK_ERR_TIMEOUT, "an earlier bounded wait of this plan gave up (read sck_plan_wait_status)");
  if (plan->mode == SCK_MODE_QUAD && quad_measure_fused(plan)) {
    if (plan->quad_group > 0) {
      int dev = -1;
      rc = cuda_status(cudaGetDevice(&dev), "interleaved pipeline");
      if (rc != SCK_OK) return rc;
      if (plan->pipe_device != dev)
        return fail(SCK_ERR_INVALID, "the pipeline's counters belong to another device: call sck_plan_pipeline here");
      return launch_quad_pipeline_measure(plan, buf, n_sweeps, E, M, workspace, s);
    }
    if (n_sweeps > 1) {
      rc = sck_sweep(plan, buf, n_sweeps - 1, stream);
      if (rc != SCK_OK) return rc;
    }
    return launch_quad_measure_sweep(plan, buf, E, M, workspace, s);
  }
  rc = sck_sweep(plan, buf, n_sweeps, stream);
  if (rc != SCK_OK) return rc;
  const int storage = plan->mode == SCK_MODE_QUAD ? SCK_MODE_QUAD
                      : (plan->mode == SCK_MODE_BITWISE || plan->mode == SCK_MODE_BITWISE_INDEP) ? SCK_MODE_PACKED
                      : plan->mode;
  return launch_observables(plan, buf->spins, storage, plan->batch, buf->mask, buf->k1, E, M, workspace, s);
}

int sck_observables_accumulate(const sck_plan* plan, const sck_buffers* buf, const void* spins, int32_t storage,
                               int32_t batch, double n_active, const double* E_ref, double* E, double* M,
                               double* acc, double* accv, void* workspace, void* stream) {
  if (E == nullptr || M == nullptr || E_ref == nullptr || acc == nullptr || accv == nullptr)
    return fail(SCK_ERR_INVALID, "null observation or accumulator buffer");
  if (!(n_active >= 1.0)) return fail(SCK_ERR_INVALID, "n_active must be at least 1");
  int rc = sck_observables(plan, buf, spins, storage, batch, E, M, workspace, stream);
  if (rc != SCK_OK) return rc;
  return launch_observables_fold(plan, batch, E, M, n_active, E_ref, acc, accv, (cudaStream_t)stream);
}

int sck_topological_charge(const sck_plan* plan, const sck_buffers* buf, const float* spins, int32_t batch,
                           int32_t layer, double* Q, void* stream) {
  if (plan == nullptr || buf == nullptr || spins == nullptr || Q == nullptr)
    return fail(SCK_ERR_INVALID, "null plan, buffers, spins or output");
  const Geometry& g = plan->geom;
  if (g.n != 3 || plan->mode != SCK_MODE_F32) return fail(SCK_ERR_INVALID, "the charge needs float32 Heisenberg spins");
  if (g.dim != 3 && layer != 0) return fail(SCK_ERR_INVALID, "a 2D system has one layer: 0");
  if (layer < 0 || layer >= g.L3) return fail(SCK_ERR_INVALID, "layer outside 0..L3-1");
  if (batch < 1 || batch > plan->batch) return fail(SCK_ERR_INVALID, "batch outside 1..the plan's batch");
  if (g.L1 < 2 || g.L2 < 2) return fail(SCK_ERR_INVALID, "a layer needs at least 2 x 2 sites");
  if (g.has_mask && buf->mask == nullptr) return fail(SCK_ERR_INVALID, "the system has a mask: pass it");
  return launch_topological_charge(plan, spins, buf->mask, batch, layer, Q, (cudaStream_t)stream);
}

int sck_quad_pack(const sck_plan* plan, const float* spins, void* quads, void* stream) {
  if (plan == nullptr || spins == nullptr || quads == nullptr) return fail(SCK_ERR_INVALID, "null argument");
  if (plan->mode != SCK_MODE_QUAD) return fail(SCK_ERR_UNSUPPORTED, "interleaved storage needs a plan of SCK_MODE_QUAD");
  if (!is_aligned16(quads)) return fail(SCK_ERR_INVALID, "interleaved storage needs 16-byte alignment");
  return launch_quad_convert(plan, (float*)spins, (float4*)quads, 0, (cudaStream_t)stream);
}

int sck_quad_unpack(const sck_plan* plan, const void* quads, float* spins, void* stream) {
  if (plan == nullptr || spins == nullptr || quads == nullptr) return fail(SCK_ERR_INVALID, "null argument");
  if (plan->mode != SCK_MODE_QUAD) return fail(SCK_ERR_UNSUPPORTED, "interleaved storage needs a plan of SCK_MODE_QUAD");
  if (!is_aligned16(quads)) return fail(SCK_ERR_INVALID, "interleaved storage needs 16-byte alignment");
  return launch_quad_convert(plan, spins, (float4*)quads, 1, (cudaStream_t)stream);
}

int sck_pack(const sck_plan* plan, const int8_t* spins, int32_t* words, void* stream) {
  if (plan == nullptr || spins == nullptr || words == nullptr) return fail(SCK_ERR_INVALID, "null argument");
  if (plan->geom.n != 1) return fail(SCK_ERR_UNSUPPORTED, "packing is for Ising (n = 1) only");
  return launch_pack(plan, spins, words, (cudaStream_t)stream);
}

int sck_unpack(const sck_plan* plan, const int32_t* words, const int8_t* mask, int8_t* spins, void* stream) {
  if (plan == nullptr || spins == nullptr || words == nullptr) return fail(SCK_ERR_INVALID, "null argument");
  if (plan->geom.n != 1) return fail(SCK_ERR_UNSUPPORTED, "packing is for Ising (n = 1) only");
  return launch_unpack(plan, words, plan->geom.has_mask ? mask : nullptr, spins, (cudaStream_t)stream);
}

int sck_advance(int64_t* state, int32_t n, void* stream) {
  if (state == nullptr) return fail(SCK_ERR_INVALID, "null state");
  return launch_advance(state, n, (cudaStream_t)stream);
}

}  // extern "C"
