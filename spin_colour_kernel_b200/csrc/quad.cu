// Interleaved storage for vector models (SCK_MODE_QUAD): host side (plans, launches, measure steps, the L2
// pipeline's set-up), the layout conversions and the measure step's final sums. The lattice kernels live in
// quad.cuh and are instantiated per lattice in quad_<lattice>.cu.
#include <string.h>

#include <string>

#include "quad.cuh"

namespace sck {

// ------------------------------------------------------------------------------------------ layout changes
__device__ __forceinline__ void quad_coords(uint32_t e, const Geometry& g, int hp, int P, int& a, int& z, int& y,
                                            int& k, int& x) {
  // e = element index within a quad: (((a L3 + z) L2 + y) N + k) L1 + xs
  const int xs = (int)(e % (uint32_t)g.L1);
  uint32_t r = e / (uint32_t)g.L1;
  k = (int)(r % (uint32_t)g.n);
  r /= (uint32_t)g.n;
  y = (int)(r % (uint32_t)g.L2);
  r /= (uint32_t)g.L2;
  z = (int)(r % (uint32_t)g.L3);
  a = (int)(r / (uint32_t)g.L3);
  const int res = xs / hp;
  x = (xs - res * hp) * P + res;
}

// float32 S[B][N][b][L3][L2][L1] -> quads (lanes of replicas >= B are zero). Grid (element blocks, quads).
__global__ void quad_pack_kernel(const float* __restrict__ src, float4* __restrict__ dst, Geometry g, int hp, int P,
                                 int B) {
  const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t per = (uint32_t)g.n * (uint32_t)g.nsite;
  if (e >= per) return;
  const int q = blockIdx.y;
  int a, z, y, k, x;
  quad_coords(e, g, hp, P, a, z, y, k, x);
  const size_t site = (size_t)a * g.plane + ((size_t)z * g.L2 + y) * g.L1 + x;
  float v[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int rep = 4 * q + j;
    v[j] = rep < B ? src[((size_t)rep * g.n + k) * g.nsite + site] : 0.0f;
  }
  dst[(size_t)q * per + e] = make_float4(v[0], v[1], v[2], v[3]);
}

__global__ void quad_unpack_kernel(const float4* __restrict__ src, float* __restrict__ dst, Geometry g, int hp, int P,
                                   int B) {
  const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t per = (uint32_t)g.n * (uint32_t)g.nsite;
  if (e >= per) return;
  const int q = blockIdx.y;
  int a, z, y, k, x;
  quad_coords(e, g, hp, P, a, z, y, k, x);
  const size_t site = (size_t)a * g.plane + ((size_t)z * g.L2 + y) * g.L1 + x;
  const float4 v = src[(size_t)q * per + e];
  const float w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int rep = 4 * q + j;
    if (rep < B) dst[((size_t)rep * g.n + k) * g.nsite + site] = w[j];
  }
}


// the fixed-order block sum of quad.cuh, for the measure step's final sums
template <int V>
__device__ __forceinline__ void finish_block_sum(double (&x)[V], double (*red)[8]) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int i = 0; i < V; ++i) {
    double v = x[i];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xFFFFFFFFu, v, off);
    if (lane == 0) red[i][warp] = v;
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < V; ++i) {
    double v = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) v += red[i][w];
    x[i] = v;
  }
  __syncthreads();
}

// --------------------------------------------------------------------------------------------- host side
static int quad_period(const sck_plan* plan) { return plan->P; }

// The systems the interleaved kernels serve: vector models with a compile-time lattice table, every axis
// periodic, no mask, a colouring of x-period 1 or 2 that divides L1.
bool quad_ok(const sck_plan* plan, std::string* why) {
  auto no = [&](const char* m) {
    if (why) *why = m;
    return false;
  };
  const Geometry& g = plan->geom;
  if (g.n < 2) return no("interleaved storage is for vector models (n = 2 or 3)");
  if (find_spec(plan) == 0)
    return no("interleaved storage needs a crystal with a compile-time bond table (square, triangular, sc, bcc, "
              "bcc J1-J2, fcc) and no extra bond matrices");
  if (g.has_mask) return no("interleaved storage does not take a site mask");
  if (!g.per[0] || !g.per[1] || (g.dim == 3 && !g.per[2])) return no("interleaved storage needs a periodic box");
  if (plan->P != 1 && plan->P != 2) return no("interleaved storage needs a colouring of x-period 1 or 2");
  if (g.L1 % plan->P != 0) return no("the colouring's x-period must divide L1");
  return true;
}

static QuadParams quad_params(const sck_plan* plan, const sck_buffers* buf, int colour, int alpha) {
  QuadParams p;
  memset(&p, 0, sizeof(p));
  p.g = plan->geom;
  p.col = plan->col;
  for (int r = 0; r < SCK_MAX_FACTORS; ++r) p.fd_m[r] = make_fastdiv((uint32_t)plan->col.m[r]);
  p.hp = plan->geom.L1 / quad_period(plan);
  p.fd_hp = make_fastdiv((uint32_t)p.hp);
  p.fd_L2 = make_fastdiv((uint32_t)plan->geom.L2);
  for (int a = 0; a < SCK_MAX_BASIS; ++a)
    for (int gi = 0; gi < SCK_MAX_GROUPS; ++gi) p.J[a][gi] = plan->sub[a].J[gi];
  for (int k = 0; k < 3; ++k) {
    p.h[k] = plan->desc.h[k];
    p.hnz[k] = (k < plan->geom.n && plan->desc.h[k] != 0.0f) ? 1 : 0;
  }
  p.k2 = plan->desc.k2;
  p.spins = (float4*)buf->spins;
  p.k1 = buf->k1;
  p.beta = buf->beta;
  p.state = buf->state;
  p.colour = colour;
  p.alpha = alpha;
  return p;
}

static void launch_quad_grid(const sck_plan* plan, const QuadParams& p, dim3 grid, cudaStream_t s) {
  switch (plan->spec) {
    case Lat_square_1::id: quad_grid<Lat_square_1>(plan, p, grid, s); break;
    case Lat_triangular_1::id: quad_grid<Lat_triangular_1>(plan, p, grid, s); break;
    case Lat_sc_1::id: quad_grid<Lat_sc_1>(plan, p, grid, s); break;
    case Lat_bcc_1::id: quad_grid<Lat_bcc_1>(plan, p, grid, s); break;
    case Lat_bcc_1_2::id: quad_grid<Lat_bcc_1_2>(plan, p, grid, s); break;
    default: quad_grid<Lat_fcc_1>(plan, p, grid, s); break;
  }
}

static int quad_blocks_x(const sck_plan* plan) {
  const uint32_t per = (uint32_t)plan->geom.L3 * plan->geom.L2 * (plan->geom.L1 / plan->P);
  return (int)((per + 255) / 256);
}

static int launch_quad_params(const sck_plan* plan, QuadParams& p, cudaStream_t s) {
  const int Q = plan->Bp / 4;
  for (int q0 = 0; q0 < Q; q0 += 65535) {
    p.q0 = q0;
    const int nq = Q - q0 < 65535 ? Q - q0 : 65535;
    launch_quad_grid(plan, p, dim3((unsigned)quad_blocks_x(plan), (unsigned)nq), s);
    const int rc = cuda_status(cudaGetLastError(), "interleaved class launch");
    if (rc != SCK_OK) return rc;
  }
  return SCK_OK;
}

// One class of every quad (sweep offset 0: the sweep state[1] names).
int launch_quad_class(const sck_plan* plan, const sck_buffers* buf, int colour, int alpha, cudaStream_t s) {
  QuadParams p = quad_params(plan, buf, colour, alpha);
  return launch_quad_params(plan, p, s);
}

// ------------------------------------------------------------------------------------------ measure sweeps
// The coupling groups of class ci's sublattice whose bonds all reach classes earlier in the sweep order, or
// false when some group mixes earlier and later neighbours. For a linear colouring the neighbour's colour along
// bond (alpha -> alpha2, delta) is the site's colour shifted by K delta + o_alpha2 - o_alpha in every factor,
// the same for every site of the class, so the answer is one per (class, bond).
static bool class_lower_groups(const sck_plan* plan, int ci, unsigned* mask) {
  const sck_system_desc& d = plan->desc;
  const Colouring& col = plan->col;
  const int colour = d.classes[ci][0], alpha = d.classes[ci][1];
  int digit[SCK_MAX_FACTORS] = {0, 0, 0, 0};
  for (int r = col.r - 1, c = colour; r >= 0; --r) {
    digit[r] = c % col.m[r];
    c /= col.m[r];
  }
  const sck_sublattice& sub = d.sub[alpha];
  unsigned out = 0;
  int bi = 0;
  for (int gi = 0; gi < sub.n_groups; ++gi) {
    int lower = 0, later = 0;
    for (; bi < sub.group_end[gi]; ++bi) {
      const sck_bond& bd = sub.bonds[bi];
      int c2 = 0;
      for (int r = 0; r < col.r; ++r) {
        long long v = digit[r] + (long long)col.K[r][0] * bd.d[0] + (long long)col.K[r][1] * bd.d[1] +
                      (long long)col.K[r][2] * bd.d[2] + col.o[bd.alpha2][r] - col.o[alpha][r];
        v %= col.m[r];
        if (v < 0) v += col.m[r];
        c2 = c2 * col.m[r] + (int)v;
      }
      int idx = -1;
      for (int j = 0; j < d.n_classes; ++j)
        if (d.classes[j][0] == c2 && d.classes[j][1] == bd.alpha2) idx = j;
      if (idx < 0 || idx == ci) return false;   // a neighbour in no class, or in its own class: not a colouring
      (idx < ci ? lower : later) += 1;
    }
    if (lower && later) return false;
    if (lower) out |= 1u << gi;
  }
  *mask = out;
  return true;
}

bool quad_measure_fused(const sck_plan* plan) {
  if (plan->desc.n_classes > 64) return false;
  unsigned m = 0;
  for (int ci = 0; ci < plan->desc.n_classes; ++ci)
    if (!class_lower_groups(plan, ci, &m)) return false;
  return true;
}

size_t quad_measure_workspace(const sck_plan* plan) {
  const size_t fused = (size_t)plan->batch * plan->desc.n_classes * quad_blocks_x(plan) * (1 + plan->geom.n);
  const size_t exact = (size_t)plan->batch * quad_obs_blocks(plan) * OBS_VALUES;
  return (fused > exact ? fused : exact) * sizeof(double);
}

struct MeasureFinishParams {
  int n_classes, blocks_x, n, b;
  int cls_alpha[64];
};

// E[r] = sum of every class's and block's energy shares, M[r][alpha][k] = sum over the classes of sublattice
// alpha; one block per replica, fixed-order sums.
__global__ void __launch_bounds__(128) quad_measure_finish(const double* __restrict__ partial,
                                                           const __grid_constant__ MeasureFinishParams f,
                                                           double* __restrict__ E, double* __restrict__ M) {
  const int rep = blockIdx.x;
  const int V = 1 + f.n;
  const int per = f.n_classes * f.blocks_x;
  double acc[1 + SCK_MAX_BASIS * 3];
#pragma unroll
  for (int i = 0; i < 1 + SCK_MAX_BASIS * 3; ++i) acc[i] = 0.0;
  const double* src = partial + (size_t)rep * per * V;
  for (int i = threadIdx.x; i < per; i += blockDim.x) {
    const int a = f.cls_alpha[i / f.blocks_x];
    acc[0] += src[(size_t)i * V];
#pragma unroll
    for (int aa = 0; aa < SCK_MAX_BASIS; ++aa)
      if (aa == a)
#pragma unroll
        for (int k = 0; k < 3; ++k)
          if (k < f.n) acc[1 + aa * 3 + k] += src[(size_t)i * V + 1 + k];
  }
  __shared__ double red[1 + SCK_MAX_BASIS * 3][8];
  finish_block_sum<1 + SCK_MAX_BASIS * 3>(acc, red);
  if (threadIdx.x == 0) {
    if (E != nullptr) E[rep] = acc[0];
    if (M != nullptr)
      for (int a = 0; a < f.b; ++a)
        for (int k = 0; k < f.n; ++k) M[((size_t)rep * f.b + a) * f.n + k] = acc[1 + a * 3 + k];
  }
}

// One sweep whose class launches also accumulate the FP64 observables of the configuration it leaves (E and M
// of the first plan->batch replicas), then the counter advance. Needs quad_measure_fused(plan).
static int launch_measure_finish(const sck_plan* plan, const void* workspace, double* E, double* M, cudaStream_t s,
                                 int blocks_x);

// The pipeline's tickets per quad and class: site blocks of 256 threads grouped plan->quad_cpt to a ticket.
static int quad_pipe_tickets(const sck_plan* plan) {
  const int cpt = plan->quad_cpt > 0 ? plan->quad_cpt : 1;
  return (quad_blocks_x(plan) + cpt - 1) / cpt;
}

int launch_quad_measure_sweep(const sck_plan* plan, const sck_buffers* buf, double* E, double* M, void* workspace,
                              cudaStream_t s) {
  const int C = plan->desc.n_classes;
  for (int ci = 0; ci < C; ++ci) {
    QuadParams p = quad_params(plan, buf, plan->desc.classes[ci][0], plan->desc.classes[ci][1]);
    if (!class_lower_groups(plan, ci, &p.lower_groups)) {
      set_error("measure sweep: a coupling group mixes earlier and later classes");
      return SCK_ERR_UNSUPPORTED;
    }
    p.measure_ci = ci;
    p.n_classes = C;
    p.blocks_x = quad_blocks_x(plan);
    p.B = plan->batch;
    p.partial = (double*)workspace;
    const int rc = launch_quad_params(plan, p, s);
    if (rc != SCK_OK) return rc;
  }
  const int rc = launch_advance(buf->state, 1, s);
  if (rc != SCK_OK) return rc;
  return launch_measure_finish(plan, workspace, E, M, s, quad_blocks_x(plan));
}

static int launch_measure_finish(const sck_plan* plan, const void* workspace, double* E, double* M, cudaStream_t s,
                                 int blocks_x) {
  const int C = plan->desc.n_classes;
  MeasureFinishParams f;
  memset(&f, 0, sizeof(f));
  f.n_classes = C;
  f.blocks_x = blocks_x;
  f.n = plan->geom.n;
  f.b = plan->geom.b;
  for (int ci = 0; ci < C; ++ci) f.cls_alpha[ci] = plan->desc.classes[ci][1];
  quad_measure_finish<<<plan->batch, 128, 0, s>>>((const double*)workspace, f, E, M);
  return cuda_status(cudaGetLastError(), "measure sweep finish");
}

// Reference layout <-> interleaved storage: to_flat = 0 packs `flat` (B x N x sites floats) into `quads`,
// to_flat = 1 unpacks `quads` into `flat` (padding lanes are dropped).
int launch_quad_convert(const sck_plan* plan, float* flat, float4* quads, int to_flat, cudaStream_t s) {
  const Geometry& g = plan->geom;
  const uint32_t per = (uint32_t)g.n * (uint32_t)g.nsite;
  const int Q = plan->Bp / 4;
  const int hp = g.L1 / plan->P;
  for (int q0 = 0; q0 < Q; q0 += 65535) {
    const int nq = Q - q0 < 65535 ? Q - q0 : 65535;
    const dim3 grid((per + 255) / 256, (unsigned)nq);
    const size_t off4 = (size_t)q0 * per;
    if (to_flat)
      quad_unpack_kernel<<<grid, 256, 0, s>>>(quads + off4, flat + off4 * 4, g, hp, plan->P, plan->batch - 4 * q0);
    else
      quad_pack_kernel<<<grid, 256, 0, s>>>(flat + off4 * 4, quads + off4, g, hp, plan->P, plan->batch - 4 * q0);
    const int rc = cuda_status(cudaGetLastError(), to_flat ? "interleaved unpack" : "interleaved pack");
    if (rc != SCK_OK) return rc;
  }
  return SCK_OK;
}

int quad_obs_blocks(const sck_plan* plan) {
  const int Q = plan->Bp / 4;
  const int per_a = plan->geom.L3 * plan->geom.L2 * plan->geom.L1;
  const int most = (per_a + 255) / 256;
  const int want = (148 * 8 + Q - 1) / Q;
  return want < most ? (want < 1 ? 1 : want) : most;
}

int launch_quad_observables(const sck_plan* plan, const void* spins, int batch, const float* k1, double* E, double* M,
                            void* workspace, cudaStream_t s) {
  QuadObsParams p;
  memset(&p, 0, sizeof(p));
  p.g = plan->geom;
  for (int a = 0; a < SCK_MAX_BASIS; ++a) p.obs[a] = plan->obs[a];
  for (int k = 0; k < 3; ++k) p.h64[k] = plan->desc.h64[k];
  p.k2 = plan->desc.k2_64;
  p.hp = plan->geom.L1 / plan->P;
  p.blocks_per_quad = quad_obs_blocks(plan);
  p.B = batch;
  p.spins = (const float4*)spins;
  p.k1 = k1;
  p.partial = (double*)workspace;
  const int Q = (batch + 3) / 4;
  if (Q > 65535) return cuda_status(cudaErrorInvalidConfiguration, "interleaved observables: too many quads");
  const dim3 grid((unsigned)p.blocks_per_quad, (unsigned)Q);
  switch (plan->spec) {
    case Lat_square_1::id: quad_obs<Lat_square_1>(plan, p, grid, s); break;
    case Lat_triangular_1::id: quad_obs<Lat_triangular_1>(plan, p, grid, s); break;
    case Lat_sc_1::id: quad_obs<Lat_sc_1>(plan, p, grid, s); break;
    case Lat_bcc_1::id: quad_obs<Lat_bcc_1>(plan, p, grid, s); break;
    case Lat_bcc_1_2::id: quad_obs<Lat_bcc_1_2>(plan, p, grid, s); break;
    default: quad_obs<Lat_fcc_1>(plan, p, grid, s); break;
  }
  const int rc = cuda_status(cudaGetLastError(), "interleaved observables");
  if (rc != SCK_OK) return rc;
  return launch_observables_finish(p.partial, batch, p.blocks_per_quad, plan->geom.b, plan->geom.n, E, M, s);
}

// ---------------------------------------------------------------------------------------- pipeline host
size_t quad_pipe_counter_bytes(const sck_plan* plan) {
  const int Q = plan->Bp / 4;
  const int ngroups = (Q + plan->quad_group - 1) / plan->quad_group;
  return (size_t)(1 + ngroups * plan->desc.n_classes) * sizeof(unsigned);
}

int launch_quad_pipeline(const sck_plan* plan, const sck_buffers* buf, int n_sweeps, cudaStream_t s,
                         double* partial) {
  if (plan->pipe_counters == nullptr || plan->giveup_dev == nullptr) {
    set_error("the interleaved pipeline has no counters: call sck_plan_pipeline on this device");
    return SCK_ERR_INVALID;
  }
  QuadPipeParams pp;
  memset(&pp, 0, sizeof(pp));
  pp.p = quad_params(plan, buf, 0, 0);
  const int C = plan->desc.n_classes;
  pp.C = C;
  pp.D = plan->quad_skew;
  pp.group = plan->quad_group;
  pp.Q = plan->Bp / 4;
  pp.ngroups = (pp.Q + pp.group - 1) / pp.group;
  pp.blocks_x = quad_blocks_x(plan);
  pp.cpt = plan->quad_cpt > 0 ? plan->quad_cpt : 1;
  pp.tq = quad_pipe_tickets(plan);
  pp.T = pp.group * pp.tq;
  for (int ci = 0; ci < C; ++ci) {
    pp.cls[ci][0] = plan->desc.classes[ci][0];
    pp.cls[ci][1] = plan->desc.classes[ci][1];
  }
  pp.ticket = (unsigned*)plan->pipe_counters;
  pp.done = pp.ticket + 1;
  pp.wait_limit = plan->wait_limit;
  pp.giveup = plan->giveup_dev;
  pp.B = plan->batch;
  if (partial != nullptr)
    for (int ci = 0; ci < C; ++ci)
      if (!class_lower_groups(plan, ci, &pp.lower_groups[ci])) {
        set_error("measure sweep: a coupling group mixes earlier and later classes");
        return SCK_ERR_UNSUPPORTED;
      }
  const long long per_pos = (long long)(C / pp.D) * pp.T;
  const long long units_max = ((1ll << 30) / per_pos - C) / pp.D;
  const long long sweeps_per_launch = units_max / pp.ngroups;
  if (sweeps_per_launch < 1) return cuda_status(cudaErrorInvalidConfiguration, "interleaved pipeline: too many tickets");
  const size_t bytes = quad_pipe_counter_bytes(plan);
  for (int sw0 = 0; sw0 < n_sweeps; sw0 += (int)sweeps_per_launch) {
    const int n = (int)((long long)(n_sweeps - sw0) < sweeps_per_launch ? n_sweeps - sw0 : sweeps_per_launch);
    pp.units = n * pp.ngroups;
    pp.sweep_base = sw0;
    pp.partial = (partial != nullptr && sw0 + n == n_sweeps) ? partial : nullptr;
    int rc = cuda_status(cudaMemsetAsync(plan->pipe_counters, 0, bytes, s), "interleaved pipeline counters");
    if (rc != SCK_OK) return rc;
    const long long positions = (long long)pp.D * (pp.units - 1) + C;
    const unsigned blocks = (unsigned)(positions * per_pos);
    switch (plan->spec) {
      case Lat_square_1::id: quad_pipe<Lat_square_1>(plan, pp, blocks, s); break;
      case Lat_triangular_1::id: quad_pipe<Lat_triangular_1>(plan, pp, blocks, s); break;
      case Lat_sc_1::id: quad_pipe<Lat_sc_1>(plan, pp, blocks, s); break;
      case Lat_bcc_1::id: quad_pipe<Lat_bcc_1>(plan, pp, blocks, s); break;
      case Lat_bcc_1_2::id: quad_pipe<Lat_bcc_1_2>(plan, pp, blocks, s); break;
      default: quad_pipe<Lat_fcc_1>(plan, pp, blocks, s); break;
    }
    rc = cuda_status(cudaGetLastError(), "interleaved pipeline launch");
    if (rc != SCK_OK) return rc;
  }
  return SCK_OK;
}

// A measure step through the pipeline: n sweeps, the last one measured, the counter advance and the sums.
int launch_quad_pipeline_measure(const sck_plan* plan, const sck_buffers* buf, int n_sweeps, double* E, double* M,
                                 void* workspace, cudaStream_t s) {
  int rc = launch_quad_pipeline(plan, buf, n_sweeps, s, (double*)workspace);
  if (rc != SCK_OK) return rc;
  rc = launch_advance(buf->state, n_sweeps, s);
  if (rc != SCK_OK) return rc;
  return launch_measure_finish(plan, workspace, E, M, s, quad_pipe_tickets(plan));
}

}  // namespace sck
