// Specialised class kernels for the common crystals and the L2-resident group pipeline.
//
// Specialisation. When a system's bond lists equal one of the compile-time tables of lattices.h (one coupling
// group per shell, no extra matrices), its class launches run kernels in which every neighbour offset is a
// constant: the wrapped coordinates of a site are formed once for offsets -R..R per axis and every bond costs
// one add and one load per component. Ising keeps the integer key and the host table (bit-exact); vector models
// run two replicas per thread in packed float32x2 arithmetic (add.rn.f32x2 / mul.rn.f32x2, round-to-nearest
// per lane, same operation order as the generic kernel), with proposal trigonometry and exp on the SFU
// (__sinf / __cosf on [-pi, pi], __expf): per-spin differences from the reference stay ~1e-6. Vector models on
// lattices whose classes alternate along x run the segment kernels of segment.cu instead when the tuning level
// asks for them and their box allows it.
//
// Group pipeline. A sweep visits its C classes in order, and each class launch reads the whole state. When the
// state is larger than L2, the replicas are cut into groups whose C-group working set fits in L2, and launch k
// runs class c on group k - c for every c at once (a diagonal over (group, class)): the C launches that touch a
// group run back to back, so after its first read from HBM a group stays in L2 until its sweep is done. Each
// replica's chain is unchanged: its classes still run in order, one launch after another.
#include "spec_site.cuh"

namespace sck {

// ------------------------------------------------------------------------------------------------- kernels
// Grid (ceil(rows * bx / 256), n_tasks * units_per_task). Block y-slot -> (task, replica or replica pair).
template <class Lat, int N, typename ST, bool PER, int NSL>
__global__ void __launch_bounds__(256) spec_task_kernel(const __grid_constant__ SpecParams p) {
  const uint32_t per = (uint32_t)p.c.rows * (uint32_t)p.c.bx;
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= per) return;
  const int ti = blockIdx.y / p.units_per_task;
  const int unit = blockIdx.y - ti * p.units_per_task;
  const Task task = p.tasks[ti];
  constexpr int per_unit = N == 1 ? 1 : 2;
  const int rep = task.rep_begin + unit * per_unit;
  if (rep >= task.rep_end) return;
  int x, y, z;
  if (!class_site(p.c, task.colour, task.alpha, t, x, y, z)) return;
  const int32_t key = sweep_key_at(p.c.state, task.sweep_offset);
  static_for<0, Lat::b>([&](auto ac) {
    constexpr int a = decltype(ac)::value;
    if (a != task.alpha) return;
    if constexpr (N == 1) {
      ising_spec_site<Lat, a, ST, PER>(p.c, rep, x, y, z, key);
    } else {
      vec_spec_pair<Lat, a, N, PER, NSL>(p.c, p.J[a], rep, rep + 1 < task.rep_end, x, y, z, key);
    }
  });
}

// ----------------------------------------------------------------------------------- the streamed pipeline
// One launch runs the group pipeline of several sweeps. Tickets, taken from a counter in the order blocks start,
// enumerate stages k = 0, 1, ...; stage k holds class ci of unit k - ci (unit = sweep-major group) for every ci,
// each class task split into T tickets (slot of the group x chunk of site blocks). Before touching spins a
// block waits until every ticket of the task it follows has finished: class ci - 1 of its unit, or, for class
// 0, class C - 1 of the same group's previous sweep. That task holds smaller tickets, so its blocks started
// before this one and are running or done: the wait ends. Tasks of one group are therefore serialised exactly
// as class launches are, tasks of different groups overlap freely, and a group's state is read from HBM once
// per sweep while its C classes pass over it from L2.
constexpr int kStreamSiteBlocks = 1;                 // site blocks of 256 threads per ticket
static __device__ unsigned long long g_stream_wait_timeouts;

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* a) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(a) : "memory");
  return v;
}

struct StreamTask {
  int go;            // 0: no task (pipeline fill / drain) or a wait that gave up
  int rep, rep_end;  // first replica of this block's slot, end of its group
  int colour, alpha, sweep;
  int done;          // index of this task's completion counter
  uint32_t t0;       // first class-site thread of this block
};

template <class Lat, int N, typename ST, bool PER, int NSL>
__global__ void __launch_bounds__(256, 5) stream_kernel(const __grid_constant__ StreamParams p) {
  __shared__ StreamTask s;
  if (threadIdx.x == 0) {
    const unsigned tk = atomicAdd(p.ticket, 1u);
    const unsigned stage = (unsigned)p.C * (unsigned)p.T;
    const unsigned k = tk / stage;
    const unsigned r = tk - k * stage;
    const int ci = (int)(r / (unsigned)p.T), j = (int)(r - (unsigned)ci * (unsigned)p.T);
    const int u = (int)k - ci;
    s.go = 0;
    s.done = -1;
    if (u >= 0 && u < p.units) {
      const int sw = u / p.ngroups, g = u - sw * p.ngroups;
      const int q = j / p.chunks, chunk = j - q * p.chunks;
      constexpr int per_slot = N == 1 ? 1 : 2;
      s.rep = g * p.group + q * per_slot;
      s.rep_end = min(p.c.B, (g + 1) * p.group);
      s.colour = p.cls[ci][0];
      s.alpha = p.cls[ci][1];
      s.sweep = p.sweep_base + sw;
      s.done = g * p.C + ci;
      s.t0 = (uint32_t)chunk * (kStreamSiteBlocks * 256u);
      const unsigned* dep = nullptr;
      unsigned need = 0;
      if (ci > 0) {
        dep = p.done + s.done - 1;
        need = (unsigned)(sw + 1) * (unsigned)p.T;
      } else if (sw > 0) {
        dep = p.done + g * p.C + p.C - 1;
        need = (unsigned)sw * (unsigned)p.T;
      }
      int go = 1;
      if (dep != nullptr) {
        unsigned polls = 0;
        while (ld_acquire_u32(dep) < need) {
          if (++polls > p.c.wait_limit) {
            go = 0;
            atomicAdd(&g_stream_wait_timeouts, 1ull);
            if (p.c.giveup != nullptr) atomicExch_system(p.c.giveup, 1);
            break;
          }
          __nanosleep(100);
        }
      }
      s.go = go && s.rep < s.rep_end;
    }
  }
  __syncthreads();
  if (s.done < 0) return;                              // the pipeline's fill and drain: no task
  if (s.go) {
    const int rep = s.rep, rep_end = s.rep_end, alpha = s.alpha;
    const int32_t key = sweep_key_at(p.c.state, s.sweep);
    const uint32_t per = (uint32_t)p.c.rows * (uint32_t)p.c.bx;
#pragma unroll 1
    for (int sb = 0; sb < kStreamSiteBlocks; ++sb) {
      const uint32_t t = s.t0 + sb * 256u + threadIdx.x;
      int x, y, z;
      if (t < per && class_site(p.c, s.colour, alpha, t, x, y, z)) {
        static_for<0, Lat::b>([&](auto ac) {
          constexpr int a = decltype(ac)::value;
          if (a != alpha) return;
          if constexpr (N == 1) {
            ising_spec_site<Lat, a, ST, PER>(p.c, rep, x, y, z, key);
          } else {
            vec_spec_pair<Lat, a, N, PER, NSL>(p.c, p.J[a], rep, rep + 1 < rep_end, x, y, z, key);
          }
        });
      }
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    atomicAdd(p.done + s.done, 1u);   // finished (or given up): later tasks of this group may start
  }
}

int stream_wait_timeouts(unsigned long long* count) {
  return cuda_status(cudaMemcpyFromSymbol(count, g_stream_wait_timeouts, sizeof(*count)), "stream wait timeouts");
}

// ------------------------------------------------------------------------------------------ host: matching
template <class Lat>
static bool matches(const sck_plan* p) {
  const sck_system_desc& d = p->desc;
  if (d.b != Lat::b || d.dim != Lat::dim) return false;
  for (int a = 0; a < d.b; ++a) {
    const sck_sublattice& s = d.sub[a];
    if (s.n_groups != Lat::groups || s.n_bonds != Lat::n_bonds(a) || s.n_extra != 0) return false;
    for (int gi = 0; gi < s.n_groups; ++gi)
      if (!s.group_apply[gi] || s.group_end[gi] != Lat::group_end(a, gi)) return false;
    for (int i = 0; i < s.n_bonds; ++i) {
      const BondC b = Lat::bond(a, i);
      const sck_bond& e = s.bonds[i];
      if (e.alpha2 != b.a2 || e.d[0] != b.dx || e.d[1] != b.dy || e.d[2] != b.dz || e.extra != -1) return false;
    }
  }
  return true;
}

int find_spec(const sck_plan* p) {
  if (p->mode != SCK_MODE_INT8 && p->mode != SCK_MODE_F32 && p->mode != SCK_MODE_QUAD) return 0;
  if (matches<Lat_square_1>(p)) return Lat_square_1::id;
  if (matches<Lat_triangular_1>(p)) return Lat_triangular_1::id;
  if (matches<Lat_sc_1>(p)) return Lat_sc_1::id;
  if (matches<Lat_bcc_1>(p)) return Lat_bcc_1::id;
  if (matches<Lat_bcc_1_2>(p)) return Lat_bcc_1_2::id;
  if (matches<Lat_fcc_1>(p)) return Lat_fcc_1::id;
  return 0;
}

// ------------------------------------------------------------------------------------------- host: launches
template <class Lat, int N, typename ST, bool PER, int NSL, class P>
static void launch_one(const P& p, dim3 grid, cudaStream_t s) {
  if constexpr (std::is_same_v<P, SpecParams>)
    spec_task_kernel<Lat, N, ST, PER, NSL><<<grid, 256, 0, s>>>(p);
  else
    stream_kernel<Lat, N, ST, PER, NSL><<<grid, 256, 0, s>>>(p);
}

template <class Lat, int N, bool PER, class P>
static void launch_vec(const sck_plan* plan, const P& p, dim3 grid, cudaStream_t s) {
  // replicas of 2^16 .. 2^19 sites on periodic boxes: component strides up to 2 MiB fit a load's immediate offset
  if constexpr (PER) {
    const int64_t ns = plan->geom.nsite;
    if (ns == (1 << 16)) return launch_one<Lat, N, float, PER, 16>(p, grid, s);
    if (ns == (1 << 17)) return launch_one<Lat, N, float, PER, 17>(p, grid, s);
    if (ns == (1 << 18)) return launch_one<Lat, N, float, PER, 18>(p, grid, s);
    if (ns == (1 << 19)) return launch_one<Lat, N, float, PER, 19>(p, grid, s);
  }
  launch_one<Lat, N, float, PER, 0>(p, grid, s);
}

template <class Lat, bool PER, class P>
static void launch_lat_per(const sck_plan* plan, const P& p, dim3 grid, cudaStream_t s) {
  if (plan->geom.n == 1) {
    if (plan->mode == SCK_MODE_INT8)
      launch_one<Lat, 1, int8_t, PER, 0>(p, grid, s);
    else
      launch_one<Lat, 1, float, PER, 0>(p, grid, s);
  } else if (plan->geom.n == 2) {
    launch_vec<Lat, 2, PER>(plan, p, grid, s);
  } else {
    launch_vec<Lat, 3, PER>(plan, p, grid, s);
  }
}

// All axes periodic (2D: x and y) with every extent >= the bond reach: the branch-free wrap applies.
template <class Lat>
static bool periodic_box(const sck_plan* plan) {
  const Geometry& g = plan->geom;
  if (!g.per[0] || !g.per[1] || g.L1 < Lat::reach || g.L2 < Lat::reach) return false;
  return g.dim == 2 || (g.per[2] && g.L3 >= Lat::reach);
}

int spec_periodic_box(const sck_plan* plan) {
  switch (plan->spec) {
    case Lat_square_1::id: return periodic_box<Lat_square_1>(plan) ? 1 : 0;
    case Lat_triangular_1::id: return periodic_box<Lat_triangular_1>(plan) ? 1 : 0;
    case Lat_sc_1::id: return periodic_box<Lat_sc_1>(plan) ? 1 : 0;
    case Lat_bcc_1::id: return periodic_box<Lat_bcc_1>(plan) ? 1 : 0;
    case Lat_bcc_1_2::id: return periodic_box<Lat_bcc_1_2>(plan) ? 1 : 0;
    case Lat_fcc_1::id: return periodic_box<Lat_fcc_1>(plan) ? 1 : 0;
    default: return 0;
  }
}

template <class Lat, class P>
static void launch_lat(const sck_plan* plan, const P& p, dim3 grid, cudaStream_t s) {
  if (periodic_box<Lat>(plan))
    launch_lat_per<Lat, true>(plan, p, grid, s);
  else
    launch_lat_per<Lat, false>(plan, p, grid, s);
}

// replicas per grid y-slot: vector models pair two replicas per thread in the lattice kernels
template <class P>
static void launch_spec_grid(const sck_plan* plan, const P& p, dim3 grid, cudaStream_t s) {
  switch (plan->spec) {
    case Lat_square_1::id: launch_lat<Lat_square_1>(plan, p, grid, s); break;
    case Lat_triangular_1::id: launch_lat<Lat_triangular_1>(plan, p, grid, s); break;
    case Lat_sc_1::id: launch_lat<Lat_sc_1>(plan, p, grid, s); break;
    case Lat_bcc_1::id: launch_lat<Lat_bcc_1>(plan, p, grid, s); break;
    case Lat_bcc_1_2::id: launch_lat<Lat_bcc_1_2>(plan, p, grid, s); break;
    default: launch_lat<Lat_fcc_1>(plan, p, grid, s); break;
  }
}

static int slot_replicas(const sck_plan* plan) { return plan->geom.n == 1 || seg_kernel_ok(plan) ? 1 : 2; }

static int launch_tasks(const sck_plan* plan, SpecParams& p, cudaStream_t s) {
  const int per_unit = slot_replicas(plan);
  int most = 1;
  for (int i = 0; i < p.n_tasks; ++i) {
    const int n = p.tasks[i].rep_end - p.tasks[i].rep_begin;
    if (n > most) most = n;
  }
  p.units_per_task = (most + per_unit - 1) / per_unit;
  const long long ys = (long long)p.units_per_task * p.n_tasks;
  if (ys > 65535) return cuda_status(cudaErrorInvalidConfiguration, "task launch: too many replicas per launch");
  if (seg_kernel_ok(plan)) return launch_seg_tasks(plan, p, (int)ys, s);
  const uint32_t per = (uint32_t)p.c.rows * (uint32_t)p.c.bx;
  launch_spec_grid(plan, p, dim3((per + 255) / 256, (unsigned)ys), s);
  return cuda_status(cudaGetLastError(), "specialised class launch");
}

static SpecParams spec_params(const sck_plan* plan, const Common& c) {
  SpecParams p;
  memset(&p, 0, sizeof(p));
  p.c = c;
  for (int a = 0; a < SCK_MAX_BASIS; ++a)
    for (int gi = 0; gi < SCK_MAX_GROUPS; ++gi) p.J[a][gi] = plan->sub[a].J[gi];
  return p;
}

// One class over all replicas, in chunks of at most 65535 grid rows.
int launch_spec_class(const sck_plan* plan, const Common& c, int colour, int alpha, cudaStream_t s) {
  if (tile_kernel_ok(plan)) return launch_tile_class(plan, c, colour, alpha, s);
  SpecParams p = spec_params(plan, c);
  const int chunk = 65535 * slot_replicas(plan);
  for (int r0 = 0; r0 < c.B; r0 += chunk) {
    p.n_tasks = 1;
    p.tasks[0] = Task{colour, alpha, r0, r0 + chunk < c.B ? r0 + chunk : c.B, 0};
    const int rc = launch_tasks(plan, p, s);
    if (rc != SCK_OK) return rc;
  }
  return SCK_OK;
}

size_t stream_counter_bytes(const sck_plan* plan, int group) {
  const int ngroups = (plan->Bp + group - 1) / group;
  return (size_t)(1 + ngroups * plan->desc.n_classes) * sizeof(unsigned);
}

// n sweeps of the group pipeline (streamed kernel, one launch per chunk of sweeps); state[1] is advanced by
// the caller. `counters` holds stream_counter_bytes(plan, group) bytes of device memory, zeroed here before
// every launch.
int launch_spec_pipeline(const sck_plan* plan, const Common& c, int n_sweeps, int group, void* counters,
                         cudaStream_t s) {
  if (counters == nullptr) {
    set_error("the group pipeline has no completion counters (set an L2 budget with sck_plan_tune)");
    return SCK_ERR_INVALID;
  }
  const int C = plan->desc.n_classes;
  StreamParams p;
  memset(&p, 0, sizeof(p));
  p.c = c;
  for (int a = 0; a < SCK_MAX_BASIS; ++a)
    for (int gi = 0; gi < SCK_MAX_GROUPS; ++gi) p.J[a][gi] = plan->sub[a].J[gi];
  p.C = C;
  for (int ci = 0; ci < C; ++ci) {
    p.cls[ci][0] = plan->desc.classes[ci][0];
    p.cls[ci][1] = plan->desc.classes[ci][1];
  }
  p.group = group;
  p.ngroups = (c.B + group - 1) / group;
  const int per_slot = plan->geom.n == 1 ? 1 : 2;
  const long long site_blocks = ((long long)c.rows * c.bx + 255) / 256;
  p.chunks = (int)((site_blocks + kStreamSiteBlocks - 1) / kStreamSiteBlocks);
  p.T = ((group + per_slot - 1) / per_slot) * p.chunks;
  p.ticket = (unsigned*)counters;
  p.done = p.ticket + 1;
  // tickets of a launch, (units + C - 1) x C x T, stay below 2^30
  const long long stage = (long long)C * p.T;
  const long long most_units = (1ll << 30) / stage - (C - 1);
  const long long sweeps_per_launch = most_units / p.ngroups;
  if (sweeps_per_launch < 1) return cuda_status(cudaErrorInvalidConfiguration, "group pipeline: too many tickets");
  const size_t bytes = stream_counter_bytes(plan, group);
  for (int sw0 = 0; sw0 < n_sweeps; sw0 += (int)sweeps_per_launch) {
    const int n = (int)((long long)(n_sweeps - sw0) < sweeps_per_launch ? n_sweeps - sw0 : sweeps_per_launch);
    p.units = n * p.ngroups;
    p.sweep_base = sw0;
    int rc = cuda_status(cudaMemsetAsync(counters, 0, bytes, s), "group pipeline counters");
    if (rc != SCK_OK) return rc;
    launch_spec_grid(plan, p, dim3((unsigned)((p.units + C - 1) * stage)), s);
    rc = cuda_status(cudaGetLastError(), "group pipeline launch");
    if (rc != SCK_OK) return rc;
  }
  return SCK_OK;
}

}  // namespace sck
