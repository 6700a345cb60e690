// Host-side plan and the launch parameter blocks shared by the translation units of libsckb200.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "common.cuh"

namespace sck {

// Everything a class launch needs except the bond list of its sublattice.
struct Common {
  Geometry g;
  Colouring col;
  int B;             // replicas the kernel computes (32 W for packed storage)
  int W;             // words per site (packed / bitwise)
  int P, bx, rows;   // x-period of the colouring, class sites per row (ceil(L1 / P)), rows = L3 * L2
  float h[3];
  int hnz[3];
  float k2;
  int keys;          // Ising acceptance-table keys per sublattice
  int lut_rep_stride;
  int Z1, NT, field; // bitwise table: Z + 1, 2 (Z + 1)^2, field present
  const void* src;
  void* dst;
  const int8_t* mask;
  const float* k1;
  const float* beta;
  const void* table;
  const int64_t* state;
  int* giveup;       // the plan's host-mapped flag, raised (system scope) when a bounded wait gives up; may be null
  unsigned wait_limit;  // polls of a bounded wait before it gives up
  FastDiv fd_bx, fd_L1, fd_L2, fd_m[SCK_MAX_FACTORS];
};

// First x in [0, P) of row (y, z) whose site on sublattice `alpha` has colour `colour`, or L1 when the row holds
// no site of the class. Along a row the colour has period P and each colour of the row appears at most once per
// period, so stepping the per-factor residues through one period finds it.
__device__ __forceinline__ int first_class_x(const Common& c, int colour, int alpha, int y, int z) {
  int g[SCK_MAX_FACTORS];
#pragma unroll
  for (int r = 0; r < SCK_MAX_FACTORS; ++r) {
    if (r < c.col.r) {
      const uint32_t v = (uint32_t)(c.col.K[r][1] * y + c.col.K[r][2] * z + c.col.o[alpha][r]);
      g[r] = (int)(v - fdiv(v, c.fd_m[r]) * (uint32_t)c.col.m[r]);
    }
  }
  for (int q = 0; q < c.P; ++q) {
    int idx = 0;
#pragma unroll
    for (int r = 0; r < SCK_MAX_FACTORS; ++r) {
      if (r < c.col.r) {
        idx = idx * c.col.m[r] + g[r];
        g[r] += c.col.K[r][0];
        if (g[r] >= c.col.m[r]) g[r] -= c.col.m[r];
      }
    }
    if (idx == colour) return q;
  }
  return c.g.L1;
}

// (t = row * bx + j) -> class site (x, y, z) of class `colour` on sublattice `alpha`, false when the row holds
// no site of the class.
__device__ __forceinline__ bool class_site(const Common& c, int colour, int alpha, uint32_t t, int& x, int& y,
                                           int& z) {
  const uint32_t row = fdiv(t, c.fd_bx);
  const int j = (int)(t - row * (uint32_t)c.bx);
  z = (int)fdiv(row, c.fd_L2);
  y = (int)row - z * c.g.L2;
  const int x0 = colour >= 0 ? first_class_x(c, colour, alpha, y, z) : 0;
  x = x0 + c.P * j;
  return x < c.g.L1;
}

struct ClassParams {
  Common c;
  SubDev sub;
  int colour, alpha;
};

struct SeqParams {
  Common c;
  SubDev sub[SCK_MAX_BASIS];
  int n_classes;
  int classes[128][2];
};

struct ObsParams {
  Geometry g;
  int B, storage;    // 0 int8, 1 float32, 2 packed words
  SubDev sub[SCK_MAX_BASIS];
  SubObs obs[SCK_MAX_BASIS];
  double h64[3];
  double k2;
  int blocks_per_rep;
  FastDiv fd_plane, fd_L1, fd_L2;
  const void* spins;
  const int8_t* mask;
  const float* k1;
  double* partial;
};

constexpr int OBS_VALUES = 16;   // E + b * n magnetization sums (<= 12), padded

}  // namespace sck

struct sck_plan {
  sck_system_desc desc;
  sck::Geometry geom;
  sck::Colouring col;
  sck::SubDev sub[SCK_MAX_BASIS];
  sck::SubObs obs[SCK_MAX_BASIS];
  int mode, batch;
  int Bp, W, rows_storage;
  int P, bx;
  int keys;
  int Z, Z1, NP, field;
  int ising_lut;   // Ising chain with the host-built exp table (INT8, F32 with n = 1, PACKED)
  int spec;        // id of the matching compile-time lattice table (lattices.h), 0 = generic kernels
  int kernel_kind; // specialised class kernels: 1 lattice, 2 segment (segment.cu), 3 tile (tile.cu) where eligible
  long long l2_budget;  // bytes of L2 the group pipeline may fill
  long long resident_limit;  // largest replica (bytes) whose sweeps run resident in shared memory; 0 = never
  void* pipe_counters;       // device memory of the group pipeline's ticket and completion counters
  size_t pipe_bytes;
  int pipe_device;           // the device that holds them
  int quad_group, quad_skew; // interleaved pipeline: quads per group (0 = class by class) and class skew
  int quad_cpt;              //   and site blocks of 256 threads per ticket
  unsigned wait_limit;       // polls of a pipeline completion counter before a block gives up
  int* giveup_host;          // host-mapped flag a kernel raises when a bounded wait gives up (host view)
  int* giveup_dev;           //   and its device view
};

namespace sck {
void set_rows(Common& c, int P, int bx);
void set_error(const std::string& msg);
int cuda_status(cudaError_t e, const char* where);

// launchers (return SCK_OK or an error code)
int launch_class(const sck_plan* plan, const Common& c, int colour, int alpha, cudaStream_t s);
int launch_sequential(const sck_plan* plan, const Common& c, cudaStream_t s);
int launch_bitwise_class(const sck_plan* plan, const Common& c, int colour, int alpha, cudaStream_t s);
int launch_bitwise_sequential(const sck_plan* plan, const Common& c, cudaStream_t s);
int obs_blocks_per_rep(const sck_plan* plan, int batch);
int obs_launch_blocks(const sck_plan* plan, int storage, int batch);
int check_observables_request(const sck_plan* plan, int storage, int batch);
int made_wait_timeouts(unsigned long long* count);
int made_set_wait_limit(long long polls);   // polls before the tensor-core GEMM's stage waits give up   // bounded waits of the learned proposal's kernels that gave up
int launch_observables(const sck_plan* plan, const void* spins, int storage, int batch, const int8_t* mask,
                       const float* k1, double* E, double* M, void* workspace, cudaStream_t s);
int launch_observables_finish(const double* partial, int B, int blocks_per_rep, int b, int n, double* E, double* M,
                              cudaStream_t s);
int launch_observables_fold(const sck_plan* plan, int batch, const double* E, const double* M, double n_active,
                            const double* E_ref, double* acc, double* accv, cudaStream_t s);
int launch_topological_charge(const sck_plan* plan, const float* spins, const int8_t* mask, int batch, int z,
                              double* Q, cudaStream_t s);
int launch_pack(const sck_plan* plan, const int8_t* spins, int32_t* words, cudaStream_t s);
int launch_unpack(const sck_plan* plan, const int32_t* words, const int8_t* mask, int8_t* spins, cudaStream_t s);
int launch_advance(int64_t* state, int n, cudaStream_t s);
int find_spec(const sck_plan* plan);
size_t resident_bytes(const sck_plan* plan);
int launch_resident(const sck_plan* plan, const Common& c, int n_sweeps, cudaStream_t s);
int launch_spec_class(const sck_plan* plan, const Common& c, int colour, int alpha, cudaStream_t s);
int launch_spec_pipeline(const sck_plan* plan, const Common& c, int n_sweeps, int group, void* counters,
                         cudaStream_t s);
size_t stream_counter_bytes(const sck_plan* plan, int group);
int stream_wait_timeouts(unsigned long long* count);   // group pipeline waits that gave up
// interleaved storage of vector models (quad.cu)
bool quad_ok(const sck_plan* plan, std::string* why);
int launch_quad_class(const sck_plan* plan, const sck_buffers* buf, int colour, int alpha, cudaStream_t s);
int launch_quad_convert(const sck_plan* plan, float* flat, float4* quads, int to_flat, cudaStream_t s);
int quad_obs_blocks(const sck_plan* plan);
bool quad_measure_fused(const sck_plan* plan);
size_t quad_measure_workspace(const sck_plan* plan);
size_t quad_pipe_counter_bytes(const sck_plan* plan);
int launch_quad_pipeline(const sck_plan* plan, const sck_buffers* buf, int n_sweeps, cudaStream_t s,
                         double* partial);
int launch_quad_pipeline_measure(const sck_plan* plan, const sck_buffers* buf, int n_sweeps, double* E, double* M,
                                 void* workspace, cudaStream_t s);
int launch_quad_measure_sweep(const sck_plan* plan, const sck_buffers* buf, double* E, double* M, void* workspace,
                              cudaStream_t s);
int launch_quad_observables(const sck_plan* plan, const void* spins, int batch, const float* k1, double* E, double* M,
                            void* workspace, cudaStream_t s);
}  // namespace sck
