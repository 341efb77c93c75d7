// The single-scene fluid object behind the C ABI (aq_fluid), shared by the
// single-scene host code (fluid.cu) and the batch host code (batch.cu).
#pragma once

#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "../../include/aquarius_b200.h"
#include "aq_kernels.cuh"

namespace aqb {
inline aq_status fail(aq_status st, const std::string& msg) { return set_last_error(st, msg); }
struct UActs;
struct MeshState;                  // surface mesher buffers (mesh.cu)
void mesh_release(MeshState* s);

// The reference's random0to1() (Common/Commons.h:3-5) over glibc rand(),
// replayed without touching the process's own rand() state: random_r over a
// 128-byte TYPE_3 state gives the sequence of srand(seed); rand().
struct HostRand {
  struct random_data rd;
  char state[128];
  explicit HostRand(unsigned seed) {
    memset(&rd, 0, sizeof(rd));
    memset(state, 0, sizeof(state));
    initstate_r(seed, state, sizeof(state), &rd);
  }
  HostRand(const HostRand&) = delete;
  HostRand& operator=(const HostRand&) = delete;
  float random0to1() {
    int32_t v;
    random_r(&rd, &v);
    return (float)v / (float)RAND_MAX;
  }
};
}  // namespace aqb

struct aq_fluid {
  using Dims = aqb::Dims;
  using StepParams = aqb::StepParams;
  using Particles = aqb::Particles;
  using SolveState = aqb::SolveState;
  using JacobiPlan = aqb::JacobiPlan;

  aq_config cfg{};
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaStream_t side = nullptr;  // body capture
  bool own_stream = false;
  Dims d{};
  StepParams sp{};
  int n = 0;
  bool multiphase = false;
  int phase = 0;
  double time = 0.0;
  int nv_cur = 2, has_cur = 2;  // which buffer holds newVelocity / has bits
  // Stage 1 is fused with the sort; a following stage-2 call then has no work.
  bool sorted_by_stage1 = false;
  // Subtracted from cell-table and sort-index values on download (a scene
  // viewed inside a batch's concatenated arrays).
  int index_base = 0;

  Particles cur{}, tmp{};
  int *key = nullptr, *slot = nullptr, *perm_u = nullptr, *sort_index = nullptr;
  int *count = nullptr, *off = nullptr, *tile_sums = nullptr;
  float *u0 = nullptr, *v0 = nullptr, *w0 = nullptr;
  float *un1 = nullptr, *vn1 = nullptr, *wn1 = nullptr;
  float *un2 = nullptr, *vn2 = nullptr, *wn2 = nullptr;
  uint8_t *h1 = nullptr, *h2 = nullptr;
  int8_t* type = nullptr;
  float *density = nullptr, *div = nullptr, *rhs = nullptr, *pa = nullptr, *pb = nullptr;
  int* pcount = nullptr;
  float4 *vf = nullptr, *nvf = nullptr, *nvf2 = nullptr;
  uint8_t* bact = nullptr;
  double* part_b2 = nullptr;
  int* part_nf = nullptr;
  int nbricks = 0;
  double* jpart = nullptr;
  int jpart_cap = 0;
  SolveState* ss = nullptr;
  SolveState* ss_host = nullptr;
  // persistent solve
  int* items = nullptr;
  int* n_items = nullptr;
  unsigned int* bar = nullptr;
  double* ppart = nullptr;
  int ctas = 0;
  aqb::BarrierTest barrier_test{-1, 0};  // aq_fluid_test_barrier_timeout
  // resident solve (plan rows 4): tile list and CTAs of its launch
  int* tiles = nullptr;
  int* n_tiles = nullptr;
  int res_ctas = 0;

  JacobiPlan plan{4, 16, 32};
  // learned warm start (AQ_PRESSURE_LEARNED)
  aq_unet* net = nullptr;
  aqb::UActs* net_acts = nullptr;
  float *za = nullptr, *zb = nullptr;  // the zero-init path of the first sweeps
  double* jpart2 = nullptr;
  int* pick = nullptr;  // 1: the zero-init path won
  // list plan: active warp rows of the current system
  int *row_items = nullptr, *n_row_items = nullptr;
  unsigned int* resid_ticket = nullptr;  // last-block ticket of the fused residual check
  // rand() state after seeding: ink seeding continues the sequence
  std::unique_ptr<aqb::HostRand> rng;
  // ink particles (positions / velocities only; frac stays null)
  Particles ink{};
  int n_ink = 0;
  bool ink_on = false;
  aqb::MeshState* mesher = nullptr;  // made by the first aq_fluid_mesh call
  cudaGraphExec_t exec = nullptr;
  bool use_graph = true;
  int graph_launches = 0;  // launches outside the residual loop
  int body_launches = 0;   // launches per residual-loop iteration

  std::vector<void*> allocs;
  // PCG scratch (lazily allocated)
  double *pcg_b = nullptr, *pcg_x = nullptr, *pcg_r = nullptr, *pcg_z = nullptr, *pcg_p = nullptr,
         *pcg_q = nullptr, *pcg_part = nullptr;

  ~aq_fluid() {
    if (device >= 0) cudaSetDevice(device);
    if (stream) cudaStreamSynchronize(stream);
    if (exec) cudaGraphExecDestroy(exec);
    if (mesher) aqb::mesh_release(mesher);
    for (void* p : allocs) cudaFree(p);
    if (ss_host) cudaFreeHost(ss_host);
    if (side) cudaStreamDestroy(side);
    if (own_stream && stream) cudaStreamDestroy(stream);
  }

  template <typename T>
  aq_status alloc(T** p, size_t count_) {
    void* q = nullptr;
    const size_t bytes = count_ * sizeof(T) > 0 ? count_ * sizeof(T) : 16;
    cudaError_t e = cudaMalloc(&q, bytes);
    if (e != cudaSuccess)
      return aqb::fail(e == cudaErrorMemoryAllocation ? AQ_ERR_OUT_OF_MEMORY : AQ_ERR_CUDA,
                  std::string("cudaMalloc: ") + cudaGetErrorString(e));
    allocs.push_back(q);
    *p = (T*)q;
    e = cudaMemsetAsync(q, 0, bytes, stream);
    if (e != cudaSuccess) return aqb::fail(AQ_ERR_CUDA, cudaGetErrorString(e));
    return AQ_OK;
  }

  float* nvx(int which) const { return which == 1 ? un1 : un2; }
  float* nvy(int which) const { return which == 1 ? vn1 : vn2; }
  float* nvz(int which) const { return which == 1 ? wn1 : wn2; }
  uint8_t* hb(int which) const { return which == 1 ? h1 : h2; }

  aq_status allocate();
  aq_status seed_and_init();
  // stage enqueues (eager or under capture)
  aq_status enq_particles(bool move);
  aq_status enq_p2g(bool forces);
  aq_status enq_divergence();
  aq_status enq_solve_fixed(int sweeps);
  aq_status enq_solve_body(bool set_cond, unsigned long long handle, int* launches);
  aq_status enq_solve_residual_eager();
  aq_status enq_learned_start();
  int solve_sweeps_done() const;  // sweeps the warm start already did (0 without it)
  aq_status enq_row_items();       // list plan: rebuild the active-row list (no-op otherwise)
  aq_status enq_project();
  aq_status enq_extrapolate();
  aq_status enq_diffuse();
  aq_status enq_ink();     // advance the ink (no-op without ink)
  aq_status enable_ink();  // seed and allocate the ink once
  aq_status run_stage(int stage);
  aq_status enq_pre_solve();
  aq_status enq_post_solve();
  aq_status build_graph();
  aq_status step(int nsteps);
  aq_status upload(const aq_host_state* s);
  aq_status health();  // synchronises; AQ_ERR_TIMEOUT / AQ_ERR_NONFINITE from the device's records
  aq_status download(aq_host_state* s);
  aq_status derive_from_state(const std::vector<int>& content, const std::vector<float>& divv,
                              const std::vector<float>& dens);
  int count_jacobi_launches(int sweeps) const;
  void invalidate_graph() {
    if (exec) {
      cudaGraphExecDestroy(exec);
      exec = nullptr;
    }
  }
};

namespace aqb {
// FP64 diagonal-PCG on the fluid's current pressure system (as the last
// divergence stage built it); the solution is left in f->pcg_x (device).
aq_status fluid_pcg_solve(aq_fluid* f, double rel_tol, int max_iter, int* iterations, double* achieved);
}  // namespace aqb
