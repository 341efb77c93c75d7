// Host launchers of the B200 FLIP kernels.  Each returns cudaGetLastError()
// of its launch; all work is enqueued on `st`.
#pragma once

#include <string>

#include "../../include/aquarius_b200.h"
#include "aq_common.cuh"

namespace aqb {

// Records the message aq_last_error() returns on this thread; returns st.
aq_status set_last_error(aq_status st, const std::string& msg);

// ---- particles (k_particles.cu) -------------------------------------------
// Stage (d)+(a) front half: grid-to-particle FLIP/PIC blend and RK3 advection
// (move=true) or a plain copy (move=false), written in the current order to
// the temp arrays, plus the new cell key of every particle and its slot in a
// per-cell atomic count.
cudaError_t launch_particles_advance(cudaStream_t st, const Dims& d, const StepParams& sp, bool move,
                                     Particles cur, Particles tmp, const float* u0, const float* v0,
                                     const float* w0, const float* un, const float* vn, const float* wn,
                                     const float4* nvf, int* key, int* slot, int* count, int n);
// Ink particles: G2P with FLIP coefficient 1 and RK3 advection, in place.
cudaError_t launch_ink_advance(cudaStream_t st, const Dims& d, float dt, Particles ink, const float* u0,
                               const float* v0, const float* w0, const float* un, const float* vn, const float* wn,
                               int n);
// Particle-only solvers (k_sph.cu).  Constants of one solver; dt is the
// substep's.
struct SphParams {
  float dt;
  float3 g;                 // gravity
  float md, size;           // particleSpacing / 2, gridPhysicalSize
  float kr, kr2, kr6, kr9;  // kernelRadius and its powers
  int gx, gy, gz;           // hash grid
  float s_corr_den, s_corr_k, leave;  // PBF: cubic_spline_kernel(0), 1e-6, wall leave speed
  float skip_r2;            // pairs with r^2 above it are outside both kernels' support
};
constexpr int kSphArrays = 6;
struct SphArrays {
  float4* a[kSphArrays];  // null entries are skipped
};
cudaError_t launch_sph_keys(cudaStream_t st, const SphParams& p, const float4* pos, int* key, int* slot, int* count,
                            int n);
cudaError_t launch_sph_gather(cudaStream_t st, const int* key, const int* off, const int* perm_u, const SphArrays& src,
                              const SphArrays& dst, int n);
cudaError_t launch_pbf_predict(cudaStream_t st, const SphParams& p, float4* P, const float4* L, float4* V, int n);
cudaError_t launch_pbf_lambda(cudaStream_t st, const SphParams& p, const int* off, float4* P, float4* V, float4* Q,
                              bool set_rest, int n);
cudaError_t launch_pbf_delta(cudaStream_t st, const SphParams& p, const int* off, const float4* Q, float4* P, int n);
cudaError_t launch_pbf_update(cudaStream_t st, const SphParams& p, const float4* P, float4* L, float4* V, int n);
cudaError_t launch_pci_init(cudaStream_t st, float4* W, float4* F, int n);
cudaError_t launch_pci_predict(cudaStream_t st, const SphParams& p, float4* P, float4* V, float4* Q, float4* W,
                               const float4* F, bool actual, int n);
cudaError_t launch_pci_density(cudaStream_t st, const SphParams& p, const int* off, float4* P, float4* V,
                               const float4* Q, float4* W, float4* R, bool set_rest, int n);
cudaError_t launch_pci_force(cudaStream_t st, const SphParams& p, const int* off, const float4* P, const float4* R,
                             float4* F, int n);

// Surface mesher (k_mesh.cu).  SDF grid SX*SY*SZ (cell hs), its hash grid
// HX*HY*HZ = (SX-2)*(SY-2)*(SZ-2), marching-cubes grid MX*MY*MZ (cell hm).
struct MeshDims {
  int SX, SY, SZ;
  int HX, HY, HZ;
  int MX, MY, MZ;
  float hs, hm, radius;
};
cudaError_t launch_sdf_keys(cudaStream_t st, const MeshDims& m, const float* px, const float* py, const float* pz,
                            int* skey, int* scount, int n);
cudaError_t launch_sdf_scatter(cudaStream_t st, const MeshDims& m, const Dims& d, const float* px, const float* py,
                               const float* pz, const int* off, const int* skey, const int* soff, float4* spos,
                               int* bad, int n);
cudaError_t launch_sdf(cudaStream_t st, const MeshDims& m, const int* soff, const float4* spos,
                       cudaSurfaceObject_t surf);
cudaError_t launch_mc_vertices(cudaStream_t st, const MeshDims& m, cudaTextureObject_t tex, float* vv);
cudaError_t launch_mc_flags(cudaStream_t st, const MeshDims& m, const float* vv, uint8_t* ctype, int* flag);
cudaError_t launch_mc_emit(cudaStream_t st, const MeshDims& m, cudaTextureObject_t tex, const float* vv,
                           const uint8_t* ctype, const int* moff, float* out, long long capacity);
cudaError_t launch_mc_tail(cudaStream_t st, const int* total, int* prev, float* out, long long capacity);
// Per-block FP64 sums of the particle volume fractions: part[frac_sum_parts()][4].
int frac_sum_parts();
cudaError_t launch_frac_sum(cudaStream_t st, const float4* frac, int n, double* part);
// Exclusive scan of count[0..C] into off[0..C] (off[C] = N) and clears count.
cudaError_t launch_cell_scan(cudaStream_t st, int C, int* count, int* off, int* tile_sums);
size_t cell_scan_tiles(int C);
// perm_u[off[key[i]] + slot[i]] = i
cudaError_t launch_scatter(cudaStream_t st, const int* key, const int* slot, const int* off, int* perm_u, int n);
// Stable placement: particle i goes to off[key]+#{j in its cell, j < i}.
cudaError_t launch_rank_gather(cudaStream_t st, bool multiphase, const int* key, const int* off,
                               const int* perm_u, Particles tmp, Particles cur, int* sort_index, int n);

// ---- grid (k_grid.cu) -------------------------------------------------------
// Stage (b): particle-to-grid gather onto the staggered faces, weight
// normalisation, fluid marking, density/fractions and (forces=true) gravity
// and the wall clamps of fixBoundary for nodes in [0,s)^3.
// P2G kernel: 1 (default) stages each CTA's particles in shared memory, 0 is
// one thread per node reading particles through L1.  Same sums, same order.
void set_p2g_variant(int v);
int p2g_variant();
cudaError_t launch_p2g(cudaStream_t st, const Dims& d, const StepParams& sp, bool forces, Particles cur,
                       const int* off, int n, float* u0, float* v0, float* w0, float* un, float* vn,
                       float* wn, int8_t* type, float* density, float4* vf, float4* nvf);
// Gravity and wall clamps of the nodes with a coordinate equal to s (the
// reference never resets them); reads `src` (persisted) and writes dst1/dst2.
cudaError_t launch_slayer(cudaStream_t st, const Dims& d, const StepParams& sp, const int8_t* type,
                          const float* su, const float* sv, const float* sw, float* u1, float* v1, float* w1,
                          float* u2, float* v2, float* w2);
// countParticlesInCells + computeDivergence; builds rhs = -div*rho, clears air
// pressure in both buffers (all pressure when zero_init), flags active bricks
// and writes per-block FP64 partial sums of ||b||^2 and fluid counts.
cudaError_t launch_divergence(cudaStream_t st, const Dims& d, const int* off, const int8_t* type,
                              const float* density, const float* un, const float* vn, const float* wn,
                              int* pcount, float* div, float* rhs, float* pa, float* pb, bool zero_init,
                              uint8_t* brick_active, double* part_b2, int* part_nf, int* nblocks_out);
cudaError_t launch_b2_finalize(cudaStream_t st, const double* part_b2, const int* part_nf, int nblocks,
                               SolveState* ss);
// updateVelocityWithPressure on nodes in [0,s)^3: in place on u,v,w; writes has bits.
cudaError_t launch_project(cudaStream_t st, const Dims& d, const int8_t* type, const float* p,
                           const float* density, float* u, float* v, float* w, uint8_t* has);
// One extrapolateVelocityByOne pass, reading (ui,hi) and writing (uo,ho).
cudaError_t launch_extrapolate(cudaStream_t st, const Dims& d, const float* ui, const float* vi,
                               const float* wi, const uint8_t* hi, float* uo, float* vo, float* wo,
                               uint8_t* ho);
// One diffusionJacobi sweep of the phase fractions (multiphase only).
cudaError_t launch_diffuse(cudaStream_t st, const Dims& d, const int8_t* type, float lambda,
                           const float4* fin, float4* fout);

// ---- pressure (k_jacobi.cu) -------------------------------------------------
struct JacobiPlan {
  int levels;      // sweeps per launch (1,2,4,8)
  int by;          // tile rows (y threads); 0 = flat kernel; 1 = persistent solve; 2 = cube tiles
  int xc;          // x planes per CTA (cube: tile edge in x and y)
};
// Cube plans accepted by launch_jacobi (levels, tile edge).
bool cube_plan_ok(int levels, int tx);
// List plan (by = 3): the warp rows (x, y, 128-wide z block) whose bricks hold
// fluid, listed once per solve, then one sweep per launch over the list by a
// resident wave of CTAs (sz % 4 == 0).
int row_items_capacity(const Dims& d);
cudaError_t launch_row_items(cudaStream_t st, const Dims& d, const uint8_t* brick_active, int* items, int* n_items);
cudaError_t launch_jacobi_list(cudaStream_t st, const Dims& d, const float* pin, float* pout, const float* rhs,
                               const int8_t* type, const int* items, const int* n_items,
                               bool early);

// ---- persistent solve (k_jacobi.cu) ------------------------------------------
// The whole pressure solve in one cooperative launch: every CTA sweeps its
// share of a compact list of active flat work items (1 x plane x 8 rows x 128
// z cells), a bounded grid barrier separates sweeps, and the residual check
// and stop decision are made identically by every CTA.
int persist_items(const Dims& d);
int persist_ctas(int device);  // co-resident CTAs of the cooperative launch
// Builds the ordered list of active items and clears the barrier counter.
cudaError_t launch_items_compact(cudaStream_t st, const Dims& d, const uint8_t* brick_active, int* items,
                                 int* n_items, unsigned int* bar);
// Polls of a bounded grid-barrier wait before it gives up (with 32 ns sleeps
// between polls, about a second).
constexpr unsigned kSpinLimit = 1u << 25;
// Test hook of the persistent solves' bounded waits: CTA withhold_cta (-1:
// none) leaves without arriving at any barrier, and the others give up after
// spin_limit polls (0: kSpinLimit).  Either way the solve ends with
// SolveState::sync_timeout set and no CTA left waiting.
struct BarrierTest {
  int withhold_cta;
  unsigned spin_limit;
};
// ---- resident solve (k_resident.cu) ------------------------------------------
// Plan rows = 4: the whole solve in one cooperative launch, one CTA per SM;
// a CTA keeps a tile (plan.xc selects the TX x TY x TZ shape) plus a K-cell
// halo (K = plan.levels, 4) in shared memory for the whole solve and
// exchanges halos through L2 every K sweeps.  Bit for bit the flat sweep.
bool resident_plan_ok(int shape, int k);
int resident_tile_capacity(const Dims& d);        // tile-list entries any shape needs
int resident_ctas(int device, int shape, int k);  // CTAs of the launch (0: shape unusable)
long long resident_cells_updated(const Dims& d, int shape, const uint8_t* bact_host);
// Builds the tile list (and clears the barrier counter), then solves:
// fixed_sweeps > 0: that many sweeps then one residual; else residual mode
// (check every `check` sweeps, stop at tol or max_iters).  Result in pa.
cudaError_t launch_resident_solve(cudaStream_t st, const Dims& d, int shape, int k, int ctas, float* pa, float* pb,
                                  const float* rhs, const int8_t* type, const uint8_t* bact, int* tiles,
                                  int* n_tiles, unsigned int* bar, double* part, SolveState* ss, int fixed_sweeps,
                                  int check, int max_iters, double tol, BarrierTest bt);
// Counts the float bit patterns where the resident sweep's division by 6
// differs from the IEEE divide (*bad must start at 0).
cudaError_t launch_div6_check(cudaStream_t st, unsigned long long* bad);
// fixed_sweeps > 0: that many sweeps then one residual; else residual mode.
cudaError_t launch_persist_solve(cudaStream_t st, const Dims& d, int ctas, float* pa, float* pb, const float* rhs,
                                 const int8_t* type, const int* items, const int* n_items, unsigned int* bar,
                                 double* part, SolveState* ss, int fixed_sweeps, int check, int max_iters, double tol,
                                 BarrierTest bt);
// Temporally blocked Jacobi: `levels` sweeps from pin to pout; with resid it
// also writes per-CTA FP64 partial sums of ||b - A p_out||^2 to part.
cudaError_t launch_jacobi(cudaStream_t st, const Dims& d, const JacobiPlan& plan, bool resid,
                          const float* pin, float* pout, const float* rhs, const int8_t* type,
                          const uint8_t* brick_active, double* part, int* nparts_out);
int jacobi_parts(const Dims& d, const JacobiPlan& plan, bool resid);
// Cells in the output regions of the tiles a sweep does not skip.
long long jacobi_cells_updated(const Dims& d, const JacobiPlan& plan, const uint8_t* bact_host);
// Sets the dynamic shared-memory limits of every Jacobi variant (call before capture).
cudaError_t jacobi_prepare();
// FP64 ||b - A p||^2 partial sums of one iterate (flat layout; sz % 4 == 0).
cudaError_t launch_resid_flat(cudaStream_t st, const Dims& d, const float* p, const float* rhs, const int8_t* type,
                              const uint8_t* brick_active, double* part);
int resid_flat_parts(const Dims& d);
// Sums residual partials; updates ss; in a conditional loop body it also
// sets the loop's condition (continue while not converged and under cap).
// The flat residual pass and the residual check in one launch (a last-block
// ticket; ticket starts at 0 and is left at 0).
cudaError_t launch_resid_flat_fin(cudaStream_t st, const Dims& d, const float* p, const float* rhs,
                                  const int8_t* type, const uint8_t* brick_active, double* part, unsigned int* ticket,
                                  SolveState* ss, int sweeps, double tol, int max_iters, bool set_cond,
                                  unsigned long long cond_handle);
// The same for the list plan: residual of the listed rows, per-CTA partials
// (at most row_items_capacity / 8 of them).
cudaError_t launch_resid_list_fin(cudaStream_t st, const Dims& d, const float* p, const float* rhs,
                                  const int8_t* type, const int* items, const int* n_items, double* part,
                                  unsigned int* ticket, SolveState* ss, int sweeps, double tol, int max_iters,
                                  bool set_cond, unsigned long long cond_handle);
cudaError_t launch_resid_finalize(cudaStream_t st, const double* part, int nparts, SolveState* ss,
                                  int sweeps_done_per_call, double tol, int max_iters,
                                  bool set_cond, unsigned long long cond_handle);

// ---- batched scenes ------------------------------------------------------------
// CTAs of `kernel` (with `threads` per CTA) resident on the current device at once.
template <typename K>
inline int resident_ctas(K kernel, int threads, size_t smem = 0) {
  int dev = 0, sms = 0, occ = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kernel, threads, smem);
  return sms * (occ > 0 ? occ : 1);
}
// Grid of a grid-stride batched launch: one resident wave at most, capped by
// the caller's limit and by the work.
template <typename K>
inline int batch_grid(K kernel, int threads, int cap, int total) {
  int g = resident_ctas(kernel, threads);
  if (cap < g) g = cap;
  if (total < g) g = total;
  return g > 0 ? g : 1;
}

// Each launcher runs one stage for every scene of a batch: `total` virtual
// blocks (the last prefix sum of the stage's family in BatchIndex) walked by
// `grid` CTAs.  A virtual block runs the single-scene kernel's body on its
// scene's slice of the concatenated arrays, so a scene's result does not
// depend on the other scenes.  Single-phase scenes only.
cudaError_t launch_batch_particles_advance(cudaStream_t st, const BatchIndex& bi, int total, int grid, bool move,
                                           Particles cur, Particles tmp, const float* u0, const float* v0,
                                           const float* w0, const float* un, const float* vn, const float* wn,
                                           int* key, int* slot, int* count);
cudaError_t launch_batch_p2g(cudaStream_t st, const BatchIndex& bi, int total, int grid, bool forces, Particles cur,
                             const int* off, float* u0, float* v0, float* w0, float* un, float* vn, float* wn,
                             int8_t* type, float* density);
cudaError_t launch_batch_slayer(cudaStream_t st, const BatchIndex& bi, int total, int grid, const int8_t* type,
                                const float* su, const float* sv, const float* sw, float* u1, float* v1, float* w1,
                                float* u2, float* v2, float* w2);
cudaError_t launch_batch_divergence(cudaStream_t st, const BatchIndex& bi, int total, int grid, const int* off,
                                    const int8_t* type, const float* density, const float* un, const float* vn,
                                    const float* wn, int* pcount, float* div, float* rhs, float* pa, float* pb,
                                    bool zero_init, uint8_t* brick_active, double* part_b2, int* part_nf);
// One CTA per scene: ||b||^2 and fluid count; sets live[s] = 1.
cudaError_t launch_batch_b2_finalize(cudaStream_t st, const BatchIndex& bi, const double* part_b2, const int* part_nf,
                                     SolveState* ss, int* live);
cudaError_t launch_batch_project(cudaStream_t st, const BatchIndex& bi, int total, int grid, const int8_t* type,
                                 const float* p, const float* density, float* u, float* v, float* w, uint8_t* has);
cudaError_t launch_batch_extrapolate(cudaStream_t st, const BatchIndex& bi, int total, int grid, const float* ui,
                                     const float* vi, const float* wi, const uint8_t* hi, float* uo, float* vo,
                                     float* wo, uint8_t* ho);
// One Jacobi sweep of every scene with live[s] != 0 (sz % 4 == 0), packed
// rows: a warp item is xs x planes x 32/min(sz/4,32) rows x up to 128 z cells;
// bi.rows must hold the prefix sums of batch_row_items(d, xs).
int batch_row_items(const Dims& d, int xs);
// Cells the packed-row sweep writes (items with an active brick).
long long batch_row_cells_updated(const Dims& d, int xs, const uint8_t* bact_host);
// pipelined (xs > 1): plane x+1's loads are issued before plane x's arithmetic.
// list (may be NULL): the active (scene, item) pairs from launch_batch_row_list.
cudaError_t launch_batch_jacobi_rows(cudaStream_t st, const BatchIndex& bi, int total, int xs, bool pipelined,
                                     int grid, const int* live, const float* pin, float* pout, const float* rhs,
                                     const int8_t* type, const uint8_t* brick_active, const int2* list,
                                     const int* n_list);
// The (scene, local item) pairs whose bricks hold fluid (capacity: total).
cudaError_t launch_batch_row_list(cudaStream_t st, const BatchIndex& bi, int total, int xs,
                                  const uint8_t* brick_active, int2* list, int* n_list);
cudaError_t launch_batch_resid_flat(cudaStream_t st, const BatchIndex& bi, int total, int grid, const int* live,
                                    const float* p, const float* rhs, const int8_t* type,
                                    const uint8_t* brick_active, double* part);
// Per live scene: residual, stop decision (live[s] = continue).
cudaError_t launch_batch_resid_finalize(cudaStream_t st, const BatchIndex& bi, const double* part, SolveState* ss,
                                        int* live, int sweeps, double tol, int max_iters);
// Loop condition of the batched solve: any scene still live.
cudaError_t launch_batch_solve_condition(cudaStream_t st, const int* live, int n_scenes,
                                         unsigned long long cond_handle);

// ---- U-Net building blocks (k_unet.cu) ---------------------------------------
// Channels-last bf16 tensors over a grid; 3x3x3 convolution, zero padding.
// (cin, cout) must be one of the instantiated pairs (else cudaErrorInvalidValue).
cudaError_t launch_conv3_fwd(cudaStream_t st, int cin, int cout, bool relu, const void* in, const void* w,
                             const float* bias, void* out, int sx, int sy, int sz);
// dw[t][co][ci] (f32) from x (cin) and dy (cout); part: conv3_wgrad_part_floats scratch.
cudaError_t launch_conv3_wgrad(cudaStream_t st, int cin, int cout, const void* x, const void* dy, float* part,
                               float* dw, int sx, int sy, int sz);
size_t conv3_wgrad_part_floats(int cin, int cout, int voxels);
// Forward kernel variant: halo-tiled (true, default) or im2col streaming.
// 2 = tcgen05 UMMA where it fits (default), 1 = halo-tiled mma.sync, 0 = im2col mma.sync.
void set_conv_impl(int impl);
// Nonzero if a tcgen05 convolution ever gave up waiting on its mbarriers.
int conv_umma_timeouts();
// Test hook: skip != 0 makes every tcgen05 convolution issue no MMA, so its
// bounded wait runs out after wait_ns (0 = the default second); also clears
// the timeout record.
cudaError_t conv_umma_test_hook(int skip, unsigned long long wait_ns);
// wt[t][ci][co] = w[26-t][co][ci] (weights of the data gradient).
cudaError_t launch_flip_transpose(cudaStream_t st, const void* w, void* wt, int cin, int cout);

// U-Net glue (channels-last bf16, fine grid sx,sy,sz even; coarse = half).
cudaError_t launch_absmax(cudaStream_t st, const float* a, int n, float* part /*>= 1024*/, float* out);
cudaError_t launch_unet_input(cudaStream_t st, const float* rhs, const int8_t* type, const float* scale, void* out,
                              int V);
cudaError_t launch_pool2(cudaStream_t st, const void* in, void* out, int sx, int sy, int sz, int C);
cudaError_t launch_pool2_bwd(cudaStream_t st, const void* dout, void* din, int sx, int sy, int sz, int C,
                             bool accumulate);
cudaError_t launch_upcat(cudaStream_t st, const void* coarse, const void* skip, void* out, int sx, int sy, int sz,
                         int Cu, int Cs);
cudaError_t launch_upcat_bwd(cudaStream_t st, const void* dout, void* dcoarse, void* dskip, int sx, int sy, int sz,
                             int Cu, int Cs);
cudaError_t launch_relu_bwd(cudaStream_t st, void* dy, const void* y, int n);
int chan_sum_parts(int V);
cudaError_t launch_chan_sum(cudaStream_t st, const void* dy, int V, int C, float* part, float* out);
cudaError_t launch_head_fwd(cudaStream_t st, const void* h, const float* w, const float* b, float* out, int V);
// Training loss L = ||e||^2/||t||^2 + alpha ||A J^k e||^2/||A J^k t||^2 (fluid
// cells, e = out - target, J a homogeneous Jacobi sweep, A the pressure
// operator) and the head's backward pass: dh, head_sums = [dw 16, db, loss].
// Scratch: e, p0..p3, g (V floats each), part (loss_parts() * 8), sums (6),
// head_part (loss_parts() * 17).
int loss_parts();
cudaError_t launch_unet_loss_bwd(cudaStream_t st, const float* out, const float* target, const int8_t* type,
                                 const void* h, const float* w, float alpha, int k, void* dh, int sx, int sy, int sz,
                                 float* e, float* p0, float* p1, float* p2, float* p3, float* g, float* part,
                                 float* sums, float* head_part, float* head_sums);
cudaError_t launch_adam(cudaStream_t st, float* w, const float* g, float* m, float* v, int n, float lr, float b1,
                        float b2, float eps, int t, void* wb);
cudaError_t launch_f32_to_bf16(cudaStream_t st, const float* a, void* b, int n);
cudaError_t launch_unet_to_pressure(cudaStream_t st, const float* out, const float* scale, float out_scale,
                                    const int8_t* type, float* p, int V);
cudaError_t launch_unet_scale_copy(cudaStream_t st, const float* a, float k, float* b, int n);
cudaError_t launch_unet_sample(cudaStream_t st, const float* rhs, const int8_t* type, const double* p,
                               const float* scale, float* rhs_s, int8_t* type_s, float* target, int V);

// ---- FP64 PCG (k_pcg.cu) ----------------------------------------------------
cudaError_t launch_pcg_apply(cudaStream_t st, const Dims& d, const int8_t* type, const double* in,
                             double* out);  // out = A in
cudaError_t launch_pcg_dot(cudaStream_t st, int C, const double* a, const double* b, double* part,
                           int nparts);
cudaError_t launch_pcg_axpy(cudaStream_t st, int C, double alpha, const double* xv, double* yv);
cudaError_t launch_pcg_precond(cudaStream_t st, const Dims& d, const int8_t* type, const double* r,
                               double* z);
cudaError_t launch_pcg_xpby(cudaStream_t st, int C, const double* xv, double beta, double* yv);
cudaError_t launch_pcg_init(cudaStream_t st, const Dims& d, const int8_t* type, const float* rhs,
                            double* b, double* x);


// ------------------------------------------------------------ headless frame
constexpr int kRenderTile = 16;  // screen tile edge in pixels (one CTA per tile; triangle lists)
constexpr int kSpriteTile = 8;   // point-sprite lists are kept per 8x8 pixels

struct RenderParams {
  int W, H, tiles_x, tiles_y;
  int stiles_x, stiles_y;  // 8x8 sprite tiles
  int mode, env, use_phase;
  float pv[16];    // projection * view (column-major)
  float view[16];
  float proj[16];
  float model[16]; // container model
  float cmvp[16];  // (projection * view) * container model
  int ntri_container;
  float cam[3], light[3];
  float container, cornell;
  float radius, tan_half;
  int phase_count;
  float phase_colors[16];
  const uint8_t* sky;
  int face;
  const uint8_t* logo;
  int lw, lh;
};

// A triangle in window space, counter-clockwise: vertices snapped to 1/256
// pixel, window depth, 1/w and 8 varyings per vertex (world position, ndc xy,
// normal), twice the area in 1/256^2 units, top-left flags of its edges.
struct RenderTri {
  int X[3], Y[3];
  float z[3], iw[3];
  float a[3][8];
  long long area;
  int tl;
};

cudaError_t launch_sprite_setup(cudaStream_t st, const RenderParams& P, const float* pts, int n, float4* spr,
                                float4* frac, int* cnt, unsigned long long* total);
cudaError_t launch_sprite_emit(cudaStream_t st, const RenderParams& P, const float4* spr, const int* off, int n,
                               unsigned* keys, int* vals);
cudaError_t launch_tri_setup(cudaStream_t st, const RenderParams& P, const float* mesh, int ntri, RenderTri* tris,
                             int* cnt, unsigned long long* total);
cudaError_t launch_tri_emit(cudaStream_t st, const RenderParams& P, const RenderTri* tris, const int* off, int ntri,
                            unsigned* keys, int* vals);
cudaError_t launch_container_setup(cudaStream_t st, const RenderParams& P, RenderTri* tris, int* live);
// Stable LSD radix sort (k_sort.cu) of n (key, value) pairs by the low `bits`
// bits of the keys, ascending (or descending) into (k1, v1); (k0, v0) is left
// as it was.  tmp: radix_sort_temp_ints(n) ints of scratch.
size_t radix_sort_temp_ints(int n);
cudaError_t radix_sort_pairs(cudaStream_t st, const unsigned* k0, const int* v0, unsigned* k1, int* v1, int n,
                             int bits, bool descending, int* tmp);
// range[key] = [first, last+1) of each key's run in sorted keys[0..n)
cudaError_t launch_tile_ranges(cudaStream_t st, const unsigned* keys, int n, int2* range);
// The phase-thickness pass over the 8x8 sprite tiles, in the given order.
cudaError_t launch_phase(cudaStream_t st, const RenderParams& P, const int2* range, const int* order,
                         const int* vals, const float4* spr, const float4* frac, float4* phase);
// load[t] = list length of sprite tile t, ids[t] = t
cudaError_t launch_tile_load(cudaStream_t st, const int2* range, int n, unsigned* load, int* ids);
cudaError_t launch_frame(cudaStream_t st, const RenderParams& P, const RenderTri* ctris, const int* clive,
                         const int2* trange, const int* tvals, const RenderTri* tris, const int2* srange,
                         const int* svals, const float4* spr, const float4* phase, uchar4* rgba);
cudaError_t launch_points_vbo(cudaStream_t st, Particles cur, int n, int phase, float* vbo);

}  // namespace aqb
