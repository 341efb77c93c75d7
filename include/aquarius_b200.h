/*
 * aquarius_b200 — C ABI of the B200-native 3D FLIP step.
 *
 * This is the drop-in boundary for the reference solver plugin
 * (AmesingFlank/Aquarius).  Each entry point below replaces one piece of the
 * reference's `Fluid` / `Fluid_3D_FLIP::Fluid` surface:
 *
 *   reference                                           replacement
 *   -------------------------------------------------   ------------------------------
 *   FluidConfig / ConfigFLIP / InitializationVolume      aq_config / aq_volume
 *     (Fluid/FluidConfig.cuh:16-97)
 *   make_shared<Fluid_3D_FLIP::Fluid>() + init(config)   aq_fluid_create
 *     (main.cu:158-170, Fluid/Fluid_3D_FLIP.cu:435-505)
 *   Fluid::simulationStep() (Fluid/Fluid_3D_FLIP.cu:316)  aq_fluid_step
 *   Fluid::physicalTime (Fluid/Fluid.h:10)               aq_fluid_time
 *   Fluid_3D::getCenter / getContainerSize               aq_fluid_container
 *     (Fluid/Fluid_3D.cuh:7-12, Fluid/Fluid_3D_FLIP.cu:728-733)
 *   public members particles / grid->volumes / cellStart aq_fluid_download_state /
 *     / cellEnd (Fluid/Fluid_3D_FLIP.cuh:54-111)           aq_fluid_upload_state
 *   ~Fluid() (Fluid/Fluid_3D_FLIP.cu:735-748)            aq_fluid_destroy
 *   print + exit(EXIT_FAILURE) (Common/GpuCommons.h:118)  aq_status + aq_last_error
 *
 * No entry point takes or returns a framework type: plain pointers, sizes and
 * POD structs only.  Every call returns an aq_status; nothing exits or throws
 * across the boundary.
 */
#ifndef AQUARIUS_B200_H
#define AQUARIUS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define AQ_ABI_VERSION 1
#define AQ_MAX_VOLUMES 16
#define AQ_MAX_PHASES 4

/* Status codes.  The reference prints and calls exit() on any CUDA error
 * (Common/GpuCommons.h:118-142) and throws a const char* for phaseCount > 4
 * (Fluid/Fluid_3D_FLIP.cu:449-451); here both become return codes. */
typedef enum aq_status {
  AQ_OK = 0,
  AQ_ERR_INVALID_CONFIG = 1,
  AQ_ERR_INVALID_ARGUMENT = 2,
  AQ_ERR_OUT_OF_MEMORY = 3,
  AQ_ERR_CUDA = 4,
  AQ_ERR_NOT_CONVERGED = 5,
  AQ_ERR_NONFINITE = 6,
  AQ_ERR_NO_DEVICE = 7,
  AQ_ERR_TIMEOUT = 8
} aq_status;

/* ShapeType {Sphere, Square} (Fluid/FluidConfig.cuh:16-18). */
typedef enum aq_shape { AQ_SHAPE_SPHERE = 0, AQ_SHAPE_SQUARE = 1 } aq_shape;

/* Pressure initial guess for each step's solve.
 * CARRY: the reference behaviour — pressure persists across steps (it is only
 *        cleared when the grid is created, Fluid/MAC_Grid_3D.cu:54).
 * ZERO:  pressure is zeroed before every solve.
 * LEARNED: pressure is zeroed, then the warm-start network attached with
 *        aq_fluid_set_warm_start predicts it; 20 sweeps are run from the
 *        prediction and 20 from zero, and the solve continues from whichever
 *        has the lower residual (zero-init Jacobi is the fallback and the
 *        judge).  Needs sizes divisible by 4.  No counterpart in the reference. */
typedef enum aq_pressure_init {
  AQ_PRESSURE_CARRY = 0,
  AQ_PRESSURE_ZERO = 1,
  AQ_PRESSURE_LEARNED = 2
} aq_pressure_init;

/* FIXED: exactly pressure_iterations Jacobi sweeps (Fluid/Fluid_3D_common.cu:48-55).
 * RESIDUAL: sweep in blocks of check_interval until the relative residual
 *           ||b - A p||_2 / ||b||_2 over fluid cells (FP64) is <= rel_residual,
 *           or max_iterations sweeps were done.  No counterpart in the reference. */
typedef enum aq_solve_mode { AQ_SOLVE_FIXED = 0, AQ_SOLVE_RESIDUAL = 1 } aq_solve_mode;

/* InitializationVolume (Fluid/FluidConfig.cuh:20-38).  Coordinates are the
 * reference's normalised [0,1] container coordinates; ball_radius is in units
 * of the container's y extent. */
typedef struct aq_volume {
  int32_t shape;
  float box_min[3];
  float box_max[3];
  float ball_center[3];
  float ball_radius;
  int32_t phase;
} aq_volume;

/* POD mirror of FluidConfig + ConfigFLIP (Fluid/FluidConfig.cuh:41-97),
 * fixed-size so it crosses a C boundary.  aq_config_default() fills the
 * reference defaults. */
typedef struct aq_config {
  /* FluidConfig */
  int32_t volume_count;
  aq_volume volumes[AQ_MAX_VOLUMES];
  float gravity[3];
  int32_t phase_count;
  float phase_densities[4];
  float diffusion_coeff;
  /* ConfigFLIP */
  int32_t size_x, size_y, size_z;
  int32_t pressure_iterations;
  int32_t diffusion_iterations;
  float timestep;
  float flip_coeff;
  float particle_jitter;
  /* Fluid_3D_FLIP::Fluid::gridPhysicalSize (Fluid/Fluid_3D_FLIP.cuh:62) */
  float domain_size;
  /* Seed of the glibc rand() sequence used for particle jitter.  The
   * reference never calls srand(), which is the same sequence as seed 1. */
  uint32_t seed;
  /* Extensions with no counterpart in the reference. */
  int32_t pressure_init;   /* aq_pressure_init */
  int32_t solve_mode;      /* aq_solve_mode */
  float rel_residual;      /* RESIDUAL mode target, e.g. 1e-4 */
  int32_t max_iterations;  /* RESIDUAL mode cap, e.g. 2000 */
  int32_t check_interval;  /* RESIDUAL mode: sweeps between residual checks */
  int32_t device;          /* CUDA device ordinal */
  void* stream;            /* cudaStream_t to run on; NULL = library-owned stream */
} aq_config;

/* Host-side copy of the simulation state in one canonical layout.
 *   cells  (C = sx*sy*sz):          index (x*sy + y)*sz + z
 *   nodes  (F = (sx+1)(sy+1)(sz+1)): index (x*(sy+1) + y)*(sz+1) + z
 * Velocity node (x,y,z) holds u on the x-face at (x, y+1/2, z+1/2)h, v on the
 * y-face at (x+1/2, y, z+1/2)h and w on the z-face at (x+1/2, y+1/2, z)h
 * (Fluid/MAC_Grid_3D.cuh:100-130).  Multi-component fields are planar:
 * component k of element i is at [k*count + i].
 * Any pointer may be NULL, in which case that field is skipped. */
typedef struct aq_host_state {
  int32_t size_x, size_y, size_z;  /* must match the fluid */
  int32_t particle_count;          /* must match the fluid */
  double physical_time;
  float* position;          /* [3][N] */
  float* velocity_p;        /* [3][N] particle velocity */
  float* fractions;         /* [4][N] particle volume fractions */
  int32_t* content;         /* [F]   0 air, 1 fluid, 2 solid */
  float* velocity;          /* [3][F] grid velocity after the particle->grid transfer */
  float* new_velocity;      /* [3][F] grid velocity after forces, pressure, extrapolation */
  float* pressure;          /* [C] */
  float* divergence;        /* [C] */
  int32_t* particle_count_cell; /* [C] cellEnd - cellStart, as the reference stores it */
  int32_t* has_velocity;    /* [3][C] 0/1 */
  float* volume_fractions;  /* [4][C] */
  float* new_volume_fractions; /* [4][C] */
  float* density;           /* [C] */
  int32_t* cell_start;      /* [C] first sorted particle of the cell, -1 if empty */
  int32_t* cell_end;        /* [C] last sorted particle of the cell (inclusive), -1 if empty */
  int32_t* particle_hash;   /* [N] cell index of each (sorted) particle */
  int32_t* sort_index;      /* [N] pre-sort index of each sorted particle (particleIndices) */
} aq_host_state;

/* Sub-stages of one simulationStep, in order (Fluid/Fluid_3D_FLIP.cu:316-352).
 * A full step runs 1..8 and advances physical time. */
typedef enum aq_stage {
  AQ_STAGE_G2P_ADVECT = 1,  /* transferToParticles + moveParticles */
  AQ_STAGE_SORT = 2,        /* performSpatialHashing2 (hash, stable sort, cell tables) */
  AQ_STAGE_P2G = 3,         /* resetCell + P2G + divide + fractions + applyGravity + fixBoundary */
  AQ_STAGE_DIVERGENCE = 4,  /* countParticlesInCells + computeDivergence */
  AQ_STAGE_PRESSURE = 5,    /* solvePressureJacobi */
  AQ_STAGE_PROJECT = 6,     /* updateVelocityWithPressure */
  AQ_STAGE_EXTRAPOLATE = 7, /* extrapolateVelocity (3 passes) */
  AQ_STAGE_DIFFUSE = 8      /* solveDiffusionJacobi */
} aq_stage;

typedef struct aq_fluid aq_fluid;

/* Statistics of the most recent pressure solve. */
typedef struct aq_solve_stats {
  int32_t iterations;       /* Jacobi sweeps done */
  double rel_residual;      /* ||b - A p|| / ||b|| over fluid cells, FP64; -1 if not computed */
  double b_norm;            /* ||b||_2 */
  int32_t fluid_cells;
  int32_t converged;        /* RESIDUAL mode: 1 if rel_residual <= target */
  int32_t blocks;           /* residual-check blocks of the last solve */
  int64_t total_sweeps;     /* sweeps since creation */
  int64_t total_blocks;     /* residual-check blocks since creation */
  /* AQ_PRESSURE_LEARNED: 1 the network's prediction was kept, 2 the zero-init
   * fallback won, 0 no warm start this solve; the two relative residuals
   * after the first 20 sweeps (-1 if not run). */
  int32_t warm_start;
  double warm_rel_residual;
  double zero_rel_residual;
} aq_solve_stats;

/* Fills *cfg with the reference defaults (Fluid/FluidConfig.cuh:20-97):
 * 50^3, 100 Jacobi and 100 diffusion iterations, dt 0.033, FLIP 0.95,
 * jitter 0.05, gravity (0,-9.8,0), 2 phases, densities 1, D 0.001, a box
 * (0,0,0)-(1,0.1875,1) and a ball at (0.5,0.75,0.5) r 0.125, domain 10. */
aq_status aq_config_default(aq_config* cfg);

/* Validates cfg without touching the GPU. */
aq_status aq_config_validate(const aq_config* cfg);

/* Creates the solver and runs Fluid::init: grid allocation, particle seeding,
 * boundary marking and the first particle->grid transfer. */
aq_status aq_fluid_create(const aq_config* cfg, aq_fluid** out);

/* Runs n_steps simulationStep()s.  Asynchronous on the fluid's stream. */
aq_status aq_fluid_step(aq_fluid* f, int32_t n_steps);

/* Host-buffer step, for callers that keep the particle state in host memory:
 * uploads position_in/velocity_in ([3][N] each, may be NULL to keep the device
 * copy), runs n_steps, downloads position_out/velocity_out ([3][N], may be
 * NULL) and synchronizes.  Pinned buffers make the copies asynchronous.
 * Returns what aq_fluid_synchronize returns after the steps. */
aq_status aq_fluid_step_host(aq_fluid* f, int32_t n_steps,
                             const float* position_in, const float* velocity_in,
                             float* position_out, float* velocity_out);

/* use_graph = 1 (default): a step is one CUDA-graph launch.  0: the step's
 * kernels are launched one by one (RESIDUAL mode then reads the residual on
 * the host after each check block); same kernels, same results, used to
 * profile individual launches. */
aq_status aq_fluid_set_graph_mode(aq_fluid* f, int32_t use_graph);

/* Runs one sub-stage (aq_stage) of a step; used to compare stages in
 * isolation.  AQ_STAGE_DIFFUSE also advances physical time, as the last
 * statement of simulationStep does. */
aq_status aq_fluid_run_stage(aq_fluid* f, int32_t stage);

/* Waits for all work of the fluid, then reports what the device recorded
 * while stepping (a step itself is asynchronous and returns before its
 * kernels run):
 *   AQ_ERR_TIMEOUT    a bounded device wait of a persistent pressure solve
 *                     gave up (its grid barrier);
 *   AQ_ERR_NONFINITE  some step since creation or the last
 *                     aq_fluid_upload_state had a non-finite divergence norm
 *                     ||b|| or pressure residual (a NaN or Inf in the state).
 * Both are sticky until the next aq_fluid_upload_state. */
aq_status aq_fluid_synchronize(aq_fluid* f);

aq_status aq_fluid_time(const aq_fluid* f, double* physical_time);
aq_status aq_fluid_particle_count(const aq_fluid* f, int32_t* n);
/* center[3] and the container size, as Fluid_3D::getCenter/getContainerSize. */
aq_status aq_fluid_container(const aq_fluid* f, float center[3], float* size);
/* The cudaStream_t the fluid runs on. */
aq_status aq_fluid_stream(const aq_fluid* f, void** stream);

aq_status aq_fluid_download_state(aq_fluid* f, aq_host_state* s);
aq_status aq_fluid_upload_state(aq_fluid* f, const aq_host_state* s);

/* Fills *st (synchronising), then returns AQ_ERR_TIMEOUT if the last solve's
 * grid barrier gave up, AQ_ERR_NONFINITE if its residual is not finite, and
 * AQ_ERR_NOT_CONVERGED in AQ_SOLVE_RESIDUAL mode when it stopped at
 * max_iterations above rel_residual (st then holds the achieved residual);
 * otherwise AQ_OK. */
aq_status aq_fluid_solve_stats(const aq_fluid* f, aq_solve_stats* st);

/* Test hook of the bounded device waits (no counterpart in the reference):
 * from the next step on, the persistent pressure solves (Jacobi plans rows 1
 * and 4) run with CTA withhold_cta (-1: none) leaving without ever arriving
 * at a grid barrier, and the other CTAs giving up after spin_limit polls
 * (0: the default, about a second).  The solve then ends early with
 * aq_fluid_synchronize returning AQ_ERR_TIMEOUT, and the device stays usable.
 * Call with (-1, 0) to switch it off. */
aq_status aq_fluid_test_barrier_timeout(aq_fluid* f, int32_t withhold_cta, uint32_t spin_limit);

/* Particle-to-grid kernel, process-wide (set it while no step is in flight):
 * 1 (default), 2, 3 stage each CTA's particles in shared memory (cell-major
 * slots, conflict-free gathers) with 11, 7 or 16 slots per cell (particles
 * beyond them are read from global memory); 0 gathers through L1 with one
 * thread per node.  Both sum the same terms in the reference's (dx, dy, dz, j) order
 * (transferToCellAccumPhase, Fluid/Fluid_3D_FLIP.cu:8-70). */
aq_status aq_p2g_set_variant(int32_t variant);

/* Self-check of the resident solve's division by 6 (an FMA-corrected
 * reciprocal product on normal quotients) against the IEEE divide over all
 * 2^32 float bit patterns on `device`; *mismatches receives the count of
 * differing results (NaN equal to NaN).  No counterpart in the reference. */
aq_status aq_selfcheck_division(int32_t device, uint64_t* mismatches);

/* Plan of the Jacobi kernels.  rows = 0: one vectorised sweep per launch
 * (levels 1, x_planes in {1,2,4,8} planes per block; sz % 4 == 0).
 * rows = 1: the whole solve in one persistent cooperative launch with a
 * grid barrier between sweeps (levels 1; sz % 4 == 0).  rows = 3: one sweep
 * per launch over a list of the warp rows that hold fluid (levels 1,
 * x_planes 1; sz % 4 == 0).  rows = 4: the whole solve in one cooperative
 * launch of resident tiles: each CTA keeps a tile of the grid (x_planes
 * selects the shape: 0 8x40x24, 1 16x24x24, 2 8x32x24, 3 16x16x24,
 * 4 8x16x24, 5 24x16x24 cells, 6 8x40x24 with twice the threads) with a
 * `levels`-cell halo (4) in
 * shared memory for the whole solve and exchanges halos every `levels`
 * sweeps (sz % 4 == 0).  rows = 8, 16, 32:
 * the temporally blocked kernel with `levels` sweeps (1, 2, 4, 8) per launch
 * over tiles of that many rows and x_planes planes.  Chosen per grid by the
 * tuner; invalid plans are rejected. */
aq_status aq_fluid_set_jacobi_plan(aq_fluid* f, int32_t levels, int32_t rows, int32_t x_planes);
aq_status aq_fluid_get_jacobi_plan(const aq_fluid* f, int32_t* levels, int32_t* rows, int32_t* x_planes);

/* Result of aq_fluid_autotune: the chosen plan and its measured sweep time. */
typedef struct aq_tune_result {
  int32_t levels, rows, x_planes;
  float sweep_us;           /* graph-timed wall time per sweep of the chosen plan */
  int32_t candidates;       /* plans timed (0 when taken from the cache) */
  int32_t from_cache;
} aq_tune_result;

/* Project-written autotuner of the Jacobi plan.  Times every candidate plan
 * (flat with 1 or 2 planes per block, persistent cooperative, temporally
 * blocked shapes) on the fluid's current pressure system with graph-replayed
 * sweeps, keeps the fastest and sets it.  Needs a system with fluid, i.e.
 * call after at least one step; it advances the pressure iterate.
 * cache_path (may be NULL): a JSON file keyed by GPU name and grid size; a
 * hit sets the cached plan without timing, a miss appends the new choice. */
aq_status aq_fluid_autotune(aq_fluid* f, int32_t sweeps_per_trial, const char* cache_path, aq_tune_result* out);

/* FP64 preconditioned conjugate gradient on the current pressure system
 * (the one the last AQ_STAGE_DIVERGENCE built), to rel_tol.  Writes the FP64
 * solution as float into pressure_out ([C], host, may be NULL) and reports
 * the relative L2 error of the fluid's current pressure against it over
 * fluid cells.  Not part of a step; used to state pressure error. */
aq_status aq_fluid_pcg_reference(aq_fluid* f, double rel_tol, int32_t max_iter,
                                 float* pressure_out, double* rel_error,
                                 int32_t* iterations, double* achieved_residual);

/* Per-stage device times (ms) of one eagerly launched step; stage_ms[k-1]
 * receives stage k (aq_stage).  Advances the simulation by one step. */
aq_status aq_fluid_profile_step(aq_fluid* f, float stage_ms[8]);

/* Kernel launches of the last step (graph nodes included; in RESIDUAL mode
 * this depends on the residual-check blocks the last solve ran). */
aq_status aq_fluid_launches_per_step(const aq_fluid* f, int32_t* launches);
/* Kernel launches of a step outside the residual loop, and per loop block. */
aq_status aq_fluid_launch_counts(const aq_fluid* f, int32_t* per_step, int32_t* per_block);

/* Times `sweeps` Jacobi sweeps of the current pressure system on the fluid's
 * stream: the launches are captured into a CUDA graph, replayed once to warm
 * up and once between CUDA events (advances the pressure iterate twice).
 * Reports the elapsed ms, the number of launches and the cells each sweep
 * updates (cells of the tiles that hold fluid; the rest stay 0 untouched). */
aq_status aq_fluid_benchmark_pressure(aq_fluid* f, int32_t sweeps, float* ms, int32_t* launches,
                                      int64_t* cells_per_sweep);

void aq_fluid_destroy(aq_fluid* f);

/* ---- Batches of independent scenes ------------------------------------------
 * No counterpart in the reference (it simulates one scene per process).  A
 * batch steps many independent single-phase scenes, each with its own grid
 * size, volumes and seed, in one CUDA graph per step: every stage is one
 * launch over all scenes, and the pressure solve sweeps only the scenes whose
 * solve is still running.  Scene s evolves exactly as an aq_fluid created
 * from configs[s] with the default Jacobi plan would (bit for bit).
 *
 * Requirements: every config valid; size_z % 4 == 0; the same pressure
 * solver settings (pressure_iterations, pressure_init, solve_mode,
 * rel_residual, max_iterations, check_interval), device and stream in every
 * config; in AQ_SOLVE_RESIDUAL mode an even check_interval; every scene
 * single-phase (all its volumes carry one phase).  Totals must fit 32-bit
 * indices (cells, nodes and particles each < 2^31). */
typedef struct aq_batch aq_batch;

aq_status aq_batch_create(const aq_config* configs, int32_t n_scenes, aq_batch** out);
/* Enqueues n_steps steps of every scene (asynchronous on the batch stream). */
aq_status aq_batch_step(aq_batch* b, int32_t n_steps);
/* Host-buffer step: optionally uploads the particle state of all scenes
 * ([3][N] float arrays, scenes concatenated in batch order, each scene in its
 * sorted order), steps, optionally downloads it, and synchronises.  Pinned
 * memory makes the copies asynchronous. */
aq_status aq_batch_step_host(aq_batch* b, int32_t n_steps, const float* position_in, const float* velocity_in,
                             float* position_out, float* velocity_out);
aq_status aq_batch_synchronize(aq_batch* b);
/* The cudaStream_t the batch runs on. */
aq_status aq_batch_stream(const aq_batch* b, void** stream);
int32_t aq_batch_scene_count(const aq_batch* b);
/* Size and particle count of one scene. */
aq_status aq_batch_scene_info(const aq_batch* b, int32_t scene, int32_t size_xyz[3], int64_t* particle_count);
/* Cells, nodes and particles over all scenes. */
aq_status aq_batch_totals(const aq_batch* b, int64_t* cells, int64_t* nodes, int64_t* particles);
/* One scene's state in the aq_host_state layout of a fluid of that size
 * (cell tables and sort indices relative to the scene). */
aq_status aq_batch_download_scene(aq_batch* b, int32_t scene, aq_host_state* s);
aq_status aq_batch_solve_stats(aq_batch* b, int32_t scene, aq_solve_stats* st);
/* Kernel launches per step outside the residual loop, and per loop block. */
aq_status aq_batch_launch_counts(const aq_batch* b, int32_t* per_step, int32_t* per_block);
/* Caps every batched launch at multiple x SMs CTAs (default 64, i.e. as many
 * as are resident at once; a batched launch never exceeds one resident wave).
 * Results do not depend on it. */
aq_status aq_batch_set_grid_multiple(aq_batch* b, int32_t multiple);
/* Shape of the batched Jacobi sweep: x planes each warp streams (1, 2, 4 or
 * 8; default 1) and, for more than one plane, whether the next plane's loads
 * are issued before the current plane's arithmetic.  Results do not depend
 * on it. */
aq_status aq_batch_set_sweep_plan(aq_batch* b, int32_t x_planes, int32_t pipelined);
aq_status aq_batch_get_sweep_plan(const aq_batch* b, int32_t* x_planes, int32_t* pipelined);
/* Project-written autotuner of the batched sweep: times every sweep plan on
 * the current pressure systems (advances the iterates), keeps the fastest. */
aq_status aq_batch_autotune(aq_batch* b, int32_t sweeps_per_trial, int32_t* x_planes, int32_t* pipelined,
                            float* sweep_us);
/* Times `sweeps` batched Jacobi sweeps of the current pressure systems of all
 * scenes (graph capture, one warm-up replay, one timed replay; advances the
 * iterates).  cells_per_sweep: cells of the flat blocks holding fluid. */
aq_status aq_batch_benchmark_pressure(aq_batch* b, int32_t sweeps, float* ms, int64_t* cells_per_sweep);
void aq_batch_destroy(aq_batch* b);

/* ---- Learned pressure warm start: building blocks ---------------------------
 * No counterpart in the reference.  BF16 tensors are channels-last over the
 * cell layout ((x*sy + y)*sz + z)*C + c, all pointers device memory, work on
 * `stream` (NULL = legacy default stream).
 * aq_conv3_forward: out = act(bias + conv3x3x3(in, w)), zero padding,
 *   w[27][cout][cin] bf16 (tap = (dx+1)*9 + (dy+1)*3 + (dz+1)), bias f32 or
 *   NULL, relu 0/1.  (cin, cout) in {(16,16), (16,32), (32,32), (32,64),
 *   (64,64), (96,32), (48,16), (32,16), (64,32), (32,96), (16,48)}.
 * aq_conv3_weight_grad: dw[27][cout][cin] (f32) = sum over voxels of
 *   dy[v][co] * x[v + tap offset][ci]; (cin, cout) a forward layer pair.
 * aq_conv3_flip_transpose: wt[t][ci][co] = w[26-t][co][ci], the weights whose
 *   forward convolution of dy is the data gradient. */
aq_status aq_conv3_forward(int32_t cin, int32_t cout, int32_t relu, const void* in, const void* w, const float* bias,
                           void* out, int32_t sx, int32_t sy, int32_t sz, void* stream);
aq_status aq_conv3_weight_grad(int32_t cin, int32_t cout, const void* x, const void* dy, float* dw, int32_t sx,
                               int32_t sy, int32_t sz, void* stream);
aq_status aq_conv3_flip_transpose(int32_t cin, int32_t cout, const void* w, void* wt, void* stream);
/* Forward kernel used by aq_conv3_forward and the network: 2 = tcgen05
 * UMMA with TMEM accumulators (default; pairs whose halo and weights fit in
 * shared memory, cout a multiple of 16 — the others run 1), 1 = halo-tiled
 * mma.sync, 0 = im2col streaming mma.sync.  Process-wide;
 * set it while no convolution is in flight.  1 and 0 compute the same sums
 * in the same order; 2 sums the same products in the tensor core's order.
 * aq_conv3_umma_status: nonzero *timeouts if a tcgen05 convolution ever
 * gave up waiting for its MMAs (its output is then not written). */
aq_status aq_conv3_set_tiled(int32_t tiled);
aq_status aq_conv3_umma_status(int32_t* timeouts);
/* Test hook of the tcgen05 convolution's bounded mbarrier wait.  skip_mma = 1
 * makes every later tcgen05 convolution issue no MMA and no commit (nothing is
 * in flight), so each thread's wait gives up after wait_ns nanoseconds (0 = the
 * default of one second): no output is written, TMEM is freed and
 * aq_conv3_umma_status reports the timeout.  skip_mma = 0 restores normal
 * operation with the default wait.  Either call synchronizes the device and
 * clears the timeout record.  Test use only. */
aq_status aq_conv3_test_wait_timeout(int32_t skip_mma, uint64_t wait_ns);

/* ---- Learned pressure warm start: network, dataset, training ---------------
 * No counterpart in the reference.  A 3-level 3D U-Net (16/32/64 channels,
 * 3x3x3 convolutions + ReLU, average pooling, upsampling with skip
 * concatenation, 1x1x1 head), BF16 weights and activations with FP32
 * accumulation, trained by the library's own kernels (Adam, FP32 master
 * weights) on pressure systems labelled by the FP64 PCG.  Input: the pressure
 * right-hand side (-divergence x density) scaled by its max-abs, and the
 * fluid mark; output: the pressure, used to warm-start the Jacobi solve
 * (AQ_PRESSURE_LEARNED).  Grid sizes must be divisible by 4.  A network runs
 * on its own stream; it must not be trained while a fluid step that uses it
 * is in flight, and fluids sharing it must not step concurrently. */
typedef struct aq_unet aq_unet;
typedef struct aq_dataset aq_dataset;

aq_status aq_unet_create(int32_t device, uint32_t seed, aq_unet** out);
void aq_unet_destroy(aq_unet* net);
aq_status aq_unet_parameter_count(const aq_unet* net, int64_t* count);
/* Weights file: magic, version, output scale, per layer (cin, cout, f32
 * weights [27][cout][cin], f32 bias [cout]), head (16 weights, bias). */
aq_status aq_unet_save(aq_unet* net, const char* path);
aq_status aq_unet_load(aq_unet* net, const char* path);
aq_status aq_unet_get_output_scale(const aq_unet* net, float* scale);
aq_status aq_unet_set_output_scale(aq_unet* net, float scale);
/* Forward pass on device buffers (rhs [C] f32, type [C] int8 0 air / 1
 * fluid): pressure [C] = warm start (0 off fluid).  stream NULL = the
 * network's stream. */
aq_status aq_unet_predict(aq_unet* net, int32_t sx, int32_t sy, int32_t sz, const float* rhs, const int8_t* type,
                          float* pressure, void* stream);

/* Device-resident training pairs of one grid size. */
aq_status aq_dataset_create(int32_t sx, int32_t sy, int32_t sz, int32_t capacity, int32_t device, aq_dataset** out);
void aq_dataset_destroy(aq_dataset* ds);
int32_t aq_dataset_count(const aq_dataset* ds);
/* Adds the fluid's current pressure system (as its last divergence stage
 * built it) labelled by an FP64 PCG solve to pcg_rel_tol. */
aq_status aq_dataset_add_fluid(aq_dataset* ds, aq_fluid* f, double pcg_rel_tol, int32_t pcg_max_iter,
                               int32_t* pcg_iterations);
aq_status aq_dataset_target_rms(aq_dataset* ds, int32_t first, int32_t count, double* rms);
/* Host copy of sample i: rhs / max|rhs| [C], type [C], pressure / max|rhs| [C]
 * (any pointer may be NULL). */
aq_status aq_dataset_get(aq_dataset* ds, int32_t i, float* rhs, int8_t* type, float* target);
/* `steps` Adam steps (one sample each, drawn with `seed` from samples
 * [first, first+count)), cosine-decayed learning rate from lr.  out_scale <= 0
 * sets the network's output scale to the targets' RMS.  Loss over fluid
 * cells, e = prediction - target, A the pressure operator and J one
 * homogeneous Jacobi sweep: ||e||^2/||t||^2 + residual_weight *
 * ||A J^k e||^2/||A J^k t||^2 with k = residual_sweeps; the second term is the
 * square of (residual after k sweeps from the prediction) / (the same from
 * zero), the ratio the warm start's fallback rule compares at k = 20.
 * mean_loss: mean loss of the last tenth of the steps. */
aq_status aq_unet_train(aq_unet* net, aq_dataset* ds, int32_t first, int32_t count, int32_t steps, float lr,
                        uint32_t seed, float out_scale, float residual_weight, int32_t residual_sweeps,
                        float* mean_loss);
/* Mean over samples of the relative L2 error (fluid cells) of the prediction
 * against the FP64 PCG pressure. */
aq_status aq_unet_evaluate(aq_unet* net, aq_dataset* ds, int32_t first, int32_t count, double* mean_rel_error);
/* Mean over samples of (relative residual after `sweeps` Jacobi sweeps from
 * the prediction) / (the same from zero): the ratio the warm start's
 * fallback rule compares at 20 sweeps (below 1, the prediction is kept). */
aq_status aq_unet_evaluate_warm(aq_unet* net, aq_dataset* ds, int32_t first, int32_t count, int32_t sweeps,
                                double* mean_ratio);
/* The gradients of the last training step, in weights-file order (per layer
 * weights then bias, then head weights and bias); n = parameter count. */
aq_status aq_unet_gradients(aq_unet* net, float* out, int64_t n);

/* Concentration mass per phase: the sum over particles of their volume
 * fractions (FP64; single-phase fluids: the particle count in their phase).
 * No counterpart in the reference; its change over a run is the
 * concentration-mass conservation error of multiphase diffusion. */
aq_status aq_fluid_phase_mass(aq_fluid* f, double mass[4]);

/* Ink particles: massless tracers the reference builds but leaves switched
 * off (its calls are commented out at Fluid/Fluid_3D_FLIP.cu:349-350 and
 * :498).  aq_fluid_enable_ink replaces Fluid::initInkRenderer
 * (Fluid/Fluid_3D_FLIP.cu:676-709): it seeds the ink once, at spacing h/4
 * over the initial volumes (createSquareInk / createSphereInk,
 * Fluid/Fluid_3D_FLIP.cu:600-664), continuing the particle seeding's rand()
 * sequence, so the ink is the one Fluid::init would have made whenever it is
 * called; count (may be NULL) receives the ink particle count.  From then on
 * every step ends by advancing the ink as transferToInkParticles +
 * moveInkParticles(timestep) would (Fluid/Fluid_3D_FLIP.cu:711-725): G2P with
 * FLIP coefficient 1 and RK3 advection in the step's grid velocities.
 * aq_fluid_ink_advance runs that advance alone on the current grids.
 * Positions and velocities are [3][count] planes; either pointer may be NULL.
 * The download / upload / advance calls fail with AQ_ERR_INVALID_ARGUMENT
 * before aq_fluid_enable_ink. */
aq_status aq_fluid_enable_ink(aq_fluid* f, int32_t* count);
aq_status aq_fluid_ink_count(const aq_fluid* f, int32_t* count);
aq_status aq_fluid_download_ink(aq_fluid* f, float* position, float* velocity);
aq_status aq_fluid_upload_ink(aq_fluid* f, const float* position, const float* velocity);
aq_status aq_fluid_ink_advance(aq_fluid* f);

/* Surface mesher: replaces Mesher::mesh (Rendering/Renderer3D/Mesher.cuh:
 * 140-178, Mesher.cu:321-630) as Fluid::init builds it
 * (Fluid/Fluid_3D_FLIP.cu:495) and draw() calls it (:404): a particle SDF on
 * a grid of cell h/2 (computeSDF, Mesher.cuh:20-84) and marching cubes on a
 * fixed 128^3 grid of cell size_x*h/126 spanning [-cell, 127*cell] on every
 * axis (marchingCubes, Mesher.cu:322-425).
 *
 * Output layout, the reference's mesh VBO: one record per occupied cube
 * (a cube whose type has triangles), 15 vertex slots of 6 floats (position
 * xyz, normal xyz); slots the cube's triangles do not use are zero.  Records
 * come in cube order (x slowest, z fastest) — the reference appends them in
 * atomic order, so the set of records is the same, the order deterministic.
 * Unlike the reference, the fluid's particle order is left as the step left
 * it (the reference re-sorts the particle array by the SDF grid).
 *
 * aq_fluid_mesh writes into a DEVICE buffer of capacity_records records (the
 * reference passes its mapped VBO): records past capacity are dropped,
 * everything after the last record is zero (a buffer is cleared whole the
 * first time it is seen); cubes (may be NULL) receives the occupied-cube
 * count, which may exceed capacity.  aq_fluid_download_mesh does the same
 * into HOST memory.  aq_fluid_download_sdf copies the last mesh's SDF grid,
 * [sdf_x][sdf_y][sdf_z] with z fastest.  The particles must be sorted by
 * cell, as any step, the init or the sort stage leaves them; otherwise the
 * calls fail with AQ_ERR_INVALID_ARGUMENT. */
typedef struct {
  int32_t sdf_size[3];  /* 3 + size*h/(h/2) per axis (Mesher.cu:589-591) */
  int32_t mesh_size[3]; /* 128 per axis (Mesher.cuh:104-106) */
  float sdf_cell;       /* h/2 */
  float mesh_cell;      /* size_x*h/126 */
  float particle_radius; /* h/2 */
} aq_mesh_info;
aq_status aq_fluid_mesh_info(const aq_fluid* f, aq_mesh_info* info);
aq_status aq_fluid_mesh(aq_fluid* f, float* output, int64_t capacity_records, int32_t* cubes);
aq_status aq_fluid_download_mesh(aq_fluid* f, float* records, int64_t capacity_records, int32_t* cubes);
aq_status aq_fluid_download_sdf(aq_fluid* f, float* sdf);

/* Attaches the network used by AQ_PRESSURE_LEARNED (NULL detaches).  The
 * network must outlive the fluid's steps; allocate-once buffers for the
 * fluid's grid are made here, so call it before the first step. */
aq_status aq_fluid_set_warm_start(aq_fluid* f, aq_unet* net);

/* Largest grid (sx*sy*sz cells) aq_jacobi_sweeps_noalloc accepts. */
#define AQ_NOALLOC_MAX_CELLS (64 * 64 * 64)

/* Pressure Jacobi sweeps on caller-owned device buffers that allocate
 * nothing.  No counterpart in the reference: it is for callers that cannot
 * allocate device memory while they run the solver (a fixed memory pool
 * handed over by a host application, a memory-budgeted frame loop, a plugin
 * that must not touch its host process's allocator).
 *
 * cell_type [C] (1 fluid; any other value, such as 0 air or 2 solid, is
 * not fluid and its pressure is set to 0, as the pressure stage does), rhs
 * [C] (-divergence*density on fluid cells) and pressure [C] (initial guess
 * in, result out) are device buffers in the cell layout of aq_host_state;
 * `sweeps` Jacobi sweeps are run on
 * `stream` (NULL = the legacy default stream) exactly as the pressure stage
 * of aq_fluid_step does in AQ_SOLVE_FIXED mode, including clearing air
 * pressure first.  The second Jacobi buffer and the activity flags are a
 * fixed device array of AQ_NOALLOC_MAX_CELLS floats that every GPU loading
 * this library holds until exit; larger grids return AQ_ERR_INVALID_ARGUMENT.
 * The first call on a device looks the array up (cudaGetSymbolAddress) and
 * must come before any stream capture.  All calls on a device share the
 * array, so calls that overlap on the GPU race: serialise them. */
aq_status aq_jacobi_sweeps_noalloc(int32_t sx, int32_t sy, int32_t sz, const int8_t* cell_type,
                                   const float* rhs, float* pressure, int32_t sweeps, void* stream);
/* AQ_NOALLOC_MAX_CELLS, as compiled into the library. */
int32_t aq_jacobi_noalloc_max_cells(void);

/* Thread-local message of the last failed call ("" if none). */
const char* aq_last_error(void);

/* Library ABI version (AQ_ABI_VERSION). */
int32_t aq_abi_version(void);

/* ------------------------------------------------------------ SPH solvers
 * The reference's two particle-only solvers, which share the FLIP path's
 * spatial hash and stable sort: position-based fluids
 * (Fluid_3D_PBF::Fluid, Fluid/Fluid_3D_PBF.cuh:49-133, Fluid_3D_PBF.cu)
 * and predictive-corrective SPH (Fluid_3D_PCISPH::Fluid,
 * Fluid/Fluid_3D_PCISPH.cuh:47-124, Fluid_3D_PCISPH.cu).  Both run in the
 * reference's fixed 10 x 10 x 10 container (gridPhysicalSize), with a
 * particle spacing derived from max_particle_count and a hash grid of cell
 * = kernel radius.  aq_sph_create = make_shared<Fluid>() + init(config)
 * (main.cu:158-170); aq_sph_step = simulationStep(). */
typedef enum aq_sph_method { AQ_SPH_PBF = 0, AQ_SPH_PCISPH = 1 } aq_sph_method;

/* FluidConfig + ConfigPBF / ConfigPCISPH (Fluid/FluidConfig.cuh:52-66). */
typedef struct aq_sph_config {
  int32_t method;              /* aq_sph_method */
  int32_t volume_count;
  aq_volume volumes[AQ_MAX_VOLUMES]; /* phase is ignored */
  float gravity[3];
  float timestep;              /* ConfigPBF 0.033 / ConfigPCISPH 0.005 */
  int32_t substeps;            /* 4 / 1 */
  int32_t iterations;          /* 2 / 4 */
  int32_t max_particle_count;  /* 3e5 / 3e5: sets the particle spacing */
  float particle_jitter;       /* PBF only, 0.05 */
  float stiffness;             /* PCISPH only, 15 (read but unused by the reference) */
  uint32_t seed;               /* glibc rand() seed of the seeding jitter (reference: 1) */
  int32_t device;
  void* stream;                /* cudaStream_t; NULL = library-owned stream */
} aq_sph_config;

/* Reference defaults for the method, with the default volumes and gravity. */
aq_status aq_sph_config_default(int32_t method, aq_sph_config* cfg);

/* Host copy of the particle state, [3][n] planes or [n]; any pointer may be
 * NULL.  The reference's Particle structs (Fluid/Fluid_3D_PBF.cuh:23-44,
 * Fluid/Fluid_3D_PCISPH.cuh:20-45) in planar form. */
typedef struct aq_sph_state {
  int32_t particle_count;       /* must match */
  double physical_time;
  float* position;              /* [3][n] */
  float* velocity;              /* [3][n] velosity */
  float* density;               /* [n] */
  float* rest_density;          /* [n] restDensity */
  float* last_position;         /* [3][n] PBF lastPosition */
  float* lambda;                /* [n]    PBF */
  float* pressure;              /* [n]    PCISPH */
  float* pressure_force;        /* [3][n] PCISPH pressureForces */
  float* predicted_position;    /* [3][n] PCISPH predictedPosition */
  float* predicted_velocity;    /* [3][n] PCISPH predictedVelocity */
} aq_sph_state;

typedef struct aq_sph_info {
  int32_t particle_count;
  float particle_spacing;       /* particleSpacing */
  float kernel_radius;          /* kernelRadius = spacing * 2.01 (PBF) / 2 (PCISPH) */
  int32_t grid_size[3];         /* hash grid, ceil(10 / kernelRadius) per axis */
  float container_size;         /* gridPhysicalSize, 10 */
} aq_sph_info;

typedef struct aq_sph aq_sph;

aq_status aq_sph_create(const aq_sph_config* cfg, aq_sph** out);
void aq_sph_destroy(aq_sph* s);
aq_status aq_sph_info_get(const aq_sph* s, aq_sph_info* info);
aq_status aq_sph_step(aq_sph* s, int32_t nsteps);
aq_status aq_sph_synchronize(aq_sph* s);
/* Kernel launches in one step (the step runs as one CUDA graph). */
aq_status aq_sph_launches_per_step(const aq_sph* s, int32_t* launches);
aq_status aq_sph_download_state(aq_sph* s, aq_sph_state* st);
/* Replaces fields; positions are kept in the container.  Uploaded particles
 * need not be sorted: every step starts with the spatial hash. */
aq_status aq_sph_upload_state(aq_sph* s, const aq_sph_state* st);


/* ---------------------------------------------------------------- frames
 * Headless frame of the reference's renderer: the GL draw calls of one frame
 * (main.cu:111-145: glClear, Skybox::draw, Container::drawFace, Fluid::draw)
 * restated as CUDA kernels that write an RGBA8 image into a DEVICE buffer,
 * with no graphics API.  The shading is the arithmetic of the reference's
 * shaders (resources/Shaders/Skybox_fs.glsl, Container_face_fs.glsl,
 * RayTraceEnvironment.glsl, PointSprites_points_vs.glsl,
 * PointSprites_phase_fs.glsl, PointSprites_simple_fs.glsl,
 * FluidMeshRenderer_vs.glsl, FluidMeshRenderer_fs.glsl); the fixed-function
 * GL stages (clipping, point and triangle rasterisation, the 24-bit depth
 * test GL_LESS, blending into an RGBA8 framebuffer) follow the GL rules as
 * restated in the frame kernels' header comment.
 *
 *   reference                                            replacement
 *   ---------------------------------------------------  ------------------------
 *   DrawCommand (Rendering/DrawCommand.h:37-59)          aq_draw_command
 *   Camera(center) + glm::lookAt / glm::perspective      aq_draw_command_default
 *     (Rendering/Renderer3D/camera.h:65-125, main.cu:115-133)
 *   updatePositionsAndPhasesVBO                          aq_fluid_points_vbo
 *     (Fluid/Fluid_3D_kernels.cuh:69-91)
 *   Skybox / Container / PointSprites /                  aq_renderer_create,
 *     FluidMeshRenderer construction and textures          aq_renderer_set_skybox,
 *     (Skybox.cu:5-58, Container.cu:8-40)                  aq_renderer_set_logo
 *   Fluid::draw (Fluid/Fluid_3D_FLIP.cu:396-430)         aq_fluid_draw
 *   the frame's draws (main.cu:136-143,                  aq_renderer_draw
 *     FluidMeshRenderer.cu:56-126, PointSprites.cu:196-256,
 *     Container.cu:71-120, Skybox.cu:60-78)
 *
 * The image is row-major with row 0 at the BOTTOM of the window (the order
 * glReadPixels returns), 4 bytes per pixel. */
typedef enum aq_render_mode {  /* RenderMode (Rendering/DrawCommand.h:5-19) */
  AQ_RENDER_MULTIPHASE_MESH = 0,
  AQ_RENDER_WATER_MESH = 1,
  AQ_RENDER_FLAT_MESH = 2,
  AQ_RENDER_NORMAL_MESH = 3,
  AQ_RENDER_MIRROR_MESH = 4,
  AQ_RENDER_REFRACT_MESH = 5,
  AQ_RENDER_PHASE0_MESH = 6,
  AQ_RENDER_PHASE1_MESH = 7,
  AQ_RENDER_PARTICLES = 8,
  AQ_RENDER_NONE = 9
} aq_render_mode;

typedef enum aq_environment_mode {  /* EnvironmentMode (Rendering/DrawCommand.h:21-26) */
  AQ_ENV_SKYBOX = 0,
  AQ_ENV_CORNELL_BOX = 1,
  AQ_ENV_CHESS_BOARD = 2
} aq_environment_mode;

typedef struct aq_draw_command {
  /* DrawCommand */
  float view[16];        /* column-major (glm layout): element (row r, col c) at [c*4 + r] */
  float projection[16];
  float camera_position[3];
  int32_t window_width, window_height;
  float fov;             /* Camera::FOV (45); the projection above already holds it */
  float near_plane, far_plane;
  int32_t render_mode;   /* aq_render_mode */
  int32_t environment_mode; /* aq_environment_mode */
  float light_position[3];
  float container_size;
  float cornell_box_size;
  /* what Fluid::draw passes along (Fluid/Fluid_3D_FLIP.cu:396-430) */
  float point_radius;    /* phase-thickness sprites: cellPhysicalSize; AQ_RENDER_PARTICLES: renderRadius */
  int32_t phase_count;   /* FluidConfig::phaseCount */
  float phase_colors[4][4]; /* FluidConfig::phaseColors, rgba */
} aq_draw_command;

/* The first frame's DrawCommand of main.cu for a fluid of physical size
 * domain_size with size_y cells along y and particles_per_cell particles per
 * cell: Camera(center) as constructed (yaw 180, pitch -30, global yaw 0,
 * global pitch 30, radius 18, looking at the centre), glm::lookAt,
 * glm::perspective(45, width/height, 0.1, 1000) (45 taken as radians, as
 * glm 0.9.9 does), light (cx, 15, cy), container size domain_size, Cornell
 * box 4x that, render mode AQ_RENDER_MULTIPHASE_MESH, environment
 * AQ_ENV_SKYBOX, point radius cellPhysicalSize, the default phase colours. */
aq_status aq_draw_command_default(aq_draw_command* dc, int32_t width, int32_t height, float domain_size,
                                  int32_t size_y);

/* Fills the reference's point-sprite VBO: 7 floats per particle (position
 * xyz, volume fractions xyzw) into a DEVICE buffer of 7*N floats, in the
 * fluid's particle order. */
aq_status aq_fluid_points_vbo(aq_fluid* f, float* vbo);

typedef struct aq_renderer aq_renderer;

/* stream: cudaStream_t (NULL: a renderer-owned stream). */
aq_status aq_renderer_create(int32_t device, void* stream, aq_renderer** out);
void aq_renderer_destroy(aq_renderer* r);

/* Skybox cube map: six face_size x face_size RGB8 images in the order posx,
 * negx, posy, negy, posz, negz (Skybox.cu:24-44), each row-major with its
 * first row at t = 0, as glTexImage2D receives them.  Sampled with linear
 * filtering, clamped to the edge.  NULL clears it (samples are black). */
aq_status aq_renderer_set_skybox(aq_renderer* r, const uint8_t* faces_rgb, int32_t face_size);

/* The Cornell box's logo texture (Container::loadOxLogo, Container.cu:16-40):
 * width x height RGB8, first row at t = 0; linear, clamped.  NULL clears it. */
aq_status aq_renderer_set_logo(aq_renderer* r, const uint8_t* rgb, int32_t width, int32_t height);

/* One frame.  points: DEVICE point-sprite VBO (7 floats per point) or NULL
 * when n_points is 0; mesh: DEVICE mesh VBO (6 floats per vertex, position
 * and normal, triangles of 3 consecutive vertices; aq_fluid_mesh writes 90
 * floats per record = 15 vertices) or NULL when n_vertices is 0; rgba:
 * DEVICE buffer of window_width*window_height*4 bytes, or NULL for the
 * renderer's own image buffer.  The mesh modes use
 * the points only for the phase thickness (modes 0, 5, 6, 7).  Enqueued on
 * the renderer's stream; aq_renderer_synchronize waits for it. */
aq_status aq_renderer_draw(aq_renderer* r, const aq_draw_command* dc, const float* points, int32_t n_points,
                           const float* mesh, int64_t n_vertices, uint8_t* rgba);
aq_status aq_renderer_synchronize(aq_renderer* r);

/* Fluid::draw(drawCommand) (Fluid/Fluid_3D_FLIP.cu:396-430): meshes the
 * current particles (mesh modes; the reference re-meshes whenever the
 * simulation is not paused), fills the point-sprite VBO and draws, all into
 * renderer-owned buffers, the image into rgba (DEVICE, W*H*4 bytes) or, when
 * rgba is NULL, into a renderer-owned image that aq_renderer_download_image
 * copies out. */
aq_status aq_fluid_draw(aq_fluid* f, aq_renderer* r, const aq_draw_command* dc, uint8_t* rgba);

/* The last frame's image (W*H*4 bytes, row 0 at the bottom) into HOST memory. */
aq_status aq_renderer_download_image(aq_renderer* r, uint8_t* host);

/* The last frame's phase-thickness texture (PointSprites::phaseThicknessTexture):
 * window_width*window_height*4 floats, row 0 at the bottom, into HOST memory.
 * Zero when the last frame had no phase pass. */
aq_status aq_renderer_download_phase_thickness(aq_renderer* r, float* host);

/* Kernel launches of the last aq_renderer_draw. */
aq_status aq_renderer_launches(const aq_renderer* r, int32_t* launches);

#ifdef __cplusplus
}
#endif

#endif /* AQUARIUS_B200_H */
