/*
 * CPU oracle of the Aquarius 3D FLIP step — TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C (OpenMP) restatement of Fluid_3D_FLIP::Fluid::init and
 * ::simulationStep (AmesingFlank/Aquarius, Fluid/Fluid_3D_FLIP.cu:316-594,
 * Fluid/Fluid_3D_kernels.cu, Fluid/Fluid_3D_common.{cu,cuh},
 * Fluid/MAC_Grid_3D.cuh, Fluid/WeightKernels.cuh:131-146).  It is the checker
 * for the CUDA library and the timed CPU baseline; the library never links,
 * loads or calls it.
 *
 * Where the reference kernels race (in-place Jacobi, in-place diffusion,
 * in-place extrapolation, read-modify-write gravity on neighbour faces) this
 * oracle uses the race-free reading: every sweep/pass reads the previous
 * sweep's values.  Air-cell pressure is cleared before the first sweep.
 *
 * Parity is pinned against the reference's own kernels built headless
 * (oracle/_ref, see oracle/Makefile) through fixtures under tests/golden/.
 */
#ifndef AQ_FLIP_ORACLE_H
#define AQ_FLIP_ORACLE_H

#include "../include/aquarius_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_fluid orc_fluid;

/* Fluid::init (Fluid/Fluid_3D_FLIP.cu:435-505). NULL on invalid config. */
orc_fluid* orc_create(const aq_config* cfg);
void orc_destroy(orc_fluid* o);

int orc_particle_count(const orc_fluid* o);
/* One sub-stage (aq_stage numbering); returns 0 on success. */
int orc_run_stage(orc_fluid* o, int stage);
/* n full simulationStep()s. */
int orc_step(orc_fluid* o, int n);

/* Copies the state out / in using the canonical aq_host_state layout.
 * Returns 0 on success, nonzero on a size mismatch. */
int orc_get_state(const orc_fluid* o, aq_host_state* s);
int orc_set_state(orc_fluid* o, const aq_host_state* s);

/* Last pressure solve: sweeps, relative residual (FP64), ||b||, fluid cells. */
void orc_solve_stats(const orc_fluid* o, int* iters, double* rel_res, double* b_norm, int* fluid_cells);

/* Relative residual of the current pressure for the current system. */
double orc_pressure_residual(const orc_fluid* o);

/* 0 (default): the race-free reading of the reference's in-place Jacobi and
 * extrapolation.  1: those two stages in place in a serial schedule of the
 * reference's launch (blocks in launch order, warps in order, each warp
 * reading before it writes), another outcome the racy kernels allow; used by
 * the tests to bound how far the race can move the reference's result. */
void orc_set_schedule(orc_fluid* o, int schedule);

/* Fills a default config (same values as aq_config_default). */
void orc_config_default(aq_config* cfg);

/* Number of OpenMP threads the oracle uses (omp_get_max_threads). */
int orc_threads(void);

/* Ink particles (Fluid_3D_FLIP.cu:600-725): seeds them once (continuing the
 * fluid seeding's rand() sequence; returns the count), advances them with
 * the current grid velocities (FLIP coefficient 1, then RK3), host copies
 * of positions / velocities ([3][n], either may be NULL).  Once seeded, the
 * diffusion stage (the end of every step) also advances them. */
int orc_ink_create(orc_fluid* o);
int orc_ink_count(const orc_fluid* o);
void orc_ink_advance(orc_fluid* o);
void orc_ink_get(const orc_fluid* o, float* pos, float* vel);
void orc_ink_set(orc_fluid* o, const float* pos, const float* vel);

/* Surface mesher (Rendering/Renderer3D/Mesher.cuh:20-178, Mesher.cu:321-630)
 * on the current particles in their array order.  Grid sizes as Fluid::init
 * builds the Mesher: SDF cell h/2 and sdf[k] = 3 + size_k * h / (h/2) cells,
 * a 128^3 marching-cubes grid of cell size_x * h / 126. */
typedef struct {
  int sdf[3], mesh[3];
  float h_sdf, h_mesh, radius;
} orc_mesh_dims;
void orc_mesh_dims_of(const orc_fluid* o, orc_mesh_dims* m);
/* sdf_out ([sdf x][y][z], z fastest) and records ([capacity][15][6]) may be
 * NULL; cubes receives the occupied-cube count (records past capacity are
 * dropped).  Returns 0, or 1 when out of memory. */
int orc_mesh(orc_fluid* o, float* sdf_out, float* records, long long capacity, int* cubes);
/* The mesher's model of the texture unit's linear filter on a [w][h][d]
 * field (z fastest) at coords ([n][3], x y z). */
void orc_tex_linear(const float* field, int w, int h, int d, const float* coords, float* out, int n);

#ifdef __cplusplus
}
#endif
#endif
