/*
 * CPU oracle of the reference's particle-only solvers, position-based
 * fluids (Fluid/Fluid_3D_PBF.cu) and PCISPH (Fluid/Fluid_3D_PCISPH.cu) —
 * TEST INFRASTRUCTURE ONLY.  The checker for the library's aq_sph_* path and
 * its CPU baseline; the library never links, loads or calls it.
 */
#ifndef AQ_SPH_ORACLE_H
#define AQ_SPH_ORACLE_H

#include "../include/aquarius_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_sph orc_sph;

/* Fluid::init: seeding with the glibc rand() sequence of cfg->seed, the
 * spatial hash and the rest densities.  NULL on an invalid config. */
orc_sph* orc_sph_create(const aq_sph_config* cfg);
void orc_sph_destroy(orc_sph* o);
int orc_sph_count(const orc_sph* o);
/* particleSpacing, kernelRadius, gridSize (any may be NULL). */
void orc_sph_info(const orc_sph* o, float* spacing, float* kernel_radius, int* grid);
/* n simulationStep()s; returns 0. */
int orc_sph_step(orc_sph* o, int n);
/* State exchange in the aq_sph_state layout; nonzero on a count mismatch. */
int orc_sph_get(const orc_sph* o, aq_sph_state* s);
int orc_sph_set(orc_sph* o, const aq_sph_state* s);

#ifdef __cplusplus
}
#endif

#endif
