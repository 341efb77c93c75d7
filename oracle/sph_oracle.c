/*
 * CPU oracle of the reference's particle-only solvers — TEST INFRASTRUCTURE
 * ONLY.  A plain-C restatement of Fluid_3D_PBF::Fluid (Fluid/Fluid_3D_PBF.cu)
 * and Fluid_3D_PCISPH::Fluid (Fluid/Fluid_3D_PCISPH.cu): seeding, the
 * spatial hash with its stable sort (performSpatialHashing2,
 * Fluid/Fluid_3D_common.cuh:27-56), and every kernel of simulationStep, each
 * function citing the lines it follows.  Every float operation rounds as
 * written (-ffp-contract=off); where the reference evaluates in double (a
 * double literal in the expression) so does this file.
 */
#define _GNU_SOURCE /* random_r, initstate_r */
#include "sph_oracle.h"

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include <omp.h>

#define SPH_PI 3.14159265358979323846f /* PI, Fluid/WeightKernels.cuh:8 */

typedef struct {
  struct random_data rd;
  char state[128];
} sph_rng;

static float rnd01(sph_rng* r) { /* random0to1, Common/Commons.h:3-5 */
  int32_t v;
  random_r(&r->rd, &v);
  return (float)v / (float)RAND_MAX;
}

struct orc_sph {
  aq_sph_config cfg;
  int method, n;
  float size; /* gridPhysicalSize (10, 10, 10) */
  float spacing, kr, kr2, kr3, kr5, kr6, kr9;
  int gx, gy, gz, cells;
  double time;
  /* [3][n] planes and [n] arrays, in the current (sorted) order */
  float *pos, *vel, *density, *rest, *last, *lambda, *delta, *pressure, *force, *ppos, *pvel;
  int *key, *order, *start; /* start[cells + 1] */
};

static void* zalloc(size_t n, size_t s) { return calloc(n ? n : 1, s); }

/* ------------------------------------------------------------- kernels */

/* poly6 (Fluid/WeightKernels.cuh:13-26) */
static inline float poly6(float vx, float vy, float vz, float h2, float h9) {
  const float r2 = vx * vx + vy * vy + vz * vz;
  if (r2 <= h2) {
    const float t = h2 - r2;
    const float t3 = t * t * t;
    return t3 * 315.f / (64.f * SPH_PI * h9);
  }
  return 0;
}

/* spikey_grad (Fluid/WeightKernels.cuh:43-58) */
static inline void spikey_grad(float vx, float vy, float vz, float h, float h6, float* gx, float* gy, float* gz) {
  const float r = sqrtf(vx * vx + vy * vy + vz * vz);
  float ux = vx, uy = vy, uz = vz;
  if (r != 0) { ux /= r; uy /= r; uz /= r; }
  if (0 <= r && r <= h) {
    const float hr = h - r, d = SPH_PI * h6;
    *gx = -ux * hr * hr * 45.f / d;
    *gy = -uy * hr * hr * 45.f / d;
    *gz = -uz * hr * hr * 45.f / d;
  } else {
    *gx = *gy = *gz = 0;
  }
}

/* cubic_spline_kernel (Fluid/WeightKernels.cuh:196-206) */
static float cubic_spline(float r, float radius, float radius3) {
  const float q = 2.0f * r / radius;
  if (q > 2.0f) return 0.0f;
  const float a = 0.25f / (SPH_PI * radius3);
  return a * ((q > 1.0f) ? (2.0f - q) * (2.0f - q) * (2.0f - q) : ((3.0f * q - 6.0f) * q * q + 4.0f));
}

/* ---------------------------------------------------------- seeding */

typedef struct {
  float* p;
  int n, cap;
} plist3;

static void push3(plist3* l, float x, float y, float z) {
  if (l->n == l->cap) {
    l->cap = l->cap ? 2 * l->cap : 4096;
    l->p = (float*)realloc(l->p, sizeof(float) * 3 * (size_t)l->cap);
  }
  l->p[3 * l->n] = x; l->p[3 * l->n + 1] = y; l->p[3 * l->n + 2] = z;
  l->n++;
}

static inline float clampf(float v, float lo, float hi) { return fminf(hi, fmaxf(lo, v)); }

/* createSquareFluid (Fluid_3D_PBF.cu:397-437, Fluid_3D_PCISPH.cu:254-292):
 * a lattice of the particle spacing, loops x, y, z; jitter magnitude
 * spacing * particleJitter (PBF) or spacing / 2 (PCISPH). */
static void square(const orc_sph* o, sph_rng* rng, plist3* out, const aq_volume* v) {
  const float S = o->size, sp = o->spacing;
  const float md = sp / 2.f;
  const float shrink = (float)((double)md - 1e-3);
  const float x0 = v->box_min[0] * S + md, y0 = v->box_min[1] * S + md, z0 = v->box_min[2] * S + md;
  const float x1 = v->box_max[0] * S - shrink, y1 = v->box_max[1] * S - shrink, z1 = v->box_max[2] * S - shrink;
  const float mag = o->method == AQ_SPH_PBF ? sp * o->cfg.particle_jitter : sp / 2.f;
  for (float x = x0; x <= x1; x += sp)
    for (float y = y0; y <= y1; y += sp)
      for (float z = z0; z <= z1; z += sp) {
        float jx = (float)((double)rnd01(rng) - 0.5);
        float jy = (float)((double)rnd01(rng) - 0.5);
        float jz = (float)((double)rnd01(rng) - 0.5);
        jx *= mag; jy *= mag; jz *= mag;
        push3(out, clampf(x + jx, md, S - md), clampf(y + jy, md, S - md), clampf(z + jz, md, S - md));
      }
}

/* createSphereFluid (Fluid_3D_PBF.cu:438-472, Fluid_3D_PCISPH.cu:293-323):
 * a lattice over the whole container from spacing/2, kept inside the ball.
 * PBF adds a jitter of (r - 0.5) * spacing * 0.5 first; PCISPH draws the
 * same three numbers (scale 0.01) but never adds them. */
static void sphere(const orc_sph* o, sph_rng* rng, plist3* out, const aq_volume* v) {
  const float S = o->size, sp = o->spacing;
  const float lo = sp * 0.5f, hi = S - sp * 0.5f;
  const float cx = v->ball_center[0] * S, cy = v->ball_center[1] * S, cz = v->ball_center[2] * S;
  const float R = v->ball_radius * S;
  const double scale = o->method == AQ_SPH_PBF ? 0.5 : 0.01;
  for (float x = lo; x < hi; x += sp)
    for (float y = lo; y < hi; y += sp)
      for (float z = lo; z < hi; z += sp) {
        float px = x, py = y, pz = z;
        const float jx = (float)(((double)rnd01(rng) - 0.5) * sp * scale);
        const float jy = (float)(((double)rnd01(rng) - 0.5) * sp * scale);
        const float jz = (float)(((double)rnd01(rng) - 0.5) * sp * scale);
        if (o->method == AQ_SPH_PBF) { px += jx; py += jy; pz += jz; }
        const float ex = px - cx, ey = py - cy, ez = pz - cz;
        if (sqrtf(ex * ex + ey * ey + ez * ez) < R) push3(out, px, py, pz);
      }
}

/* ------------------------------------------------------- spatial hash */

/* performSpatialHashing2 with the kernel radius as cell size: calcHashImpl
 * (Fluid_3D_kernels.cuh:8-27), a stable sort of the particles by cell, and
 * the cell ranges (here CSR starts). */
static void sph_sort(orc_sph* o) {
  const int n = o->n;
  memset(o->start, 0, sizeof(int) * ((size_t)o->cells + 1));
  for (int i = 0; i < n; ++i) {
    const int x = (int)(o->pos[i] / o->kr), y = (int)(o->pos[n + i] / o->kr), z = (int)(o->pos[2 * n + i] / o->kr);
    o->key[i] = x * o->gy * o->gz + y * o->gz + z;
    o->start[o->key[i] + 1]++;
  }
  for (int c = 0; c < o->cells; ++c) o->start[c + 1] += o->start[c];
  int* fill = (int*)malloc(sizeof(int) * (size_t)o->cells);
  memcpy(fill, o->start, sizeof(int) * (size_t)o->cells);
  for (int i = 0; i < n; ++i) o->order[fill[o->key[i]]++] = i;
  free(fill);
  float* tmp = (float*)malloc(sizeof(float) * 3 * (size_t)(n > 0 ? n : 1));
  float* planes3[] = {o->pos, o->vel, o->last, o->force, o->ppos, o->pvel};
  for (size_t q = 0; q < sizeof(planes3) / sizeof(planes3[0]); ++q) {
    float* a = planes3[q];
    for (int k = 0; k < 3; ++k)
      for (int i = 0; i < n; ++i) tmp[(size_t)k * n + i] = a[(size_t)k * n + o->order[i]];
    memcpy(a, tmp, sizeof(float) * 3 * (size_t)n);
  }
  float* planes1[] = {o->density, o->rest, o->lambda, o->pressure};
  for (size_t q = 0; q < sizeof(planes1) / sizeof(planes1[0]); ++q) {
    float* a = planes1[q];
    for (int i = 0; i < n; ++i) tmp[i] = a[o->order[i]];
    memcpy(a, tmp, sizeof(float) * (size_t)n);
  }
  free(tmp);
}

/* Cell of a position and the 27-cell neighbourhood walk, dx, dy, dz from -1
 * to 1, cells outside the grid skipped (Fluid_3D_PBF.cu:35-58). */
#define FOR_NEIGHBOURS(o, X, Y, Z, J)                                                   \
  const int cx_ = (int)((X) / (o)->kr), cy_ = (int)((Y) / (o)->kr), cz_ = (int)((Z) / (o)->kr); \
  for (int dx_ = -1; dx_ <= 1; ++dx_)                                                   \
    for (int dy_ = -1; dy_ <= 1; ++dy_)                                                 \
      for (int dz_ = -1; dz_ <= 1; ++dz_)                                               \
        for (int x_ = cx_ + dx_, y_ = cy_ + dy_, z_ = cz_ + dz_, once_ = 1; once_; once_ = 0) \
          if (!(x_ < 0 || x_ >= (o)->gx || y_ < 0 || y_ >= (o)->gy || z_ < 0 || z_ >= (o)->gz)) \
            for (int h_ = x_ * (o)->gy * (o)->gz + y_ * (o)->gz + z_, J = (o)->start[h_]; J < (o)->start[h_ + 1]; ++J)

/* ------------------------------------------------------------------ PBF */

/* computeDensityAndLambdaImpl (Fluid_3D_PBF.cu:28-110) */
static void pbf_lambda(orc_sph* o, int set_rest) {
  const int n = o->n;
  const float *px = o->pos, *py = o->pos + n, *pz = o->pos + 2 * n;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; ++i) {
    float gx = 0, gy = 0, gz = 0, sdot = 0, density = 0;
    FOR_NEIGHBOURS(o, px[i], py[i], pz[i], j) {
      const float dx = px[i] - px[j], dy = py[i] - py[j], dz = pz[i] - pz[j];
      density += poly6(dx, dy, dz, o->kr2, o->kr9);
      float wx, wy, wz;
      spikey_grad(dx, dy, dz, o->kr, o->kr6, &wx, &wy, &wz);
      gx += wx; gy += wy; gz += wz;
      sdot += wx * wx + wy * wy + wz * wz;
    }
    o->density[i] = density;
    if (set_rest) o->rest[i] = density;
    const float rho0 = o->rest[i];
    const float ci = o->density[i] / rho0 - 1;
    const float q = (sdot + (gx * gx + gy * gy + gz * gz)) / (rho0 * rho0);
    const float den = (float)(1e-3 + (double)q);
    float lambda = -ci / den;
    if (ci < 0) lambda = (float)((double)lambda * 1e-2);
    o->lambda[i] = lambda;
  }
}

/* computeDeltaPositionImpl then applyDeltaPositionImpl
 * (Fluid_3D_PBF.cu:114-206). */
static void pbf_delta(orc_sph* o) {
  const int n = o->n;
  const float *px = o->pos, *py = o->pos + n, *pz = o->pos + 2 * n;
  const float s_corr_k = 1e-6f;
  const float s_den = cubic_spline(0, o->kr, o->kr3);
  const float md = o->spacing / 2.f, S = o->size;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; ++i) {
    float ax = 0, ay = 0, az = 0;
    FOR_NEIGHBOURS(o, px[i], py[i], pz[i], j) {
      const float dx = px[i] - px[j], dy = py[i] - py[j], dz = pz[i] - pz[j];
      float wx, wy, wz;
      spikey_grad(dx, dy, dz, o->kr, o->kr6, &wx, &wy, &wz);
      const float w = poly6(dx, dy, dz, o->kr2, o->kr9);
      const float t = w / s_den;
      const float t2 = t * t;
      const float t4 = t2 * t2;
      const float sc = t4 * (-s_corr_k);
      const float f = o->lambda[i] + o->lambda[j] + sc;
      ax += wx * f / o->rest[i];
      ay += wy * f / o->rest[i];
      az += wz * f / o->rest[i];
    }
    o->delta[i] = ax; o->delta[n + i] = ay; o->delta[2 * n + i] = az;
  }
  for (int i = 0; i < n; ++i)
    for (int k = 0; k < 3; ++k) o->pos[(size_t)k * n + i] = clampf(o->pos[(size_t)k * n + i] + o->delta[(size_t)k * n + i], md, S - md);
}

static void pbf_step(orc_sph* o) { /* Fluid::simulationStep (Fluid_3D_PBF.cu:489-517) */
  const int n = o->n;
  const float dt = o->cfg.timestep / (float)o->cfg.substeps;
  const float md = o->spacing / 2.f, S = o->size;
  sph_sort(o);
  for (int s = 0; s < o->cfg.substeps; ++s) {
    for (int i = 0; i < n; ++i) /* applyForcesImpl, predictPositionImpl (:6-26) */
      for (int k = 0; k < 3; ++k) {
        const size_t q = (size_t)k * n + i;
        o->vel[q] = o->vel[q] + dt * o->cfg.gravity[k];
        o->pos[q] = clampf(o->last[q] + dt * o->vel[q], md, S - md);
      }
    sph_sort(o);
    for (int it = 0; it < o->cfg.iterations; ++it) {
      pbf_lambda(o, 0);
      pbf_delta(o);
    }
    /* updatePositionAndVelocityImpl (:209-267) */
    const float leave = (float)((double)md / ((double)dt * 1e2));
    const float bounce = -0.5f;
    for (int i = 0; i < n; ++i) {
      float p[3], v[3];
      for (int k = 0; k < 3; ++k) {
        const size_t q = (size_t)k * n + i;
        v[k] = (o->pos[q] - o->last[q]) / dt;
        o->last[q] = o->pos[q];
        p[k] = o->pos[q];
      }
      if (p[0] == md) v[0] = v[0] == 0 ? leave : v[0] * bounce;
      if (p[0] >= S - md) v[0] = v[0] == 0 ? -leave : v[0] * bounce;
      if (p[1] <= md) v[1] = v[1] == 0 ? leave : v[1] * bounce;
      if (p[1] >= S - md) v[1] = v[1] == 0 ? -leave : v[1] * bounce;
      if (p[2] <= md) v[2] = v[2] == 0 ? leave : v[2] * bounce;
      if (p[2] >= S - md) v[2] = v[2] == 0 ? -leave : v[2] * bounce;
      for (int k = 0; k < 3; ++k) o->vel[(size_t)k * n + i] = v[k];
    }
  }
}

/* --------------------------------------------------------------- PCISPH */

/* predictVelocityAndPositionImpl (Fluid_3D_PCISPH.cu:32-86) */
static void pci_predict(orc_sph* o, int actual) {
  const int n = o->n;
  const float dt = o->cfg.timestep / (float)o->cfg.substeps;
  const float md = o->spacing / 2, S = o->size;
  const float bounce = -0.0f;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; ++i) {
    float p[3], v[3];
    for (int k = 0; k < 3; ++k) {
      const size_t q = (size_t)k * n + i;
      const float acc = o->cfg.gravity[k] + o->force[q];
      v[k] = o->vel[q] + acc * dt;
      p[k] = o->pos[q] + v[k] * dt;
    }
    for (int k = 0; k < 3; ++k) {
      if (p[k] < md) { p[k] = md; v[k] *= bounce; }
      if (p[k] > S - md) { p[k] = S - md; v[k] *= bounce; }
    }
    float* dp = actual ? o->pos : o->ppos;
    float* dv = actual ? o->vel : o->pvel;
    for (int k = 0; k < 3; ++k) { dp[(size_t)k * n + i] = p[k]; dv[(size_t)k * n + i] = v[k]; }
  }
}

/* predictDensityAndPressureImpl (Fluid_3D_PCISPH.cu:88-159): the cell comes
 * from the position, distances from the predicted positions; the
 * correction coefficient is the constant 50 the kernel ends up using. */
static void pci_density(orc_sph* o, int set_rest) {
  const int n = o->n;
  const float *qx = o->ppos, *qy = o->ppos + n, *qz = o->ppos + 2 * n;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; ++i) {
    const float rho0 = o->rest[i];
    float density = 0;
    FOR_NEIGHBOURS(o, o->pos[i], o->pos[n + i], o->pos[2 * n + i], j) {
      density += poly6(qx[i] - qx[j], qy[i] - qy[j], qz[i] - qz[j], o->kr2, o->kr9);
    }
    o->density[i] = density;
    if (set_rest) o->rest[i] = density;
    const float err = density - rho0;
    const float coeff = 50.0f;
    o->pressure[i] += coeff * err;
  }
}

/* computePressureForceImpl (Fluid_3D_PCISPH.cu:161-202) */
static void pci_force(orc_sph* o) {
  const int n = o->n;
  const float *qx = o->ppos, *qy = o->ppos + n, *qz = o->ppos + 2 * n;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; ++i) {
    float fx = 0, fy = 0, fz = 0;
    const float own = o->pressure[i] / (o->density[i] * o->density[i]);
    FOR_NEIGHBOURS(o, o->pos[i], o->pos[n + i], o->pos[2 * n + i], j) {
      float wx, wy, wz;
      spikey_grad(qx[i] - qx[j], qy[i] - qy[j], qz[i] - qz[j], o->kr, o->kr6, &wx, &wy, &wz);
      const float s = o->pressure[j] / (o->density[j] * o->density[j]) + own;
      fx -= wx * s; fy -= wy * s; fz -= wz * s;
    }
    o->force[i] = fx; o->force[n + i] = fy; o->force[2 * n + i] = fz;
  }
}

static void pci_step(orc_sph* o) { /* Fluid::simulationStep (Fluid_3D_PCISPH.cu:424-448) */
  const int n = o->n;
  for (int s = 0; s < o->cfg.substeps; ++s) {
    sph_sort(o);
    /* computeExternalForcesImpl, initPressureImpl (:13-30): acceleration is
     * the gravity, read in predict */
    memset(o->pressure, 0, sizeof(float) * (size_t)n);
    memset(o->force, 0, sizeof(float) * 3 * (size_t)n);
    for (int it = 0; it < o->cfg.iterations; ++it) {
      pci_predict(o, 0);
      pci_density(o, 0);
      pci_force(o);
    }
    pci_predict(o, 1);
  }
}

/* ------------------------------------------------------------ lifecycle */

orc_sph* orc_sph_create(const aq_sph_config* cfg) {
  if (!cfg || (cfg->method != AQ_SPH_PBF && cfg->method != AQ_SPH_PCISPH) || cfg->substeps <= 0 ||
      cfg->max_particle_count <= 0 || cfg->volume_count < 0 || cfg->volume_count > AQ_MAX_VOLUMES)
    return NULL;
  orc_sph* o = (orc_sph*)calloc(1, sizeof(orc_sph));
  o->cfg = *cfg;
  o->method = cfg->method;
  o->size = 10.f;
  /* init (Fluid_3D_PBF.cu:275-300, Fluid_3D_PCISPH.cu:325-340) */
  const float full = (float)cfg->max_particle_count;
  o->spacing = (float)pow((double)(o->size * o->size * o->size / full), 1.0 / 3.0);
  o->spacing = o->size / ceilf(o->size / o->spacing);
  o->kr = o->spacing * (o->method == AQ_SPH_PBF ? 2.01f : 2.f);
  o->kr2 = o->kr * o->kr;
  o->kr3 = o->kr2 * o->kr;
  o->kr5 = o->kr3 * o->kr2;
  o->kr6 = o->kr2 * o->kr2 * o->kr2;
  o->kr9 = o->kr6 * o->kr2 * o->kr;
  sph_rng rng;
  memset(&rng, 0, sizeof(rng));
  initstate_r(cfg->seed, rng.state, sizeof(rng.state), &rng.rd);
  plist3 pl = {NULL, 0, 0};
  for (int v = 0; v < cfg->volume_count; ++v) {
    if (cfg->volumes[v].shape == AQ_SHAPE_SQUARE) square(o, &rng, &pl, &cfg->volumes[v]);
    else if (cfg->volumes[v].shape == AQ_SHAPE_SPHERE) sphere(o, &rng, &pl, &cfg->volumes[v]);
  }
  const int n = pl.n;
  o->n = n;
  o->gx = (int)ceilf(o->size / o->kr);
  o->gy = o->gx;
  o->gz = o->gx;
  o->cells = o->gx * o->gy * o->gz;
  float** p3[] = {&o->pos, &o->vel, &o->last, &o->delta, &o->force, &o->ppos, &o->pvel};
  for (size_t q = 0; q < sizeof(p3) / sizeof(p3[0]); ++q) *p3[q] = (float*)zalloc(3 * (size_t)n, sizeof(float));
  float** p1[] = {&o->density, &o->rest, &o->lambda, &o->pressure};
  for (size_t q = 0; q < sizeof(p1) / sizeof(p1[0]); ++q) *p1[q] = (float*)zalloc((size_t)n, sizeof(float));
  o->key = (int*)zalloc((size_t)n, sizeof(int));
  o->order = (int*)zalloc((size_t)n, sizeof(int));
  o->start = (int*)zalloc((size_t)o->cells + 1, sizeof(int));
  /* Particle(float3): position = lastPosition = predictedPosition */
  for (int i = 0; i < n; ++i)
    for (int k = 0; k < 3; ++k) {
      const float v = pl.p[3 * (size_t)i + k];
      o->pos[(size_t)k * n + i] = v;
      o->last[(size_t)k * n + i] = v;
      o->ppos[(size_t)k * n + i] = v;
    }
  free(pl.p);
  /* computeRestDensity: sort, then the density kernel with
   * setDensityAsRestDensity / setAsRest (rest density 0 before) */
  sph_sort(o);
  if (o->method == AQ_SPH_PBF) pbf_lambda(o, 1);
  else pci_density(o, 1);
  return o;
}

void orc_sph_destroy(orc_sph* o) {
  if (!o) return;
  void* ptrs[] = {o->pos, o->vel, o->density, o->rest, o->last, o->lambda, o->delta, o->pressure,
                  o->force, o->ppos, o->pvel, o->key, o->order, o->start};
  for (size_t i = 0; i < sizeof(ptrs) / sizeof(ptrs[0]); ++i) free(ptrs[i]);
  free(o);
}

int orc_sph_count(const orc_sph* o) { return o->n; }

void orc_sph_info(const orc_sph* o, float* spacing, float* kernel_radius, int* grid) {
  if (spacing) *spacing = o->spacing;
  if (kernel_radius) *kernel_radius = o->kr;
  if (grid) { grid[0] = o->gx; grid[1] = o->gy; grid[2] = o->gz; }
}

int orc_sph_step(orc_sph* o, int nsteps) {
  for (int s = 0; s < nsteps; ++s) {
    if (o->method == AQ_SPH_PBF) pbf_step(o);
    else pci_step(o);
    o->time += o->cfg.timestep;
  }
  return 0;
}

#define COPY(dst, src, cnt) do { if (dst) memcpy((dst), (src), sizeof(float) * (cnt)); } while (0)

int orc_sph_get(const orc_sph* o, aq_sph_state* s) {
  if (s->particle_count != o->n) return 1;
  const size_t n = (size_t)o->n;
  s->physical_time = o->time;
  COPY(s->position, o->pos, 3 * n);
  COPY(s->velocity, o->vel, 3 * n);
  COPY(s->density, o->density, n);
  COPY(s->rest_density, o->rest, n);
  COPY(s->last_position, o->last, 3 * n);
  COPY(s->lambda, o->lambda, n);
  COPY(s->pressure, o->pressure, n);
  COPY(s->pressure_force, o->force, 3 * n);
  COPY(s->predicted_position, o->ppos, 3 * n);
  COPY(s->predicted_velocity, o->pvel, 3 * n);
  return 0;
}

#define COPYIN(dst, src, cnt) do { if (src) memcpy((dst), (src), sizeof(float) * (cnt)); } while (0)

int orc_sph_set(orc_sph* o, const aq_sph_state* s) {
  if (s->particle_count != o->n) return 1;
  const size_t n = (size_t)o->n;
  o->time = s->physical_time;
  COPYIN(o->pos, s->position, 3 * n);
  COPYIN(o->vel, s->velocity, 3 * n);
  COPYIN(o->density, s->density, n);
  COPYIN(o->rest, s->rest_density, n);
  COPYIN(o->last, s->last_position, 3 * n);
  COPYIN(o->lambda, s->lambda, n);
  COPYIN(o->pressure, s->pressure, n);
  COPYIN(o->force, s->pressure_force, 3 * n);
  COPYIN(o->ppos, s->predicted_position, 3 * n);
  COPYIN(o->pvel, s->predicted_velocity, 3 * n);
  return 0;
}
