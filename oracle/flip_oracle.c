/*
 * CPU oracle of the Aquarius 3D FLIP step — TEST INFRASTRUCTURE ONLY
 * (see flip_oracle.h).  Compile with -ffp-contract=off so that float
 * expressions round exactly as written (the reference's host code has no FMA
 * contraction on x86-64).
 *
 * Reference file:line citations are paths inside AmesingFlank/Aquarius.
 */
#define _DEFAULT_SOURCE
#include "flip_oracle.h"
#include "../aquarius_b200/csrc/mc_table.h"

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define AIR 0   /* CONTENT_AIR   Fluid/MAC_Grid_3D.cuh:15 */
#define FLUID 1 /* CONTENT_FLUID Fluid/MAC_Grid_3D.cuh:16 */
#define SOLID 2 /* CONTENT_SOLID Fluid/MAC_Grid_3D.cuh:17 */

/* glibc rand() state; random_r with a 128-byte TYPE_3 state reproduces
 * srand(seed); rand() exactly.  The reference uses rand() unseeded
 * (Common/Commons.h:3-5), i.e. seed 1. */
typedef struct {
  struct random_data rd;
  char state[128];
} orc_rng;

struct orc_fluid {
  aq_config cfg;
  int sx, sy, sz;
  int C, F;
  float h; /* cellPhysicalSize = gridPhysicalSize / sizeY (Fluid_3D_FLIP.cu:444) */
  double time;
  int n;
  float *pos, *vel, *frac;    /* [3][n], [3][n], [4][n] */
  float *pos2, *vel2, *frac2; /* sort scratch */
  int *hash, *sort_index, *counts;
  int* content;               /* [F] */
  float *velocity, *new_velocity, *nv_tmp; /* [3][F] */
  float *pressure, *p_tmp, *divergence, *density; /* [C] */
  int* pcount;                /* [C] */
  int *has, *has_tmp;         /* [3][C] */
  float *vf, *nvf, *nvf_tmp;  /* [4][C] */
  int *cstart, *cend;         /* [C] */
  /* last solve */
  int iters;
  double rel_res, b_norm;
  int fluid_cells;
  /* rand() state after seeding (ink continues the sequence), ink particles */
  orc_rng rng;
  int n_ink;
  float *ink_pos, *ink_vel; /* [3][n_ink] */
  /* 0: race-free reading of the reference's in-place stages (default);
   * 1: those stages in place, in a serial schedule of the reference's launch
   *    (orc_set_schedule) */
  int schedule;
};

/* ---------------------------------------------------------------- helpers */

static inline int cidx(const orc_fluid* o, int x, int y, int z) {
  return (x * o->sy + y) * o->sz + z;
}
static inline int nidx(const orc_fluid* o, int x, int y, int z) {
  return (x * (o->sy + 1) + y) * (o->sz + 1) + z;
}
static inline int divUp(int a, int b) { /* Common/Commons.h:7-13 */
  if (b == 0) return 1;
  return (a % b != 0) ? (a / b + 1) : (a / b);
}
static inline int imin(int a, int b) { return a < b ? a : b; }
static inline int iclamp(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

int orc_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

void orc_config_default(aq_config* c) {
  /* Fluid/FluidConfig.cuh:20-97 */
  memset(c, 0, sizeof(*c));
  c->volume_count = 2;
  c->volumes[0].shape = AQ_SHAPE_SQUARE;
  c->volumes[1].shape = AQ_SHAPE_SPHERE;
  for (int i = 0; i < 2; ++i) {
    aq_volume* v = &c->volumes[i];
    v->box_min[0] = 0; v->box_min[1] = 0; v->box_min[2] = 0;
    v->box_max[0] = 1; v->box_max[1] = 0.1875f; v->box_max[2] = 1;
    v->ball_center[0] = 0.5f; v->ball_center[1] = 0.75f; v->ball_center[2] = 0.5f;
    v->ball_radius = 0.125f;
    v->phase = 0;
  }
  c->gravity[0] = 0; c->gravity[1] = -9.8f; c->gravity[2] = 0;
  c->phase_count = 2;
  for (int i = 0; i < 4; ++i) c->phase_densities[i] = 1;
  c->diffusion_coeff = 0.001f;
  c->size_x = c->size_y = c->size_z = 50;
  c->pressure_iterations = 100;
  c->diffusion_iterations = 100;
  c->timestep = 0.033f;
  c->flip_coeff = 0.95f;
  c->particle_jitter = 0.05f;
  c->domain_size = 10.f;
  c->seed = 1;
  c->pressure_init = AQ_PRESSURE_CARRY;
  c->solve_mode = AQ_SOLVE_FIXED;
  c->rel_residual = 1e-4f;
  c->max_iterations = 2000;
  c->check_interval = 40;
  c->device = 0;
  c->stream = NULL;
}

/* ----------------------------------------------------- particle seeding */


static float random0to1(orc_rng* r) { /* Common/Commons.h:3-5 */
  int32_t v;
  random_r(&r->rd, &v);
  return (float)v / (float)RAND_MAX;
}

typedef struct {
  float* data; /* interleaved pos xyz + frac xyzw, 7 floats per particle */
  int n, cap;
} plist;

static void plist_push(plist* l, float x, float y, float z, int phase) {
  if (l->n == l->cap) {
    l->cap = l->cap ? l->cap * 2 : 4096;
    l->data = (float*)realloc(l->data, sizeof(float) * 7 * (size_t)l->cap);
  }
  float* p = l->data + 7 * (size_t)l->n;
  p[0] = x; p[1] = y; p[2] = z;
  /* Particle(float3 pos, int phase): one-hot fractions (Fluid_3D_FLIP.cuh:31-47) */
  p[3] = phase == 0 ? 1.f : 0.f;
  p[4] = phase == 1 ? 1.f : 0.f;
  p[5] = phase == 2 ? 1.f : 0.f;
  p[6] = phase == 3 ? 1.f : 0.f;
  l->n++;
}

typedef struct {
  int is_sphere;
  float cx, cy, cz, r;
} seed_filter;

/* Fluid::createParticlesAt (Fluid_3D_FLIP.cu:508-538).  The jitter draws
 * happen before the filter, so filtered-out sub-cells still consume rand(). */
static void create_particles_at(orc_fluid* o, orc_rng* rng, plist* out, float cx, float cy,
                                float cz, const seed_filter* f, float spacing, int phase) {
  const float jit = o->cfg.particle_jitter;
  for (float dx = 0; dx <= 1; ++dx) {
    for (float dy = 0; dy <= 1; ++dy) {
      for (float dz = 0; dz <= 1; ++dz) {
        float px = (float)(dx - 0.5) * spacing + cx;
        float py = (float)(dy - 0.5) * spacing + cy;
        float pz = (float)(dz - 0.5) * spacing + cz;
        float xj = random0to1(rng) - 0.5f;
        float yj = random0to1(rng) - 0.5f;
        float zj = random0to1(rng) - 0.5f;
        px += xj * spacing * jit;
        py += yj * spacing * jit;
        pz += zj * spacing * jit;
        float md = spacing / 2;
        float hx = (float)o->sx * o->h - md, hy = (float)o->sy * o->h - md, hz = (float)o->sz * o->h - md;
        px = fmaxf(md, fminf(hx, px));
        py = fmaxf(md, fminf(hy, py));
        pz = fmaxf(md, fminf(hz, pz));
        int keep = 1;
        if (f->is_sphere) {
          float ex = px - f->cx, ey = py - f->cy, ez = pz - f->cz;
          float len = sqrtf(ex * ex + ey * ey + ez * ez);
          keep = len < f->r * o->h * (float)o->sy;
        }
        if (keep) plist_push(out, px, py, pz, phase);
      }
    }
  }
}

static int check_coord_valid(const float c[3]) { /* Fluid_3D_FLIP.cu:542-550 */
  if (c[0] < 0 || c[1] < 0 || c[2] < 0) return 0;
  if (c[0] > 1 || c[1] > 1 || c[2] > 1) return 0;
  return 1;
}

/* Fluid::createSquareFluid (Fluid_3D_FLIP.cu:552-569): loops z, x, y. */
static void create_square(orc_fluid* o, orc_rng* rng, plist* out, const aq_volume* v) {
  if (!check_coord_valid(v->box_min) || !check_coord_valid(v->box_max)) return;
  seed_filter f = {0, 0, 0, 0, 0};
  for (int z = (int)(v->box_min[2] * (float)o->sz); (float)z < v->box_max[2] * (float)o->sz; ++z)
    for (int x = (int)(v->box_min[0] * (float)o->sx); (float)x < v->box_max[0] * (float)o->sx; ++x)
      for (int y = (int)(v->box_min[1] * (float)o->sy); (float)y < v->box_max[1] * (float)o->sy; ++y)
        create_particles_at(o, rng, out, ((float)x + 0.5f) * o->h, ((float)y + 0.5f) * o->h,
                            ((float)z + 0.5f) * o->h, &f, o->h / 2, v->phase);
}

/* Fluid::createSphereFluid (Fluid_3D_FLIP.cu:571-594): loops y, x, z over all cells. */
static void create_sphere(orc_fluid* o, orc_rng* rng, plist* out, const aq_volume* v) {
  if (!check_coord_valid(v->ball_center)) return;
  seed_filter f;
  f.is_sphere = 1;
  f.cx = v->ball_center[0] * (float)o->sx * o->h;
  f.cy = v->ball_center[1] * (float)o->sy * o->h;
  f.cz = v->ball_center[2] * (float)o->sz * o->h;
  f.r = v->ball_radius;
  for (int y = 0; y < o->sy; ++y)
    for (int x = 0; x < o->sx; ++x)
      for (int z = 0; z < o->sz; ++z)
        create_particles_at(o, rng, out, ((float)x + 0.5f) * o->h, ((float)y + 0.5f) * o->h,
                            ((float)z + 0.5f) * o->h, &f, o->h / 2, v->phase);
}

/* ------------------------------------------------------ grid primitives */

/* fixBoundary (Fluid_3D_common.cu:13-41; kernels Fluid_3D_kernels.cu:44-98).
 * Each launch covers only ceil(s1*s2/1024)*1024 of the (s1+1)(s2+1) faces. */
static int covered_faces(int s1, int s2) {
  int total = s1 * s2;
  int nt = imin(1024, total);
  int nb = divUp(total, nt);
  int t = nb * nt;
  int faces = (s1 + 1) * (s2 + 1);
  return t < faces ? t : faces;
}

static void fix_boundary(orc_fluid* o) {
  const int sx = o->sx, sy = o->sy, sz = o->sz, F = o->F;
  float *u = o->new_velocity, *v = o->new_velocity + F, *w = o->new_velocity + 2 * F;
  int cx = covered_faces(sy, sz);
  for (int i = 0; i < cx; ++i) { /* fixBoundaryX */
    int y = i / (sz + 1), z = i - y * (sz + 1);
    int a = nidx(o, 0, y, z), b = nidx(o, sx, y, z);
    u[a] = fmaxf(0.f, u[a]);
    u[b] = fminf(0.f, u[b]);
    o->content[b] = SOLID;
  }
  int cy = covered_faces(sx, sz);
  for (int i = 0; i < cy; ++i) { /* fixBoundaryY */
    int x = i / (sz + 1), z = i - x * (sz + 1);
    int a = nidx(o, x, 0, z), b = nidx(o, x, sy, z);
    v[a] = fmaxf(0.f, v[a]);
    v[b] = fminf(0.f, v[b]);
    o->content[b] = SOLID;
  }
  int cz = covered_faces(sx, sy);
  for (int i = 0; i < cz; ++i) { /* fixBoundaryZ */
    int x = i / (sy + 1), y = i - x * (sy + 1);
    int a = nidx(o, x, y, 0), b = nidx(o, x, y, sz);
    w[a] = fmaxf(0.f, w[a]);
    w[b] = fminf(0.f, w[b]);
    o->content[b] = SOLID;
  }
}

/* MAC_Grid_3D::getInterpolatedValueAtPoint (MAC_Grid_3D.cuh:66-97) on one
 * component of a node field; lerp(a,b,t) = a + t*(b-a) (helper_math.h). */
static inline float lerpf(float a, float b, float t) { return a + t * (b - a); }

static float interp(const orc_fluid* o, const float* fld, float x, float y, float z) {
  x = fmaxf(fminf(x, (float)o->sx - 1.f), 0.f);
  y = fmaxf(fminf(y, (float)o->sy - 1.f), 0.f);
  z = fmaxf(fminf(z, (float)o->sz - 1.f), 0.f);
  int i = (int)floorf(x), j = (int)floorf(y), k = (int)floorf(z);
  float tx = x - (float)i, ty = y - (float)j, tz = z - (float)k;
  float x0y0 = lerpf(fld[nidx(o, i, j, k)], fld[nidx(o, i, j, k + 1)], tz);
  float x0y1 = lerpf(fld[nidx(o, i, j + 1, k)], fld[nidx(o, i, j + 1, k + 1)], tz);
  float x1y0 = lerpf(fld[nidx(o, i + 1, j, k)], fld[nidx(o, i + 1, j, k + 1)], tz);
  float x1y1 = lerpf(fld[nidx(o, i + 1, j + 1, k)], fld[nidx(o, i + 1, j + 1, k + 1)], tz);
  float x0 = lerpf(x0y0, x0y1, ty);
  float x1 = lerpf(x1y0, x1y1, ty);
  return lerpf(x0, x1, tx);
}

/* getPointVelocity / getPointNewVelocity (MAC_Grid_3D.cuh:100-130). */
static void point_velocity(const orc_fluid* o, const float* f3, float px, float py, float pz,
                           float* ox, float* oy, float* oz) {
  const int F = o->F;
  float x = px / o->h, y = py / o->h, z = pz / o->h;
  *ox = interp(o, f3, x, y - 0.5f, z - 0.5f);
  *oy = interp(o, f3 + F, x - 0.5f, y, z - 0.5f);
  *oz = interp(o, f3 + 2 * F, x - 0.5f, y - 0.5f, z);
}

/* trilinearUnitKernel / trilinearHatKernel (WeightKernels.cuh:131-146). */
static inline float unit_kernel(float r) {
  r = fabsf(r);
  if (r > 1) return 0;
  return 1 - r;
}
static inline float hat(float rx, float ry, float rz, float s) {
  return unit_kernel(rx / s) * unit_kernel(ry / s) * unit_kernel(rz / s);
}

/* ------------------------------------------------------------- stages */

/* transferToParticlesImpl's velocity update (Fluid_3D_FLIP.cu:189-227) with
 * FLIP coefficient c, then moveParticlesImpl (Fluid_3D_FLIP.cu:229-285):
 * Ralston RK3 in newVelocity, clamped to [h/4, s*h - h/4] with the velocity
 * component reflected. */
static void g2p_move(const orc_fluid* o, float c, float dt, float* ppx, float* ppy, float* ppz, float* pvx,
                     float* pvy, float* pvz) {
  const float h = o->h;
  float nx, ny, nz, ox, oy, oz;
  point_velocity(o, o->new_velocity, *ppx, *ppy, *ppz, &nx, &ny, &nz);
  point_velocity(o, o->velocity, *ppx, *ppy, *ppz, &ox, &oy, &oz);
  float dvx = nx - ox, dvy = ny - oy, dvz = nz - oz;
  float fx = *pvx + dvx, fy = *pvy + dvy, fz = *pvz + dvz;
  float vx = c * fx + (1.0f - c) * nx;
  float vy = c * fy + (1.0f - c) * ny;
  float vz = c * fz + (1.0f - c) * nz;
  float bx = *ppx, by = *ppy, bz = *ppz;
  float u1x, u1y, u1z, u2x, u2y, u2z, u3x, u3y, u3z;
  point_velocity(o, o->new_velocity, bx, by, bz, &u1x, &u1y, &u1z);
  point_velocity(o, o->new_velocity, bx + dt * u1x / 2, by + dt * u1y / 2, bz + dt * u1z / 2, &u2x, &u2y, &u2z);
  point_velocity(o, o->new_velocity, bx + dt * u2x * 3 / 4, by + dt * u2y * 3 / 4, bz + dt * u2z * 3 / 4, &u3x,
                 &u3y, &u3z);
  float dx = bx + dt * (u1x * 2 / 9 + u2x * 3 / 9 + u3x * 4 / 9);
  float dy = by + dt * (u1y * 2 / 9 + u2y * 3 / 9 + u3y * 4 / 9);
  float dz = bz + dt * (u1z * 2 / 9 + u2z * 3 / 9 + u3z * 4 / 9);
  float md = h / 4;
  float gx = (float)o->sx * h, gy = (float)o->sy * h, gz = (float)o->sz * h;
  if (dx < md) { dx = md; vx *= -1; }
  if (dx > gx - md) { dx = gx - md; vx *= -1; }
  if (dy < md) { dy = md; vy *= -1; }
  if (dy > gy - md) { dy = gy - md; vy *= -1; }
  if (dz < md) { dz = md; vz *= -1; }
  if (dz > gz - md) { dz = gz - md; vz *= -1; }
  *ppx = dx; *ppy = dy; *ppz = dz;
  *pvx = vx; *pvy = vy; *pvz = vz;
}

/* transferToParticlesImpl (Fluid_3D_FLIP.cu:189-227) then moveParticlesImpl
 * (Fluid_3D_FLIP.cu:229-285), particle by particle. */
static void stage_g2p_advect(orc_fluid* o) {
  const int n = o->n, C = o->C;
  const float h = o->h, c = o->cfg.flip_coeff, dt = o->cfg.timestep;
  float *px = o->pos, *py = o->pos + n, *pz = o->pos + 2 * n;
  float *vx = o->vel, *vy = o->vel + n, *vz = o->vel + 2 * n;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; ++i) {
    /* transferToParticlesImpl: fractions from the cell of the unmoved particle */
    int cx = (int)floorf(px[i] / h), cy = (int)floorf(py[i] / h), cz = (int)floorf(pz[i] / h);
    cx = iclamp(cx, 0, o->sx - 1); cy = iclamp(cy, 0, o->sy - 1); cz = iclamp(cz, 0, o->sz - 1);
    int cell = cidx(o, cx, cy, cz);
    float f0 = o->nvf[cell], f1 = o->nvf[C + cell], f2 = o->nvf[2 * C + cell], f3 = o->nvf[3 * C + cell];
    float sum = f0 * 1 + f1 * 1 + f2 * 1 + f3 * 1;
    if (sum > 0) { f0 /= sum; f1 /= sum; f2 /= sum; f3 /= sum; }
    o->frac[i] = f0; o->frac[n + i] = f1; o->frac[2 * n + i] = f2; o->frac[3 * n + i] = f3;
    g2p_move(o, c, dt, &px[i], &py[i], &pz[i], &vx[i], &vy[i], &vz[i]);
  }
}

static void* xcalloc(size_t n, size_t s) {
  void* p = calloc(n ? n : 1, s);
  return p;
}

/* ------------------------------------------------------------------- ink
 * Ink particles (Fluid_3D_FLIP.cu:600-725, disabled in the reference's
 * step): massless tracers seeded at spacing h/4 over the initial volumes,
 * continuing the fluid seeding's rand() sequence, and advected at the end of
 * a step by transferToParticlesImpl with FLIP coefficient 1 and
 * moveParticlesImpl on the step's grid velocities. */

/* Fluid::createSquareInk (Fluid_3D_FLIP.cu:600-640): a jittered lattice. */
static void create_square_ink(orc_fluid* o, orc_rng* rng, plist* out, const aq_volume* v, float spacing) {
  const float md = spacing / 2.f;
  const float gx = (float)o->sx * o->h, gy = (float)o->sy * o->h, gz = (float)o->sz * o->h;
  const float shrink = (float)((double)md - 1e-3);
  const float x0 = v->box_min[0] * gx + md, y0 = v->box_min[1] * gy + md, z0 = v->box_min[2] * gz + md;
  const float x1 = v->box_max[0] * gx - shrink, y1 = v->box_max[1] * gy - shrink, z1 = v->box_max[2] * gz - shrink;
  for (float x = x0; x <= x1; x += spacing)
    for (float y = y0; y <= y1; y += spacing)
      for (float z = z0; z <= z1; z += spacing) {
        const float mag = spacing / 2.f;
        /* (random0to1() - 0.5) is evaluated in double, then stored as float */
        float jx = (float)((double)random0to1(rng) - 0.5);
        float jy = (float)((double)random0to1(rng) - 0.5);
        float jz = (float)((double)random0to1(rng) - 0.5);
        jx *= mag; jy *= mag; jz *= mag;
        float px = x + jx, py = y + jy, pz = z + jz;
        px = fminf(gx - md, fmaxf(md, px));
        py = fminf(gy - md, fmaxf(md, py));
        pz = fminf(gz - md, fmaxf(md, pz));
        plist_push(out, px, py, pz, v->phase);
      }
}

/* Fluid::createSphereInk (Fluid_3D_FLIP.cu:642-664): createParticlesAt (sub-
 * spacing h/2) at every point of a spacing lattice from 0, loops z, y, x. */
static void create_sphere_ink(orc_fluid* o, orc_rng* rng, plist* out, const aq_volume* v, float spacing) {
  if (!check_coord_valid(v->ball_center)) return;
  seed_filter f;
  f.is_sphere = 1;
  f.cx = v->ball_center[0] * (float)o->sx * o->h;
  f.cy = v->ball_center[1] * (float)o->sy * o->h;
  f.cz = v->ball_center[2] * (float)o->sz * o->h;
  f.r = v->ball_radius;
  const float gx = (float)o->sx * o->h, gy = (float)o->sy * o->h, gz = (float)o->sz * o->h;
  for (float z = 0; z < gz; z += spacing)
    for (float y = 0; y < gy; y += spacing)
      for (float x = 0; x < gx; x += spacing) create_particles_at(o, rng, out, x, y, z, &f, o->h / 2, v->phase);
}

int orc_ink_create(orc_fluid* o) {
  if (o->ink_pos) return o->n_ink;
  plist pl = {NULL, 0, 0};
  const float spacing = o->h / 4;
  for (int i = 0; i < o->cfg.volume_count; ++i) {
    const aq_volume* v = &o->cfg.volumes[i];
    if (v->shape == AQ_SHAPE_SQUARE) create_square_ink(o, &o->rng, &pl, v, spacing);
    else if (v->shape == AQ_SHAPE_SPHERE) create_sphere_ink(o, &o->rng, &pl, v, spacing);
  }
  const int n = pl.n;
  o->n_ink = n;
  o->ink_pos = (float*)xcalloc(3 * (size_t)(n > 0 ? n : 1), sizeof(float));
  o->ink_vel = (float*)xcalloc(3 * (size_t)(n > 0 ? n : 1), sizeof(float));
  for (int i = 0; i < n; ++i)
    for (int d = 0; d < 3; ++d) o->ink_pos[d * n + i] = pl.data[7 * (size_t)i + d];
  free(pl.data);
  return n;
}

int orc_ink_count(const orc_fluid* o) { return o->n_ink; }

void orc_ink_advance(orc_fluid* o) {
  const int n = o->n_ink;
  float *p = o->ink_pos, *v = o->ink_vel;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; ++i)
    g2p_move(o, 1.0f, o->cfg.timestep, &p[i], &p[n + i], &p[2 * n + i], &v[i], &v[n + i], &v[2 * n + i]);
}

void orc_ink_get(const orc_fluid* o, float* pos, float* vel) {
  const size_t n = (size_t)o->n_ink;
  if (pos) memcpy(pos, o->ink_pos, sizeof(float) * 3 * n);
  if (vel) memcpy(vel, o->ink_vel, sizeof(float) * 3 * n);
}

void orc_ink_set(orc_fluid* o, const float* pos, const float* vel) {
  const size_t n = (size_t)o->n_ink;
  if (pos) memcpy(o->ink_pos, pos, sizeof(float) * 3 * n);
  if (vel) memcpy(o->ink_vel, vel, sizeof(float) * 3 * n);
}

/* ---------------------------------------------------------------- mesher
 * The surface mesher (Rendering/Renderer3D/Mesher.cuh:20-178,
 * Mesher.cu:321-630) as Fluid::init builds it (Fluid_3D_FLIP.cu:495):
 * container = size * h, particle spacing h/2.  A particle SDF on a grid of
 * cell h/2 (computeSDF: a dunfanKernel-weighted mean of the particles near a
 * cell centre, minus the particle radius), then marching cubes on a fixed
 * 128^3 grid spanning the container's x extent, sampling the SDF by
 * trilinear interpolation.  Output: one record per occupied cube in cube
 * order, 15 slots of (position, normal), unused slots zero. */

void orc_mesh_dims_of(const orc_fluid* o, orc_mesh_dims* m) {
  const float h = o->h;
  const float cx = (float)o->sx * h, cy = (float)o->sy * h, cz = (float)o->sz * h;
  const float spacing = h / 2; /* Mesher(containerSize, cellPhysicalSize / 2, ...) */
  m->h_sdf = spacing;          /* Mesher.cu:583-584 */
  m->radius = spacing;
  m->mesh[0] = m->mesh[1] = m->mesh[2] = 128; /* Mesher.cuh:104-106 */
  m->h_mesh = cx / (float)(128 - 2);          /* Mesher.cu:587 */
  m->sdf[0] = (int)(3 + cx / m->h_sdf);        /* Mesher.cu:589-591 */
  m->sdf[1] = (int)(3 + cy / m->h_sdf);
  m->sdf[2] = (int)(3 + cz / m->h_sdf);
}

/* dunfanKernel (Fluid/WeightKernels.cuh:183-189) */
static inline float dunfan(float rx, float ry, float rz, float support) {
  const float r2 = rx * rx + ry * ry + rz * rz;
  const float h2 = support * support;
  if (r2 > h2) return 0;
  const float t = 1.f - r2 / (h2 * 3.f);
  return fmaxf(0.f, t * t * t);
}

/* computeSDF (Mesher.cuh:20-84) after performSpatialHashing2 on the SDF grid
 * (Mesher.cuh:160): particles stably sorted by their SDF hash cell, then per
 * SDF cell the 4x4x4 hash cells x-3..x (flat index, as the reference walks
 * them) in order.  sdf: [sx][sy][sz] of the SDF grid, z fastest. */
static void mesh_sdf(const orc_fluid* o, const orc_mesh_dims* m, float* sdf) {
  const int n = o->n;
  const float hs = m->h_sdf;
  const int HX = m->sdf[0] - 2, HY = m->sdf[1] - 2, HZ = m->sdf[2] - 2;
  const long long HC = (long long)HX * HY * HZ;
  const int SX = m->sdf[0], SY = m->sdf[1], SZ = m->sdf[2];
  const long long SC = (long long)SX * SY * SZ;
  const float *px = o->pos, *py = o->pos + n, *pz = o->pos + 2 * n;
  int* key = (int*)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
  int* start = (int*)calloc((size_t)HC + 1, sizeof(int));
  int* order = (int*)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
  for (int i = 0; i < n; ++i) { /* calcHashImpl (Fluid_3D_kernels.cuh:8-27) */
    const int x = (int)(px[i] / hs), y = (int)(py[i] / hs), z = (int)(pz[i] / hs);
    key[i] = x * (HY * HZ) + y * HZ + z;
    start[key[i] + 1]++;
  }
  for (long long c = 0; c < HC; ++c) start[c + 1] += start[c];
  {
    int* fill = (int*)malloc(sizeof(int) * (size_t)HC);
    memcpy(fill, start, sizeof(int) * (size_t)HC);
    for (int i = 0; i < n; ++i) order[fill[key[i]]++] = i; /* stable */
    free(fill);
  }
  const float R = hs * 2.f;
#pragma omp parallel for schedule(static)
  for (long long idx = 0; idx < SC; ++idx) {
    const int x = (int)(idx / ((long long)SY * SZ));
    const int y = (int)((idx / SZ) % SY);
    const int z = (int)(idx % SZ);
    const float cx = (float)(x - 1) * hs, cy = (float)(y - 1) * hs, cz = (float)(z - 1) * hs;
    float sw = 0, sx_ = 0, sy_ = 0, sz_ = 0;
    for (int dx = -2; dx <= 1; ++dx)
      for (int dy = -2; dy <= 1; ++dy)
        for (int dz = -2; dz <= 1; ++dz) {
          const long long cell = (long long)(x + dx - 1) * HY * HZ + (long long)(y + dy - 1) * HZ + (z + dz - 1);
          if (cell < 0 || cell >= SC || cell >= HC) continue; /* cells past the hash grid are empty */
          for (int j = start[cell]; j < start[cell + 1]; ++j) {
            const int p = order[j];
            const float w = dunfan(px[p] - cx, py[p] - cy, pz[p] - cz, R);
            sw += w;
            sx_ += w * px[p];
            sy_ += w * py[p];
            sz_ += w * pz[p];
          }
        }
    float v = hs; /* "set to some positive value first" */
    if (sw != 0) {
      const float mx = sx_ / sw, my = sy_ / sw, mz = sz_ / sw;
      const float ex = mx - cx, ey = my - cy, ez = mz - cz;
      v = sqrtf(ex * ex + ey * ey + ez * ez) - m->radius;
    }
    sdf[((size_t)x * SY + y) * SZ + z] = v;
  }
  free(key);
  free(start);
  free(order);
}

/* tex3D on the SDF (linear filter, unnormalised coordinates, border in x,
 * clamp in y and z; Mesher.cu:627, Fluid/VolumeData.cuh:44-76): texel
 * centres at i + 0.5.  The texture unit filters with 8-bit fixed-point
 * weights (CUDA Programming Guide, "Linear Filtering": 9-bit fixed point with
 * 8 fractional bits).  The weights below are a model of what it returns,
 * fitted to probes of the reference's own texture (tests/golden/
 * texture_linear_probe.npz): per axis the fraction rounded half up to 1/256;
 * per texel the x and z weights multiplied and rounded half down to 1/256,
 * then the y weight, rounded half up.  It reproduces the probes exactly for
 * about 92% of samples and within 1.3% of the texel range for the rest. */
static float tex_linear(int SX, int SY, int SZ, const float* t, float cx, float cy, float cz) {
  const float xb = cx - 0.5f, yb = cy - 0.5f, zb = cz - 0.5f;
  const float fx = floorf(xb), fy = floorf(yb), fz = floorf(zb);
  const float qa = floorf((xb - fx) * 256.f + 0.5f), qb = floorf((yb - fy) * 256.f + 0.5f),
              qc = floorf((zb - fz) * 256.f + 0.5f);
  const int i = (int)fx, j = (int)fy, k = (int)fz;
  float v = 0.f;
  for (int di = 0; di < 2; ++di)
    for (int dj = 0; dj < 2; ++dj)
      for (int dk = 0; dk < 2; ++dk) {
        const int ii = i + di, jj = iclamp(j + dj, 0, SY - 1), kk = iclamp(k + dk, 0, SZ - 1);
        const float T = (ii < 0 || ii >= SX) ? 0.f : t[((size_t)ii * SY + jj) * SZ + kk];
        const float wx = di ? qa : 256.f - qa, wy = dj ? qb : 256.f - qb, wz = dk ? qc : 256.f - qc;
        const float wxz = ceilf(wx * wz / 256.f - 0.5f);
        const float w = floorf(wxz * wy / 256.f + 0.5f);
        v += (w / 256.f) * T;
      }
  return v;
}

static float sdf_sample(const orc_mesh_dims* m, const float* sdf, float cx, float cy, float cz) {
  return tex_linear(m->sdf[0], m->sdf[1], m->sdf[2], sdf, cx, cy, cz);
}

/* The same filter on any [w][h][d] field (z fastest), for the probe test. */
void orc_tex_linear(const float* field, int w, int h, int d, const float* coords, float* out, int n) {
  for (int q = 0; q < n; ++q) out[q] = tex_linear(w, h, d, field, coords[3 * q], coords[3 * q + 1], coords[3 * q + 2]);
}

/* getSDF on mesh vertices (Mesher.cu:294-308): 0 on the two outer layers. */
static float mesh_vertex_sdf(const orc_mesh_dims* m, const float* sdf, int x, int y, int z) {
  if (x == 0 || y == 0 || z == 0 || x >= m->mesh[0] - 1 || y >= m->mesh[1] - 1 || z >= m->mesh[2] - 1) return 0;
  const float hm = m->h_mesh, hs = m->h_sdf;
  const float px = (float)(x - 1) * hm, py = (float)(y - 1) * hm, pz = (float)(z - 1) * hm;
  return sdf_sample(m, sdf, 1.f + px / hs, 1.f + py / hs, 1.f + pz / hs);
}

/* getSDF at a world position (Mesher.cu:312-318). */
static float mesh_point_sdf(const orc_mesh_dims* m, const float* sdf, float px, float py, float pz) {
  const float hs = m->h_sdf;
  return sdf_sample(m, sdf, 1.f + px / hs, 1.f + py / hs, 1.f + pz / hs);
}

/* marchingCubes (Mesher.cu:322-425) for one cube into rec[90]. */
static void mesh_cube(const orc_mesh_dims* m, const float* sdf, int x, int y, int z, int type, float* rec) {
  const uint64_t row = AQ_MC_TRIANGLES[type];
  const float hm = m->h_mesh;
  const float bx = (float)(x - 1) * hm, by = (float)(y - 1) * hm, bz = (float)(z - 1) * hm;
  for (int i = 0; i < 15; ++i) {
    float* out = rec + 6 * i;
    const int e = aq_mc_entry(row, i);
    if (e < 0) {
      for (int k = 0; k < 6; ++k) out[k] = 0;
      continue;
    }
    const int* ca = AQ_MC_VERTEX[AQ_MC_EDGE[e][0]];
    const int* cb = AQ_MC_VERTEX[AQ_MC_EDGE[e][1]];
    const float sa = mesh_vertex_sdf(m, sdf, ca[0] + x, ca[1] + y, ca[2] + z);
    const float sb = mesh_vertex_sdf(m, sdf, cb[0] + x, cb[1] + y, cb[2] + z);
    const float f = -sa / (sb - sa);
    const float g = 1.f - f;
    const float px = bx + ((float)ca[0] * g + (float)cb[0] * f) * hm;
    const float py = by + ((float)ca[1] * g + (float)cb[1] * f) * hm;
    const float pz = bz + ((float)ca[2] * g + (float)cb[2] * f) * hm;
    const float d = hm / 2;
    const float l = mesh_point_sdf(m, sdf, px + -d, py, pz), r = mesh_point_sdf(m, sdf, px + d, py, pz);
    const float u = mesh_point_sdf(m, sdf, px, py + d, pz), dn = mesh_point_sdf(m, sdf, px, py + -d, pz);
    const float fr = mesh_point_sdf(m, sdf, px, py, pz + d), bk = mesh_point_sdf(m, sdf, px, py, pz + -d);
    const float nx = r - l, ny = u - dn, nz = fr - bk;
    const float inv = 1.f / sqrtf(nx * nx + ny * ny + nz * nz);
    out[0] = px; out[1] = py; out[2] = pz;
    out[3] = nx * inv; out[4] = ny * inv; out[5] = nz * inv;
  }
}

int orc_mesh(orc_fluid* o, float* sdf_out, float* records, long long capacity, int* cubes) {
  orc_mesh_dims m;
  orc_mesh_dims_of(o, &m);
  const size_t SCn = (size_t)m.sdf[0] * m.sdf[1] * m.sdf[2];
  float* sdf = (float*)malloc(sizeof(float) * SCn);
  if (!sdf) return 1;
  mesh_sdf(o, &m, sdf);
  const int MX = m.mesh[0], MY = m.mesh[1], MZ = m.mesh[2];
  const int VY = MY + 1, VZ = MZ + 1;
  const size_t NV = (size_t)(MX + 1) * VY * VZ;
  float* vv = (float*)malloc(sizeof(float) * NV);
  if (!vv) { free(sdf); return 1; }
#pragma omp parallel for schedule(static)
  for (long long idx = 0; idx < (long long)NV; ++idx) {
    const int x = (int)(idx / ((long long)VY * VZ)), y = (int)((idx / VZ) % VY), z = (int)(idx % VZ);
    vv[idx] = mesh_vertex_sdf(&m, sdf, x, y, z);
  }
  long long count = 0;
  for (int x = 0; x < MX; ++x)
    for (int y = 0; y < MY; ++y)
      for (int z = 0; z < MZ; ++z) {
        int type = 0;
        for (int v = 0; v < 8; ++v) {
          const int* c = AQ_MC_VERTEX[v];
          if (vv[((size_t)(x + c[0]) * VY + (y + c[1])) * VZ + (z + c[2])] < 0) type |= 1 << v;
        }
        if (type == 0 || type == 255) continue; /* rows without triangles */
        if (records && count < capacity) mesh_cube(&m, sdf, x, y, z, type, records + 90 * (size_t)count);
        ++count;
      }
  if (cubes) *cubes = (int)count;
  if (sdf_out) memcpy(sdf_out, sdf, sizeof(float) * SCn);
  free(vv);
  free(sdf);
  return 0;
}

/* performSpatialHashing2 (Fluid_3D_common.cuh:27-56): calcHashImpl
 * (Fluid_3D_kernels.cuh:8-27), a stable sort of indices by hash (thrust
 * sort_by_key, a stable radix sort), applySortImpl (:95-102) and
 * findCellStartEndImpl (Fluid_kernels.cuh:3-22, inclusive end). */
static void stage_sort(orc_fluid* o) {
  const int n = o->n, C = o->C, sy = o->sy, sz = o->sz;
  const float h = o->h;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; ++i) {
    int x = (int)(o->pos[i] / h);
    int y = (int)(o->pos[n + i] / h);
    int z = (int)(o->pos[2 * n + i] / h);
    o->hash[i] = x * (sy * sz) + y * sz + z;
  }
  memset(o->counts, 0, sizeof(int) * (size_t)C);
  for (int i = 0; i < n; ++i) o->counts[o->hash[i]]++;
  int run = 0;
  for (int c = 0; c < C; ++c) {
    int k = o->counts[c];
    o->cstart[c] = k ? run : -1;
    o->cend[c] = k ? run + k - 1 : -1;
    o->counts[c] = run; /* next free slot */
    run += k;
  }
  for (int i = 0; i < n; ++i) o->sort_index[o->counts[o->hash[i]]++] = i;
#pragma omp parallel for schedule(static)
  for (int k = 0; k < n; ++k) {
    int s = o->sort_index[k];
    for (int d = 0; d < 3; ++d) {
      o->pos2[d * n + k] = o->pos[d * n + s];
      o->vel2[d * n + k] = o->vel[d * n + s];
    }
    for (int d = 0; d < 4; ++d) o->frac2[d * n + k] = o->frac[d * n + s];
  }
  float* t;
  t = o->pos; o->pos = o->pos2; o->pos2 = t;
  t = o->vel; o->vel = o->vel2; o->vel2 = t;
  t = o->frac; o->frac = o->frac2; o->frac2 = t;
  /* particleHashes end up sorted */
  for (int c = 0, k = 0; c < C; ++c)
    for (int e = o->cstart[c]; e >= 0 && e <= o->cend[c]; ++e) o->hash[k++] = c;
}

/* resetCellImpl, transferToCellAccumPhase, transferToCellDividePhase,
 * transferVolumeFractionsToCell (Fluid_3D_FLIP.cu:8-166, 287-302) and, when
 * forces is set, applyGravityImpl (Fluid_3D_kernels.cu:4-39) and fixBoundary. */
static void stage_p2g(orc_fluid* o, int forces) {
  const int sx = o->sx, sy = o->sy, sz = o->sz, C = o->C, F = o->F, n = o->n;
  const float h = o->h;
  const float* pxa = o->pos;
  const float* pya = o->pos + n;
  const float* pza = o->pos + 2 * n;
  /* resetCellImpl: [0,s) only; the s-th layer keeps its values */
#pragma omp parallel for schedule(static)
  for (int x = 0; x < sx; ++x)
    for (int y = 0; y < sy; ++y)
      for (int z = 0; z < sz; ++z) {
        int ni = nidx(o, x, y, z), ci = cidx(o, x, y, z);
        o->content[ni] = AIR;
        for (int d = 0; d < 3; ++d) {
          o->has[d * C + ci] = 0;
          o->velocity[d * F + ni] = 0;
          o->new_velocity[d * F + ni] = 0;
        }
      }
#pragma omp parallel for schedule(static)
  for (int x = 0; x < sx; ++x)
    for (int y = 0; y < sy; ++y)
      for (int z = 0; z < sz; ++z) {
        /* transferToCellAccumPhase */
        float ux = (float)x * h, uy = (float)(y + 0.5) * h, uz = (float)(z + 0.5) * h;
        float vxp = (float)(x + 0.5) * h, vyp = (float)y * h, vzp = (float)(z + 0.5) * h;
        float wxp = (float)(x + 0.5) * h, wyp = (float)(y + 0.5) * h, wzp = (float)z * h;
        float sv0 = 0, sv1 = 0, sv2 = 0, w0 = 0, w1 = 0, w2 = 0;
        for (int dx = -1; dx <= 1; ++dx)
          for (int dy = -1; dy <= 1; ++dy)
            for (int dz = -1; dz <= 1; ++dz) {
              int cell = (x + dx) * sy * sz + (y + dy) * sz + z + dz;
              if (cell >= 0 && cell < C) {
                for (int j = o->cstart[cell]; j <= o->cend[cell]; ++j) {
                  if (j >= 0 && j < n) {
                    float px = pxa[j], py = pya[j], pz = pza[j];
                    float wx = hat(px - ux, py - uy, pz - uz, h);
                    float wy = hat(px - vxp, py - vyp, pz - vzp, h);
                    float wz = hat(px - wxp, py - wyp, pz - wzp, h);
                    sv0 += wx * o->vel[j];
                    sv1 += wy * o->vel[n + j];
                    sv2 += wz * o->vel[2 * n + j];
                    w0 += wx; w1 += wy; w2 += wz;
                  }
                }
              }
            }
        /* transferToCellDividePhase */
        int ni = nidx(o, x, y, z), ci = cidx(o, x, y, z);
        if (w0 > 0) { sv0 /= w0; o->has[ci] = 1; }
        if (w1 > 0) { sv1 /= w1; o->has[C + ci] = 1; }
        if (w2 > 0) { sv2 /= w2; o->has[2 * C + ci] = 1; }
        o->velocity[ni] = sv0; o->velocity[F + ni] = sv1; o->velocity[2 * F + ni] = sv2;
        o->new_velocity[ni] = sv0; o->new_velocity[F + ni] = sv1; o->new_velocity[2 * F + ni] = sv2;
        for (int j = o->cstart[ci]; j <= o->cend[ci]; ++j) {
          if (j >= 0 && j < n) { o->content[ni] = FLUID; break; }
        }
        /* transferVolumeFractionsToCell: own cell only */
        float cxp = (float)(x + 0.5) * h, cyp = (float)(y + 0.5) * h, czp = (float)(z + 0.5) * h;
        float f0 = 0, f1 = 0, f2 = 0, f3 = 0, wt = 0;
        for (int j = o->cstart[ci]; j <= o->cend[ci]; ++j) {
          if (j >= 0 && j < n) {
            float tw = hat(pxa[j] - cxp, pya[j] - cyp, pza[j] - czp, h);
            f0 += tw * o->frac[j]; f1 += tw * o->frac[n + j];
            f2 += tw * o->frac[2 * n + j]; f3 += tw * o->frac[3 * n + j];
            wt += tw;
          }
        }
        if (wt > 0) {
          f0 /= wt; f1 /= wt; f2 /= wt; f3 /= wt;
          float s = f0 + f1 + f2 + f3;
          f0 /= s; f1 /= s; f2 /= s; f3 /= s;
        }
        const float* d = o->cfg.phase_densities;
        o->density[ci] = d[0] * f0 + d[1] * f1 + d[2] * f2 + d[3] * f3;
        o->vf[ci] = o->nvf[ci] = f0; o->vf[C + ci] = o->nvf[C + ci] = f1;
        o->vf[2 * C + ci] = o->nvf[2 * C + ci] = f2; o->vf[3 * C + ci] = o->nvf[3 * C + ci] = f3;
      }
  if (!forces) return;
  /* applyGravityImpl.  The reference's read-modify-write of neighbour faces
   * races when more than one gravity component is nonzero; here each add is
   * applied once.  Own and neighbour adds are exclusive (FLUID vs AIR). */
  const float dt = o->cfg.timestep;
  const float gdx = o->cfg.gravity[0] * dt, gdy = o->cfg.gravity[1] * dt, gdz = o->cfg.gravity[2] * dt;
  float *u = o->new_velocity, *v = o->new_velocity + F, *w = o->new_velocity + 2 * F;
  for (int x = 0; x < sx; ++x)
    for (int y = 0; y < sy; ++y)
      for (int z = 0; z < sz; ++z) {
        int ni = nidx(o, x, y, z);
        if (o->content[ni] != FLUID) continue;
        u[ni] += gdx; v[ni] += gdy; w[ni] += gdz;
        int nb;
        nb = nidx(o, x + 1, y, z);
        if (o->content[nb] == AIR && o->cfg.gravity[0] != 0) { u[nb] += gdx; v[nb] += gdy; w[nb] += gdz; }
        nb = nidx(o, x, y + 1, z);
        if (o->content[nb] == AIR && o->cfg.gravity[1] != 0) { u[nb] += gdx; v[nb] += gdy; w[nb] += gdz; }
        nb = nidx(o, x, y, z + 1);
        if (o->content[nb] == AIR && o->cfg.gravity[2] != 0) { u[nb] += gdx; v[nb] += gdy; w[nb] += gdz; }
      }
  fix_boundary(o);
}

/* countParticlesInCellsImpl (Fluid_3D_FLIP.cu:168-186) and
 * computeDivergenceImpl (Fluid_3D_kernels.cu:426-458). */
static void stage_divergence(orc_fluid* o) {
  const int sx = o->sx, sy = o->sy, sz = o->sz, F = o->F;
  const float *u = o->new_velocity, *v = o->new_velocity + F, *w = o->new_velocity + 2 * F;
#pragma omp parallel for schedule(static)
  for (int x = 0; x < sx; ++x)
    for (int y = 0; y < sy; ++y)
      for (int z = 0; z < sz; ++z) {
        int ci = cidx(o, x, y, z), ni = nidx(o, x, y, z);
        int count = o->cend[ci] - o->cstart[ci];
        o->pcount[ci] = count;
        float div = v[nidx(o, x, y + 1, z)] - v[ni] + u[nidx(o, x + 1, y, z)] - u[ni] +
                    w[nidx(o, x, y, z + 1)] - w[ni];
        div = (float)((double)div - (double)((float)count - 8.0f) * 0.001);
        o->divergence[ci] = div;
      }
}

/* Jacobi update of one cell with Neumann (clamped) out-of-domain neighbours
 * and Dirichlet 0 at air (jacobiImpl, Fluid_3D_kernels.cu:460-505). */
static inline float jacobi_cell(const orc_fluid* o, const float* p, int x, int y, int z, float rhs) {
  const int sx = o->sx, sy = o->sy, sz = o->sz;
  float self = p[cidx(o, x, y, z)];
  float s = 0;
  s += x + 1 < sx ? p[cidx(o, x + 1, y, z)] : self;
  s += x - 1 >= 0 ? p[cidx(o, x - 1, y, z)] : self;
  s += y + 1 < sy ? p[cidx(o, x, y + 1, z)] : self;
  s += y - 1 >= 0 ? p[cidx(o, x, y - 1, z)] : self;
  s += z + 1 < sz ? p[cidx(o, x, y, z + 1)] : self;
  s += z - 1 >= 0 ? p[cidx(o, x, y, z - 1)] : self;
  s += rhs;
  s /= 6;
  return s;
}

static inline int content_cell(const orc_fluid* o, int x, int y, int z) {
  return o->content[nidx(o, x, y, z)];
}

/* ||b - A p||^2 and ||b||^2 over fluid cells in FP64, A_ii = 6 - n_out,
 * A_ij = -1 for in-domain neighbours (air p = 0), b = -div * density.
 * Deterministic: per-x partial sums added in x order. */
static void residual_sums(const orc_fluid* o, const float* p, double* rr, double* bb, int* nf) {
  const int sx = o->sx, sy = o->sy, sz = o->sz;
  double* pr = (double*)calloc((size_t)sx * 2, sizeof(double));
  int* pn = (int*)calloc((size_t)sx, sizeof(int));
#pragma omp parallel for schedule(static)
  for (int x = 0; x < sx; ++x) {
    double a = 0, b = 0;
    int k = 0;
    for (int y = 0; y < sy; ++y)
      for (int z = 0; z < sz; ++z) {
        if (content_cell(o, x, y, z) == AIR) continue;
        int ci = cidx(o, x, y, z);
        double self = p[ci];
        double rhs = (double)(-o->divergence[ci] * o->density[ci]);
        double s = 0;
        s += x + 1 < sx ? (double)p[cidx(o, x + 1, y, z)] : self;
        s += x - 1 >= 0 ? (double)p[cidx(o, x - 1, y, z)] : self;
        s += y + 1 < sy ? (double)p[cidx(o, x, y + 1, z)] : self;
        s += y - 1 >= 0 ? (double)p[cidx(o, x, y - 1, z)] : self;
        s += z + 1 < sz ? (double)p[cidx(o, x, y, z + 1)] : self;
        s += z - 1 >= 0 ? (double)p[cidx(o, x, y, z - 1)] : self;
        double r = rhs + s - 6.0 * self;
        a += r * r;
        b += rhs * rhs;
        k++;
      }
    pr[2 * x] = a; pr[2 * x + 1] = b; pn[x] = k;
  }
  double a = 0, b = 0;
  int k = 0;
  for (int x = 0; x < sx; ++x) { a += pr[2 * x]; b += pr[2 * x + 1]; k += pn[x]; }
  free(pr); free(pn);
  *rr = a; *bb = b; *nf = k;
}

void orc_set_schedule(orc_fluid* o, int schedule) { o->schedule = schedule == 1 ? 1 : 0; }

double orc_pressure_residual(const orc_fluid* o) {
  double rr, bb;
  int nf;
  residual_sums(o, o->pressure, &rr, &bb, &nf);
  return bb > 0 ? sqrt(rr) / sqrt(bb) : 0.0;
}

static void jacobi_sweep(orc_fluid* o, const float* pin, float* pout) {
  const int sx = o->sx, sy = o->sy, sz = o->sz;
#pragma omp parallel for schedule(static)
  for (int x = 0; x < sx; ++x)
    for (int y = 0; y < sy; ++y)
      for (int z = 0; z < sz; ++z) {
        int ci = cidx(o, x, y, z);
        if (content_cell(o, x, y, z) == AIR) { pout[ci] = 0.f; continue; }
        float rhs = -o->divergence[ci] * o->density[ci];
        pout[ci] = jacobi_cell(o, pin, x, y, z, rhs);
      }
}

/* The reference's launch of its grid kernels (MAC_Grid_3D.cu:48): blocks of
 * 8^3 threads, threadIdx.x along x, a grid of divUp(s+1, 8) blocks per axis.
 * A warp is 32 consecutive threads: 8 x by 4 y of one z.  Serial schedule:
 * blocks in launch order (x fastest), a block's 16 warps in order, each warp
 * doing every read before any write (lockstep).  It is one of the outcomes
 * the reference's in-place stencils allow when a launch's threads read cells
 * other threads write (jacobiImpl, extrapolateVelocityByOne): each read sees
 * every update of the warps before it, the opposite extreme of the race-free
 * reading in which no read sees an update of its own launch.
 * Calls f(o, x, y, z, k) for the 32 threads of each warp with k = 0..31 in
 * the read phase, then w(o, x, y, z, k) in the write phase. */
typedef void (*serial_read_fn)(orc_fluid* o, int x, int y, int z, int k, void* scratch);
typedef void (*serial_write_fn)(orc_fluid* o, int x, int y, int z, int k, void* scratch);
static void serial_launch(orc_fluid* o, serial_read_fn rd, serial_write_fn wr, void* scratch) {
  const int gx = divUp(o->sx + 1, 8), gy = divUp(o->sy + 1, 8), gz = divUp(o->sz + 1, 8);
  for (int bz = 0; bz < gz; ++bz)
    for (int by = 0; by < gy; ++by)
      for (int bx = 0; bx < gx; ++bx)
        for (int w = 0; w < 16; ++w) {
          const int tz = w >> 1, ty0 = (w & 1) * 4;
          for (int phase = 0; phase < 2; ++phase)
            for (int k = 0; k < 32; ++k) {
              const int x = bx * 8 + (k & 7), y = by * 8 + ty0 + (k >> 3), z = bz * 8 + tz;
              if (x >= o->sx || y >= o->sy || z >= o->sz) continue;
              if (phase == 0) rd(o, x, y, z, k, scratch);
              else wr(o, x, y, z, k, scratch);
            }
        }
}

static void jacobi_serial_read(orc_fluid* o, int x, int y, int z, int k, void* scratch) {
  float* v = (float*)scratch;
  const int ci = cidx(o, x, y, z);
  if (content_cell(o, x, y, z) == AIR) { v[k] = 0.f; return; }
  v[k] = jacobi_cell(o, o->pressure, x, y, z, -o->divergence[ci] * o->density[ci]);
}
static void jacobi_serial_write(orc_fluid* o, int x, int y, int z, int k, void* scratch) {
  o->pressure[cidx(o, x, y, z)] = ((float*)scratch)[k];
}

/* solvePressureJacobi (Fluid_3D_common.cu:48-55), ping-pong.  RESIDUAL mode
 * sweeps in blocks of check_interval and stops once the FP64 relative
 * residual of the current iterate is <= rel_residual or max_iterations. */
static void stage_pressure(orc_fluid* o) {
  const int C = o->C;
  if (o->cfg.pressure_init == AQ_PRESSURE_ZERO) memset(o->pressure, 0, sizeof(float) * (size_t)C);
  for (int x = 0; x < o->sx; ++x)
    for (int y = 0; y < o->sy; ++y)
      for (int z = 0; z < o->sz; ++z)
        if (content_cell(o, x, y, z) == AIR) o->pressure[cidx(o, x, y, z)] = 0.f;
  int iters = 0;
  double rr, bb;
  int nf;
  if (o->cfg.solve_mode == AQ_SOLVE_RESIDUAL) {
    const int m = o->cfg.check_interval > 0 ? o->cfg.check_interval : 1;
    const double tol = (double)o->cfg.rel_residual;
    double rel = -1;
    for (;;) {
      for (int k = 0; k < m; ++k) {
        jacobi_sweep(o, o->pressure, o->p_tmp);
        float* t = o->pressure; o->pressure = o->p_tmp; o->p_tmp = t;
      }
      iters += m;
      residual_sums(o, o->pressure, &rr, &bb, &nf);
      rel = bb > 0 ? sqrt(rr) / sqrt(bb) : 0.0;
      if (!(rel > tol) || iters >= o->cfg.max_iterations) break;
    }
    o->rel_res = rel;
  } else {
    for (int k = 0; k < o->cfg.pressure_iterations; ++k) {
      if (o->schedule == 1) {
        float v[32];
        serial_launch(o, jacobi_serial_read, jacobi_serial_write, v);
        continue;
      }
      jacobi_sweep(o, o->pressure, o->p_tmp);
      float* t = o->pressure; o->pressure = o->p_tmp; o->p_tmp = t;
    }
    iters = o->cfg.pressure_iterations;
    residual_sums(o, o->pressure, &rr, &bb, &nf);
    o->rel_res = bb > 0 ? sqrt(rr) / sqrt(bb) : 0.0;
  }
  residual_sums(o, o->pressure, &rr, &bb, &nf);
  o->iters = iters;
  o->b_norm = sqrt(bb);
  o->fluid_cells = nf;
}

/* updateVelocityWithPressureImpl (Fluid_3D_kernels.cu:118-207). */
static void stage_project(orc_fluid* o) {
  const int sx = o->sx, sy = o->sy, sz = o->sz, C = o->C, F = o->F;
  float *u = o->new_velocity, *v = o->new_velocity + F, *w = o->new_velocity + 2 * F;
#pragma omp parallel for schedule(static)
  for (int x = 0; x < sx; ++x)
    for (int y = 0; y < sy; ++y)
      for (int z = 0; z < sz; ++z) {
        int ci = cidx(o, x, y, z), ni = nidx(o, x, y, z);
        int hx = 0, hy = 0, hz = 0;
        int c = content_cell(o, x, y, z);
        float p = o->pressure[ci], d = o->density[ci];
        if (x > 0) {
          int lc = content_cell(o, x - 1, y, z);
          float lp = o->pressure[cidx(o, x - 1, y, z)];
          if (c == FLUID || lc == FLUID) {
            float du = d, ld = o->density[cidx(o, x - 1, y, z)];
            if (c == FLUID && lc == FLUID) du = (ld + d) / 2;
            else if (lc == FLUID) du = ld;
            u[ni] = u[ni] - (p - lp) / du;
            hx = 1;
          }
        }
        if (y > 0) {
          int lc = content_cell(o, x, y - 1, z);
          float lp = o->pressure[cidx(o, x, y - 1, z)];
          if (c == FLUID || lc == FLUID) {
            float du = d, ld = o->density[cidx(o, x, y - 1, z)];
            if (c == FLUID && lc == FLUID) du = (ld + d) / 2;
            else if (lc == FLUID) du = ld;
            v[ni] = v[ni] - (p - lp) / du;
            hy = 1;
          }
        }
        if (z > 0) {
          int lc = content_cell(o, x, y, z - 1);
          float lp = o->pressure[cidx(o, x, y, z - 1)];
          if (c == FLUID || lc == FLUID) {
            float du = d, ld = o->density[cidx(o, x, y, z - 1)];
            if (c == FLUID && lc == FLUID) du = (ld + d) / 2;
            else if (lc == FLUID) du = ld;
            w[ni] = w[ni] - (p - lp) / du;
            hz = 1;
          }
        }
        o->has[ci] = hx; o->has[C + ci] = hy; o->has[2 * C + ci] = hz;
      }
}

/* One cell of extrapolateVelocityByOne (Fluid_3D_kernels.cu:210-422) read
 * from nv/hs: the extrapolated components (has_out[c] = 1, nv_out[c]) and
 * the unchanged ones as they are. */
static void extrapolate_cell(const orc_fluid* o, const float* nv, const int* hs, int x, int y, int z, float nv_out[3],
                             int has_out[3]) {
  const int sx = o->sx, sy = o->sy, sz = o->sz, C = o->C, F = o->F;
  const float eps = (float)(-1 + 1e-6);
  const int ci = cidx(o, x, y, z), ni = nidx(o, x, y, z);
  for (int comp = 0; comp < 3; ++comp) {
    has_out[comp] = hs[comp * C + ci];
    nv_out[comp] = nv[comp * F + ni];
    if (has_out[comp]) continue;
    float sum = 0;
    int cnt = 0;
    if (x > 0) {
      int nc = cidx(o, x - 1, y, z), nn = nidx(o, x - 1, y, z);
      if (hs[comp * C + nc] && nv[nn] > eps) { sum += nv[comp * F + nn]; cnt++; }
    }
    if (y > 0) {
      int nc = cidx(o, x, y - 1, z), nn = nidx(o, x, y - 1, z);
      if (hs[comp * C + nc] && nv[F + nn] > eps) { sum += nv[comp * F + nn]; cnt++; }
    }
    if (z > 0) {
      int nc = cidx(o, x, y, z - 1), nn = nidx(o, x, y, z - 1);
      if (hs[comp * C + nc] && nv[2 * F + nn] > eps) { sum += nv[comp * F + nn]; cnt++; }
    }
    if (x < sx - 1) {
      int nc = cidx(o, x + 1, y, z), nn = nidx(o, x + 1, y, z);
      if (hs[comp * C + nc] && nv[nn] < -eps) { sum += nv[comp * F + nn]; cnt++; }
    }
    if (y < sy - 1) {
      int nc = cidx(o, x, y + 1, z), nn = nidx(o, x, y + 1, z);
      if (hs[comp * C + nc] && nv[F + nn] < -eps) { sum += nv[comp * F + nn]; cnt++; }
    }
    if (z < sz - 1) {
      int nc = cidx(o, x, y, z + 1), nn = nidx(o, x, y, z + 1);
      if (hs[comp * C + nc] && nv[2 * F + nn] < -eps) { sum += nv[comp * F + nn]; cnt++; }
    }
    if (cnt > 0) {
      nv_out[comp] = sum / (float)cnt;
      has_out[comp] = 1;
    }
  }
}

typedef struct { float nv[32][3]; int has[32][3]; } extrap_scratch;
static void extrap_serial_read(orc_fluid* o, int x, int y, int z, int k, void* scratch) {
  extrap_scratch* s = (extrap_scratch*)scratch;
  extrapolate_cell(o, o->new_velocity, o->has, x, y, z, s->nv[k], s->has[k]);
}
static void extrap_serial_write(orc_fluid* o, int x, int y, int z, int k, void* scratch) {
  extrap_scratch* s = (extrap_scratch*)scratch;
  const int ci = cidx(o, x, y, z), ni = nidx(o, x, y, z);
  for (int comp = 0; comp < 3; ++comp) {
    o->new_velocity[comp * o->F + ni] = s->nv[k][comp];
    o->has[comp * o->C + ci] = s->has[k][comp];
  }
}

/* extrapolateVelocityByOne (Fluid_3D_kernels.cu:210-422), 3 passes
 * (Fluid_3D_common.cu:65-82); each pass reads the previous pass's values. */
static void stage_extrapolate(orc_fluid* o) {
  const int sx = o->sx, sy = o->sy, sz = o->sz, C = o->C, F = o->F;
  const float eps = (float)(-1 + 1e-6);
  if (o->schedule == 1) {
    extrap_scratch s;
    for (int pass = 0; pass < 3; ++pass) serial_launch(o, extrap_serial_read, extrap_serial_write, &s);
    return;
  }
  for (int pass = 0; pass < 3; ++pass) {
    const float* nv = o->new_velocity;
    const int* hs = o->has;
    memcpy(o->nv_tmp, o->new_velocity, sizeof(float) * 3 * (size_t)F);
#pragma omp parallel for schedule(static)
    for (int x = 0; x < sx; ++x)
      for (int y = 0; y < sy; ++y)
        for (int z = 0; z < sz; ++z) {
          int ci = cidx(o, x, y, z), ni = nidx(o, x, y, z);
          for (int comp = 0; comp < 3; ++comp) {
            int hv = hs[comp * C + ci];
            o->has_tmp[comp * C + ci] = hv;
            if (hv) continue;
            float sum = 0;
            int cnt = 0;
            /* neighbour order: left, down, back, right, up, front; the test
             * uses the neighbour's velocity component along the direction */
            if (x > 0) {
              int nc = cidx(o, x - 1, y, z), nn = nidx(o, x - 1, y, z);
              if (hs[comp * C + nc] && nv[nn] > eps) { sum += nv[comp * F + nn]; cnt++; }
            }
            if (y > 0) {
              int nc = cidx(o, x, y - 1, z), nn = nidx(o, x, y - 1, z);
              if (hs[comp * C + nc] && nv[F + nn] > eps) { sum += nv[comp * F + nn]; cnt++; }
            }
            if (z > 0) {
              int nc = cidx(o, x, y, z - 1), nn = nidx(o, x, y, z - 1);
              if (hs[comp * C + nc] && nv[2 * F + nn] > eps) { sum += nv[comp * F + nn]; cnt++; }
            }
            if (x < sx - 1) {
              int nc = cidx(o, x + 1, y, z), nn = nidx(o, x + 1, y, z);
              if (hs[comp * C + nc] && nv[nn] < -eps) { sum += nv[comp * F + nn]; cnt++; }
            }
            if (y < sy - 1) {
              int nc = cidx(o, x, y + 1, z), nn = nidx(o, x, y + 1, z);
              if (hs[comp * C + nc] && nv[F + nn] < -eps) { sum += nv[comp * F + nn]; cnt++; }
            }
            if (z < sz - 1) {
              int nc = cidx(o, x, y, z + 1), nn = nidx(o, x, y, z + 1);
              if (hs[comp * C + nc] && nv[2 * F + nn] < -eps) { sum += nv[comp * F + nn]; cnt++; }
            }
            if (cnt > 0) {
              o->nv_tmp[comp * F + ni] = sum / (float)cnt;
              o->has_tmp[comp * C + ci] = 1;
            }
          }
        }
    float* t = o->new_velocity; o->new_velocity = o->nv_tmp; o->nv_tmp = t;
    int* th = o->has; o->has = o->has_tmp; o->has_tmp = th;
  }
}

/* solveDiffusionJacobi / diffusionJacobiImpl (Fluid_3D_common.cu:85-91,
 * Fluid_3D_kernels.cu:520-556), ping-pong.  Air cells keep their fractions
 * and get pressure = 0, as the reference writes. */
static void stage_diffuse(orc_fluid* o) {
  const int sx = o->sx, sy = o->sy, sz = o->sz, C = o->C;
  const float h = o->h;
  const float lambda = o->cfg.diffusion_coeff * o->cfg.timestep / (h * h);
  const float center = 1.f + 2 * lambda;
  for (int it = 0; it < o->cfg.diffusion_iterations; ++it) {
    const float* f = o->nvf;
#pragma omp parallel for schedule(static)
    for (int x = 0; x < sx; ++x)
      for (int y = 0; y < sy; ++y)
        for (int z = 0; z < sz; ++z) {
          int ci = cidx(o, x, y, z);
          if (content_cell(o, x, y, z) == AIR) {
            o->pressure[ci] = 0.f;
            for (int k = 0; k < 4; ++k) o->nvf_tmp[k * C + ci] = f[k * C + ci];
            continue;
          }
          int nb[6];
          nb[0] = x + 1 < sx ? cidx(o, x + 1, y, z) : ci;
          nb[1] = x - 1 >= 0 ? cidx(o, x - 1, y, z) : ci;
          nb[2] = y + 1 < sy ? cidx(o, x, y + 1, z) : ci;
          nb[3] = y - 1 >= 0 ? cidx(o, x, y - 1, z) : ci;
          nb[4] = z + 1 < sz ? cidx(o, x, y, z + 1) : ci;
          nb[5] = z - 1 >= 0 ? cidx(o, x, y, z - 1) : ci;
          float r[4];
          for (int k = 0; k < 4; ++k) {
            float acc = 0;
            for (int q = 0; q < 6; ++q) acc += f[k * C + nb[q]] * lambda;
            acc += f[k * C + ci];
            r[k] = acc / center;
          }
          float s = r[0] + r[1] + r[2] + r[3];
          for (int k = 0; k < 4; ++k) o->nvf_tmp[k * C + ci] = r[k] / s;
        }
    float* t = o->nvf; o->nvf = o->nvf_tmp; o->nvf_tmp = t;
  }
}

/* ---------------------------------------------------------- lifecycle */

static void alloc_particles(orc_fluid* o, int n) {
  o->n = n;
  o->pos = (float*)xcalloc((size_t)3 * n, sizeof(float));
  o->vel = (float*)xcalloc((size_t)3 * n, sizeof(float));
  o->frac = (float*)xcalloc((size_t)4 * n, sizeof(float));
  o->pos2 = (float*)xcalloc((size_t)3 * n, sizeof(float));
  o->vel2 = (float*)xcalloc((size_t)3 * n, sizeof(float));
  o->frac2 = (float*)xcalloc((size_t)4 * n, sizeof(float));
  o->hash = (int*)xcalloc((size_t)n, sizeof(int));
  o->sort_index = (int*)xcalloc((size_t)n, sizeof(int));
}

orc_fluid* orc_create(const aq_config* cfg) {
  if (cfg->size_x < 4 || cfg->size_y < 4 || cfg->size_z < 4) return NULL;
  if (cfg->phase_count > AQ_MAX_PHASES) return NULL; /* Fluid_3D_FLIP.cu:449-451 */
  if (cfg->volume_count < 0 || cfg->volume_count > AQ_MAX_VOLUMES) return NULL;
  orc_fluid* o = (orc_fluid*)calloc(1, sizeof(orc_fluid));
  o->cfg = *cfg;
  o->sx = cfg->size_x; o->sy = cfg->size_y; o->sz = cfg->size_z;
  o->C = o->sx * o->sy * o->sz;
  o->F = (o->sx + 1) * (o->sy + 1) * (o->sz + 1);
  o->h = cfg->domain_size / (float)o->sy;
  const size_t C = (size_t)o->C, F = (size_t)o->F;
  o->content = (int*)xcalloc(F, sizeof(int));
  o->velocity = (float*)xcalloc(3 * F, sizeof(float));
  o->new_velocity = (float*)xcalloc(3 * F, sizeof(float));
  o->nv_tmp = (float*)xcalloc(3 * F, sizeof(float));
  o->pressure = (float*)xcalloc(C, sizeof(float));
  o->p_tmp = (float*)xcalloc(C, sizeof(float));
  o->divergence = (float*)xcalloc(C, sizeof(float));
  o->density = (float*)xcalloc(C, sizeof(float));
  o->pcount = (int*)xcalloc(C, sizeof(int));
  o->has = (int*)xcalloc(3 * C, sizeof(int));
  o->has_tmp = (int*)xcalloc(3 * C, sizeof(int));
  o->vf = (float*)xcalloc(4 * C, sizeof(float));
  o->nvf = (float*)xcalloc(4 * C, sizeof(float));
  o->nvf_tmp = (float*)xcalloc(4 * C, sizeof(float));
  o->cstart = (int*)xcalloc(C, sizeof(int));
  o->cend = (int*)xcalloc(C, sizeof(int));
  o->counts = (int*)xcalloc(C, sizeof(int));
  for (size_t c = 0; c < C; ++c) o->cstart[c] = o->cend[c] = -1;

  /* Fluid::init: the grid starts all AIR/zero (createField3D + clearField3D,
   * MAC_Grid_3D.cu:43-75), then fixBoundary, seeding and transferToGrid. */
  fix_boundary(o);
  memset(&o->rng, 0, sizeof(o->rng));
  initstate_r(cfg->seed, o->rng.state, sizeof(o->rng.state), &o->rng.rd);
  plist pl = {NULL, 0, 0};
  for (int i = 0; i < cfg->volume_count; ++i) {
    const aq_volume* v = &cfg->volumes[i];
    if (v->shape == AQ_SHAPE_SQUARE) create_square(o, &o->rng, &pl, v);
    else if (v->shape == AQ_SHAPE_SPHERE) create_sphere(o, &o->rng, &pl, v);
  }
  alloc_particles(o, pl.n);
  const int n = pl.n;
  for (int i = 0; i < n; ++i) {
    for (int d = 0; d < 3; ++d) o->pos[d * n + i] = pl.data[7 * (size_t)i + d];
    for (int d = 0; d < 4; ++d) o->frac[d * n + i] = pl.data[7 * (size_t)i + 3 + d];
  }
  free(pl.data);
  stage_sort(o);
  stage_p2g(o, 0);
  return o;
}

void orc_destroy(orc_fluid* o) {
  if (!o) return;
  void* ptrs[] = {o->pos, o->vel, o->frac, o->pos2, o->vel2, o->frac2, o->hash, o->sort_index,
                  o->counts, o->content, o->velocity, o->new_velocity, o->nv_tmp, o->pressure,
                  o->p_tmp, o->divergence, o->density, o->pcount, o->has, o->has_tmp, o->vf,
                  o->nvf, o->nvf_tmp, o->cstart, o->cend, o->ink_pos, o->ink_vel};
  for (size_t i = 0; i < sizeof(ptrs) / sizeof(ptrs[0]); ++i) free(ptrs[i]);
  free(o);
}

int orc_particle_count(const orc_fluid* o) { return o->n; }

int orc_run_stage(orc_fluid* o, int stage) {
  switch (stage) {
    case AQ_STAGE_G2P_ADVECT: stage_g2p_advect(o); return 0;
    case AQ_STAGE_SORT: stage_sort(o); return 0;
    case AQ_STAGE_P2G: stage_p2g(o, 1); return 0;
    case AQ_STAGE_DIVERGENCE: stage_divergence(o); return 0;
    case AQ_STAGE_PRESSURE: stage_pressure(o); return 0;
    case AQ_STAGE_PROJECT: stage_project(o); return 0;
    case AQ_STAGE_EXTRAPOLATE: stage_extrapolate(o); return 0;
    case AQ_STAGE_DIFFUSE:
      stage_diffuse(o);
      /* transferToInkParticles + moveInkParticles (Fluid_3D_FLIP.cu:349-350,
       * commented out in the reference), once the ink exists */
      if (o->ink_pos) orc_ink_advance(o);
      o->time += o->cfg.timestep; /* physicalTime += timestep (Fluid_3D_FLIP.cu:351) */
      return 0;
    default: return 1;
  }
}

int orc_step(orc_fluid* o, int nsteps) {
  for (int s = 0; s < nsteps; ++s)
    for (int k = AQ_STAGE_G2P_ADVECT; k <= AQ_STAGE_DIFFUSE; ++k)
      if (orc_run_stage(o, k)) return 1;
  return 0;
}

void orc_solve_stats(const orc_fluid* o, int* iters, double* rel_res, double* b_norm, int* fluid_cells) {
  if (iters) *iters = o->iters;
  if (rel_res) *rel_res = o->rel_res;
  if (b_norm) *b_norm = o->b_norm;
  if (fluid_cells) *fluid_cells = o->fluid_cells;
}

#define CPY(dst, src, cnt) \
  do { if (dst) memcpy((dst), (src), sizeof(*(src)) * (size_t)(cnt)); } while (0)

int orc_get_state(const orc_fluid* o, aq_host_state* s) {
  if (s->size_x != o->sx || s->size_y != o->sy || s->size_z != o->sz || s->particle_count != o->n) return 1;
  const int n = o->n, C = o->C, F = o->F;
  s->physical_time = o->time;
  CPY(s->position, o->pos, 3 * n);
  CPY(s->velocity_p, o->vel, 3 * n);
  CPY(s->fractions, o->frac, 4 * n);
  CPY(s->content, o->content, F);
  CPY(s->velocity, o->velocity, 3 * F);
  CPY(s->new_velocity, o->new_velocity, 3 * F);
  CPY(s->pressure, o->pressure, C);
  CPY(s->divergence, o->divergence, C);
  CPY(s->particle_count_cell, o->pcount, C);
  CPY(s->has_velocity, o->has, 3 * C);
  CPY(s->volume_fractions, o->vf, 4 * C);
  CPY(s->new_volume_fractions, o->nvf, 4 * C);
  CPY(s->density, o->density, C);
  CPY(s->cell_start, o->cstart, C);
  CPY(s->cell_end, o->cend, C);
  CPY(s->particle_hash, o->hash, n);
  CPY(s->sort_index, o->sort_index, n);
  return 0;
}

#define CPYIN(dst, src, cnt) \
  do { if (src) memcpy((dst), (src), sizeof(*(dst)) * (size_t)(cnt)); } while (0)

int orc_set_state(orc_fluid* o, const aq_host_state* s) {
  if (s->size_x != o->sx || s->size_y != o->sy || s->size_z != o->sz || s->particle_count != o->n) return 1;
  const int n = o->n, C = o->C, F = o->F;
  o->time = s->physical_time;
  CPYIN(o->pos, s->position, 3 * n);
  CPYIN(o->vel, s->velocity_p, 3 * n);
  CPYIN(o->frac, s->fractions, 4 * n);
  CPYIN(o->content, s->content, F);
  CPYIN(o->velocity, s->velocity, 3 * F);
  CPYIN(o->new_velocity, s->new_velocity, 3 * F);
  CPYIN(o->pressure, s->pressure, C);
  CPYIN(o->divergence, s->divergence, C);
  CPYIN(o->pcount, s->particle_count_cell, C);
  CPYIN(o->has, s->has_velocity, 3 * C);
  CPYIN(o->vf, s->volume_fractions, 4 * C);
  CPYIN(o->nvf, s->new_volume_fractions, 4 * C);
  CPYIN(o->density, s->density, C);
  CPYIN(o->cstart, s->cell_start, C);
  CPYIN(o->cend, s->cell_end, C);
  CPYIN(o->hash, s->particle_hash, n);
  CPYIN(o->sort_index, s->sort_index, n);
  return 0;
}
