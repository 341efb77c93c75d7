/*
 * CPU oracle of the headless frame — TEST INFRASTRUCTURE ONLY (see
 * render_oracle.h).
 *
 * Fixed-function rules (the same in the CUDA frame, aquarius_b200/csrc/
 * k_render.cu; all float arithmetic single precision, rounded as written, no
 * fused multiply-add):
 *
 *  clear     colour (0,0,0,1), depth 1.0 (main.cu:111-117).
 *  vertices  clip = M * (p, 1) with M the host's float product
 *            (projection * view) * model (projection * view for the mesh and
 *            the points, whose model is the identity), each row summed (a0+a1)+(a2+a3) as
 *            glm's mat4 * vec4 does; ndc = clip.xyz / clip.w; window
 *            x = (W/2) ndc.x + W/2, y = (H/2) ndc.y + H/2, z = ndc.z/2 + 1/2.
 *  triangles dropped whole when a vertex has w <= 0, z < -w (in front of the
 *            near plane) or |ndc.x| or |ndc.y| > 16 (no clipping); window x, y
 *            snapped to 1/256 pixel (round to nearest even); integer edge
 *            functions; zero area dropped, both windings drawn (no culling);
 *            a pixel centre on an edge belongs to the triangle when that edge
 *            is a top or left edge; depth interpolated linearly in window
 *            space, fragments outside [0,1] dropped; varyings interpolated
 *            perspective-correctly, ((q0 a0 + q1 a1) + q2 a2) / ((q0 + q1) + q2)
 *            with q_k = lambda_k / w_k.
 *  points    dropped when the vertex lies outside the clip volume; size
 *            clamped to [1, 2048]; pixel (i, j) is covered when its centre
 *            (i + 1/2, j + 1/2) lies in [x - s/2, x + s/2) x [y - s/2, y + s/2);
 *            gl_PointCoord = ((c - x)/s + 1/2), origin lower left.
 *  depth     24-bit: round((double)z * (2^24 - 1)); test GL_LESS; written by
 *            opaque passes that pass it.
 *  blending  RGBA8 framebuffer; the source is clamped to [0,1] (NaN to 0),
 *            blended SRC_ALPHA, ONE_MINUS_SRC_ALPHA on all four channels
 *            (the state Fluid::draw leaves behind, PointSprites.cu:253) and
 *            rounded to the nearest 1/255 (even on ties).
 *  textures  cube map: the major axis picks the face (x over y over z on
 *            ties), the face coordinates follow the GL cube-map table; 2D and
 *            cube faces are filtered bilinearly, clamped to the edge, texels
 *            at byte/255.  The phase-thickness texture is sampled nearest with
 *            repeat wrapping.
 *
 * Frame order (main.cu:136-143): skybox background (AQ_ENV_SKYBOX only,
 * depth not written), container faces (Container.cu:71-120), then the fluid
 * (Fluid/Fluid_3D_FLIP.cu:396-430): mesh modes draw the phase-thickness
 * sprites additively into their own float texture first (multiphase modes,
 * PointSprites.cu:217-256), then the mesh triangles in VBO order;
 * AQ_RENDER_PARTICLES draws shaded sprites with depth (PointSprites.cu:196-215).
 * AQ_RENDER_NONE leaves the cleared frame.
 */
#include "render_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef struct { float x, y, z; } v3;
typedef struct { float x, y, z, w; } v4;

static v3 V3(float x, float y, float z) { v3 r = {x, y, z}; return r; }
static v4 V4(float x, float y, float z, float w) { v4 r = {x, y, z, w}; return r; }
static v3 add3(v3 a, v3 b) { return V3(a.x + b.x, a.y + b.y, a.z + b.z); }
static v3 sub3(v3 a, v3 b) { return V3(a.x - b.x, a.y - b.y, a.z - b.z); }
static v3 mul3s(v3 a, float s) { return V3(a.x * s, a.y * s, a.z * s); }
static v3 mul3(v3 a, v3 b) { return V3(a.x * b.x, a.y * b.y, a.z * b.z); }
static float dot3(v3 a, v3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
/* glm: v * inversesqrt(dot(v, v)), inversesqrt(x) = 1 / sqrt(x) */
static v3 normalize3(v3 v) { return mul3s(v, 1.0f / sqrtf(dot3(v, v))); }
static v3 reflect3(v3 i, v3 n) { return sub3(i, mul3s(mul3s(n, dot3(n, i)), 2.0f)); }
static float gmin(float x, float y) { return y < x ? y : x; }  /* glm min */
static float gmax(float x, float y) { return x < y ? y : x; }  /* glm max */
static v4 mul4s(v4 a, float s) { return V4(a.x * s, a.y * s, a.z * s, a.w * s); }
static v4 add4(v4 a, v4 b) { return V4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w); }
static v4 mix4(v4 x, v4 y, float a) { return add4(mul4s(x, 1.0f - a), mul4s(y, a)); }

/* GLSL int(float): truncation; out-of-range values saturate, NaN gives 0. */
static int f2i_trunc(float v) {
  if (v != v) return 0;
  if (v >= 2147483647.0f) return 2147483647;
  if (v <= -2147483648.0f) return (int)0x80000000u;
  return (int)v;
}

typedef struct {
  const aq_draw_command* dc;
  const uint8_t* sky;
  int face;
  const uint8_t* logo;
  int lw, lh;
} env_t;

/* ------------------------------------------------------------ samplers */
static float texel(const uint8_t* img, int w, int h, int x, int y, int c) {
  x = x < 0 ? 0 : (x > w - 1 ? w - 1 : x);
  y = y < 0 ? 0 : (y > h - 1 ? h - 1 : y);
  return (float)img[((size_t)y * w + x) * 3 + c] / 255.0f;
}

void orc_sample_2d(const uint8_t* img, int32_t w, int32_t h, float s, float t, float out[4]) {
  out[3] = 1.0f;
  if (!img || w <= 0 || h <= 0 || !(s == s) || !(t == t)) { out[0] = out[1] = out[2] = 0.0f; return; }
  const float u = s * (float)w - 0.5f, v = t * (float)h - 0.5f;
  const float fu = floorf(u), fv = floorf(v);
  const float a = u - fu, b = v - fv;
  const int x0 = f2i_trunc(fu), y0 = f2i_trunc(fv);
  const int x1 = x0 == 2147483647 ? x0 : x0 + 1, y1 = y0 == 2147483647 ? y0 : y0 + 1;
  for (int c = 0; c < 3; ++c) {
    const float c00 = texel(img, w, h, x0, y0, c), c10 = texel(img, w, h, x1, y0, c);
    const float c01 = texel(img, w, h, x0, y1, c), c11 = texel(img, w, h, x1, y1, c);
    out[c] = (c00 * (1.0f - a) + c10 * a) * (1.0f - b) + (c01 * (1.0f - a) + c11 * a) * b;
  }
}

void orc_sample_cube(const uint8_t* sky, int32_t face, const float dir[3], float out[4]) {
  const float rx = dir[0], ry = dir[1], rz = dir[2];
  const float ax = fabsf(rx), ay = fabsf(ry), az = fabsf(rz);
  int f;
  float sc, tc, ma;
  if (ax >= ay && ax >= az) {
    ma = ax;
    if (rx >= 0.0f) { f = 0; sc = -rz; tc = -ry; } else { f = 1; sc = rz; tc = -ry; }
  } else if (ay >= az) {
    ma = ay;
    if (ry >= 0.0f) { f = 2; sc = rx; tc = rz; } else { f = 3; sc = rx; tc = -rz; }
  } else {
    ma = az;
    if (rz >= 0.0f) { f = 4; sc = rx; tc = -ry; } else { f = 5; sc = -rx; tc = -ry; }
  }
  const float s = (sc / ma + 1.0f) * 0.5f, t = (tc / ma + 1.0f) * 0.5f;
  orc_sample_2d(sky ? sky + (size_t)f * face * face * 3 : NULL, face, face, s, t, out);
}

/* ------------------------------------------------- RayTraceEnvironment.glsl */
static v3 chess_board(float x, float z) {  /* :6-13 */
  const int xi = f2i_trunc(x + 100.0f), zi = f2i_trunc(z + 100.0f);
  if ((((unsigned)xi + (unsigned)zi) & 1u) == 0u) return V3(0.5f, 0.5f, 0.5f);
  return V3(0.8f, 0.8f, 0.8f);
}

#define RT_EPS 1e-3f

static v3 cornell_color(const env_t* e, v3 pos, v3 bmin, v3 bmax) {  /* :61-97 */
  if (fabsf(pos.z - bmax.z) < RT_EPS) {
    const float fsx = bmax.x - bmin.x, fsy = bmax.y - bmin.y;
    const float lsx = 0.3f * fsx, lsy = 0.3f * fsy;
    const float lcx = 0.5f * fsx + bmin.x, lcy = 0.3f * fsy + bmin.y;
    const float lminx = lcx - lsx / 2.0f, lminy = lcy - lsy / 2.0f;
    float lx = pos.x - lminx, ly = pos.y - lminy;
    lx = lx / lsx;
    ly = ly / lsy;
    lx = 1.0f - lx;
    ly = 1.0f - ly;
    if (lx >= 0.0f && lx <= 1.0f && ly >= 0.0f && ly <= 1.0f) {
      float c[4];
      orc_sample_2d(e->logo, e->lw, e->lh, lx, ly, c);
      return V3(c[0], c[1], c[2]);
    }
  }
  if (fabsf(pos.y - bmin.y) < RT_EPS) return chess_board(pos.x, pos.z);
  return V3(0.8f, 0.8f, 0.8f);
}

static v3 cornell_normal(v3 pos, v3 bmin, v3 bmax) {  /* :100-119; no match: 0 */
  if (fabsf(pos.x - bmin.x) < 1e-3f) return V3(1, 0, 0);
  if (fabsf(pos.x - bmax.x) < 1e-3f) return V3(-1, 0, 0);
  if (fabsf(pos.y - bmin.y) < 1e-3f) return V3(0, 1, 0);
  if (fabsf(pos.y - bmax.y) < 1e-3f) return V3(0, -1, 0);
  if (fabsf(pos.z - bmin.z) < 1e-3f) return V3(0, 0, 1);
  if (fabsf(pos.z - bmax.z) < 1e-3f) return V3(0, 0, -1);
  return V3(0, 0, 0);
}

static v4 trace_env(const env_t* e, v3 o, v3 d) {  /* :122-178 */
  const aq_draw_command* dc = e->dc;
  const v3 light = V3(dc->light_position[0], dc->light_position[1], dc->light_position[2]);
  if (dc->environment_mode == AQ_ENV_CORNELL_BOX) {
    const float pad = (dc->cornell_box_size - dc->container_size) / 2.0f;
    const v3 bmin = mul3s(V3(-1.0f, 0.0f, -1.0f), pad);
    const v3 bmax = add3(bmin, V3(dc->cornell_box_size, dc->cornell_box_size, dc->cornell_box_size));
    const v3 inv = V3(1.0f / d.x, 1.0f / d.y, 1.0f / d.z);
    const v3 tbot = mul3(inv, sub3(bmin, o)), ttop = mul3(inv, sub3(bmax, o));
    const v3 tmin = V3(gmin(ttop.x, tbot.x), gmin(ttop.y, tbot.y), gmin(ttop.z, tbot.z));
    const v3 tmax = V3(gmax(ttop.x, tbot.x), gmax(ttop.y, tbot.y), gmax(ttop.z, tbot.z));
    const float t0 = gmax(tmin.x, gmax(tmin.y, tmin.z));
    const float t1 = gmin(tmax.x, gmin(tmax.y, tmax.z));
    if (t0 >= t1) return V4(0, 0, 0, 0);
    if (t1 < 0.0f) return V4(0, 0, 0, 0);
    const float t = t0 < 0.0f ? t1 : t0;
    const v3 hit = add3(o, mul3s(d, t));
    const v3 base = cornell_color(e, hit, bmin, bmax);
    const v3 n = cornell_normal(hit, bmin, bmax);
    const v3 tl = normalize3(sub3(light, hit));
    const v3 r = mul3s(base, 0.1f + 0.5f * gmax(0.0f, dot3(n, tl)));
    return V4(r.x, r.y, r.z, 1.0f);
  }
  const float tg = o.y / -d.y;
  const v3 hit = add3(o, mul3s(d, tg));
  if (dc->environment_mode == AQ_ENV_SKYBOX) {
    if (tg > 0.0f && hit.x >= 0.0f && hit.x <= dc->container_size && hit.z >= 0.0f &&
        hit.z <= dc->container_size) {
      const v3 c = chess_board(hit.x, hit.z);
      return V4(c.x, c.y, c.z, 1.0f);
    }
    float c[4];
    const float dd[3] = {d.x, d.y, d.z};
    orc_sample_cube(e->sky, e->face, dd, c);
    return V4(c[0], c[1], c[2], 1.0f);
  }
  if (tg > 0.0f) {
    const v3 tl = normalize3(sub3(light, hit));
    const v3 c = chess_board(hit.x, hit.z);
    return mul4s(V4(c.x, c.y, c.z, 1.0f), 0.1f + 0.5f * dot3(V3(0.0f, 1.0f, 0.0f), tl));
  }
  return V4(0, 0, 0, 1);
}

void orc_trace_environment(const aq_draw_command* dc, const uint8_t* sky, int32_t face, const uint8_t* logo,
                           int32_t lw, int32_t lh, const float origin[3], const float dir[3], float out[4]) {
  const env_t e = {dc, sky, face, logo, lw, lh};
  const v4 r = trace_env(&e, V3(origin[0], origin[1], origin[2]), V3(dir[0], dir[1], dir[2]));
  out[0] = r.x; out[1] = r.y; out[2] = r.z; out[3] = r.w;
}

/* -------------------------------------------- FluidMeshRenderer_fs.glsl */
static v4 shade_mesh(const env_t* e, v3 fpos, v3 fnormal, v4 texel) {
  const aq_draw_command* dc = e->dc;
  const int mode = dc->render_mode;
  const v3 light = V3(dc->light_position[0], dc->light_position[1], dc->light_position[2]);
  const v3 cam = V3(dc->camera_position[0], dc->camera_position[1], dc->camera_position[2]);
  const v3 normal = normalize3(fnormal);
  if (mode == AQ_RENDER_FLAT_MESH) {  /* lambertian, :96-99 */
    const v3 tl = normalize3(sub3(light, fpos));
    const float l = 0.3f + 0.5f * dot3(normal, tl);
    return V4(l, l, l, 1.0f);
  }
  if (mode == AQ_RENDER_NORMAL_MESH) return V4(normal.x, normal.y, normal.z, 1.0f);
  const v3 incident = normalize3(sub3(fpos, cam));
  const v3 refl = reflect3(incident, normal);
  v4 rc = trace_env(e, fpos, refl);  /* getReflectedColor, :84-94 */
  {
    const v3 tl = normalize3(sub3(light, fpos));
    if (dc->environment_mode == AQ_ENV_CHESS_BOARD || dc->environment_mode == AQ_ENV_CORNELL_BOX) {
      const float r = 0.3f;
      rc = mul4s(rc, (1.0f - r) + r * dot3(normal, tl));
    }
  }
  if (mode == AQ_RENDER_MIRROR_MESH) return rc;
  /* getRefractedRay, :63-70 */
  const float n = 1.0f / 1.333f;
  const float w = n * dot3(normal, mul3s(incident, -1.0f));
  const float k = sqrtf(1.0f + (w - n) * (w + n));
  const v3 refr = normalize3(add3(mul3s(normal, w - k), mul3s(incident, n)));
  v4 fc;
  const int multiphase = mode == AQ_RENDER_MULTIPHASE_MESH || (mode >= AQ_RENDER_REFRACT_MESH && mode <= AQ_RENDER_PHASE1_MESH);
  if (multiphase) {  /* :136-183 */
    const v4 pt = mul4s(texel, 0.1f);
    const float thickness = ((pt.x + pt.y) + pt.z) + pt.w;
    const float fr[4] = {pt.x / thickness, pt.y / thickness, pt.z / thickness, pt.w / thickness};
    const float ptv[4] = {pt.x, pt.y, pt.z, pt.w};
    v4 tint = V4(0, 0, 0, 0);
    const float ct = ((pt.x * dc->phase_colors[0][3] + pt.y * dc->phase_colors[1][3]) + pt.z * dc->phase_colors[2][3]) +
                     pt.w * dc->phase_colors[3][3];
    if (ct > 0.0f) {
      float cf[4];
      for (int i = 0; i < 4; ++i) cf[i] = ptv[i] * dc->phase_colors[i][3] / ct;
      const int pc = dc->phase_count < 4 ? dc->phase_count : 4;
      for (int i = 0; i < pc; ++i) {
        tint.x = tint.x + cf[i] * dc->phase_colors[i][0];
        tint.y = tint.y + cf[i] * dc->phase_colors[i][1];
        tint.z = tint.z + cf[i] * dc->phase_colors[i][2];
        tint.w = tint.w + fr[i] * dc->phase_colors[i][3];
      }
    }
    const float att = gmax(expf(0.2f * -ct), 0.2f);
    fc = mix4(tint, trace_env(e, fpos, refr), att);
    if (mode == AQ_RENDER_REFRACT_MESH) return fc;
    if (mode == AQ_RENDER_PHASE0_MESH) { const float v = pt.x / 50.0f; return V4(v, v, v, 1.0f); }
    if (mode == AQ_RENDER_PHASE1_MESH) { const float v = pt.y / 50.0f; return V4(v, v, v, 1.0f); }
  } else {
    const v4 tint = V4(6.0f / 256.0f, 105.0f / 256.0f, 217.0f / 256.0f, 256.0f / 256.0f);
    fc = mix4(tint, trace_env(e, fpos, refr), 0.5f);
  }
  /* schlick, :53-60 (pow(x, 1) = x) */
  const float f0a = (1.333f - 1.0f) / (1.333f + 1.0f);
  const float f0 = f0a * f0a;
  const float F = f0 + (1.0f - f0) * (1.0f - dot3(normal, mul3s(incident, -1.0f)));
  v4 c = mix4(fc, rc, F);
  c.w = 1.0f;
  return c;
}

void orc_shade_mesh(const aq_draw_command* dc, const uint8_t* sky, int32_t face, const uint8_t* logo,
                    int32_t lw, int32_t lh, const float frag_pos[3], const float frag_normal[3],
                    const float tex[4], float out[4]) {
  const env_t e = {dc, sky, face, logo, lw, lh};
  const v4 r = shade_mesh(&e, V3(frag_pos[0], frag_pos[1], frag_pos[2]),
                          V3(frag_normal[0], frag_normal[1], frag_normal[2]), V4(tex[0], tex[1], tex[2], tex[3]));
  out[0] = r.x; out[1] = r.y; out[2] = r.z; out[3] = r.w;
}

/* ------------------------------------------------------------- matrices */
typedef struct { float m[16]; } mat4;  /* column-major: m[c*4 + r] */

static mat4 mat_mul(const float* a, const float* b) {  /* glm mat4 * mat4 */
  mat4 r;
  for (int c = 0; c < 4; ++c)
    for (int k = 0; k < 4; ++k)
      r.m[c * 4 + k] = ((a[0 * 4 + k] * b[c * 4 + 0] + a[1 * 4 + k] * b[c * 4 + 1]) + a[2 * 4 + k] * b[c * 4 + 2]) +
                       a[3 * 4 + k] * b[c * 4 + 3];
  return r;
}

static v4 mat_vec(const float* m, float x, float y, float z) {  /* glm mat4 * vec4(x, y, z, 1) */
  float o[4];
  for (int k = 0; k < 4; ++k) o[k] = (m[0 * 4 + k] * x + m[1 * 4 + k] * y) + (m[2 * 4 + k] * z + m[3 * 4 + k] * 1.0f);
  return V4(o[0], o[1], o[2], o[3]);
}

static mat4 diag_model(float s, float tx, float tz) {
  mat4 r;
  memset(&r, 0, sizeof(r));
  r.m[0] = s; r.m[5] = s; r.m[10] = s; r.m[15] = 1.0f;
  r.m[12] = tx; r.m[14] = tz;
  return r;
}

/* Container::bottomData (Rendering/Renderer3D/Container.h:41-90): the unit
 * cube's faces as 12 triangles; the first two are the floor. */
static const float kCubeTris[36][3] = {
    {0, 0, 0}, {0, 0, 1}, {1, 0, 0}, {1, 0, 0}, {0, 0, 1}, {1, 0, 1},
    {0, 1, 0}, {0, 0, 0}, {1, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0},
    {0, 0, 1}, {0, 0, 0}, {0, 1, 0}, {0, 1, 0}, {0, 1, 1}, {0, 0, 1},
    {1, 0, 0}, {1, 0, 1}, {1, 1, 1}, {1, 1, 1}, {1, 1, 0}, {1, 0, 0},
    {0, 0, 1}, {0, 1, 1}, {1, 1, 1}, {1, 1, 1}, {1, 0, 1}, {0, 0, 1},
    {0, 1, 0}, {1, 1, 0}, {1, 1, 1}, {1, 1, 1}, {0, 1, 1}, {0, 1, 0},
};

/* ---------------------------------------------------------- framebuffer */
typedef struct {
  int W, H;
  uint8_t* rgba;
  uint32_t* depth;
} fb_t;

static uint8_t to_byte(float v) { return (uint8_t)rintf(v * 255.0f); }

static float clamp01(float v) { return fminf(fmaxf(v, 0.0f), 1.0f); }

static void blend(fb_t* fb, size_t px, v4 c) {
  const float src[4] = {clamp01(c.x), clamp01(c.y), clamp01(c.z), clamp01(c.w)};
  const float sa = src[3];
  uint8_t* d = fb->rgba + px * 4;
  for (int k = 0; k < 4; ++k) {
    const float dst = (float)d[k] / 255.0f;
    d[k] = to_byte(src[k] * sa + dst * (1.0f - sa));
  }
}

static uint32_t depth24(float z) { return (uint32_t)rint((double)z * 16777215.0); }

/* Window-space vertex of a triangle. */
typedef struct {
  int32_t X, Y;   /* 1/256 pixel */
  float z, iw;    /* window depth, 1 / clip w */
  float a[8];     /* varyings: world position, ndc xy, normal */
} tv_t;

/* Transforms a vertex; returns 0 when the triangle must be dropped. */
static int tri_vertex(const float* mvp, const float* model, const float* p, const float* nrm, int W, int H, tv_t* o) {
  const v4 c = mat_vec(mvp, p[0], p[1], p[2]);
  if (!(c.w > 0.0f) || c.z < -c.w) return 0;
  const float nx = c.x / c.w, ny = c.y / c.w, nz = c.z / c.w;
  if (!(fabsf(nx) <= 16.0f) || !(fabsf(ny) <= 16.0f)) return 0;
  const float hw = 0.5f * (float)W, hh = 0.5f * (float)H;
  const float xw = hw * nx + hw, yw = hh * ny + hh;
  o->X = (int32_t)rintf(xw * 256.0f);
  o->Y = (int32_t)rintf(yw * 256.0f);
  o->z = nz * 0.5f + 0.5f;
  o->iw = 1.0f / c.w;
  const v4 wp = mat_vec(model, p[0], p[1], p[2]);
  o->a[0] = wp.x / wp.w; o->a[1] = wp.y / wp.w; o->a[2] = wp.z / wp.w;
  o->a[3] = nx; o->a[4] = ny;
  o->a[5] = nrm ? nrm[0] : 0.0f; o->a[6] = nrm ? nrm[1] : 0.0f; o->a[7] = nrm ? nrm[2] : 0.0f;
  return 1;
}

static int64_t edge(int32_t ax, int32_t ay, int32_t bx, int32_t by, int32_t px, int32_t py) {
  return (int64_t)(bx - ax) * (int64_t)(py - ay) - (int64_t)(by - ay) * (int64_t)(px - ax);
}

static int top_left(int32_t ax, int32_t ay, int32_t bx, int32_t by) {
  const int32_t dx = bx - ax, dy = by - ay;
  return dy < 0 || (dy == 0 && dx < 0);
}

typedef void (*frag_fn)(void* ctx, fb_t* fb, size_t px, const float* a);

/* Rasterises one triangle in GL order: every covered pixel in turn. */
static void raster_tri(fb_t* fb, tv_t v0, tv_t v1, tv_t v2, frag_fn fn, void* ctx) {
  int64_t area = edge(v0.X, v0.Y, v1.X, v1.Y, v2.X, v2.Y);
  if (area == 0) return;
  if (area < 0) { const tv_t t = v1; v1 = v2; v2 = t; area = -area; }
  const int32_t xmin = v0.X < v1.X ? (v0.X < v2.X ? v0.X : v2.X) : (v1.X < v2.X ? v1.X : v2.X);
  const int32_t xmax = v0.X > v1.X ? (v0.X > v2.X ? v0.X : v2.X) : (v1.X > v2.X ? v1.X : v2.X);
  const int32_t ymin = v0.Y < v1.Y ? (v0.Y < v2.Y ? v0.Y : v2.Y) : (v1.Y < v2.Y ? v1.Y : v2.Y);
  const int32_t ymax = v0.Y > v1.Y ? (v0.Y > v2.Y ? v0.Y : v2.Y) : (v1.Y > v2.Y ? v1.Y : v2.Y);
  int i0 = (xmin - 128) >> 8, i1 = (xmax - 128 + 255) >> 8;
  int j0 = (ymin - 128) >> 8, j1 = (ymax - 128 + 255) >> 8;
  if (i0 < 0) i0 = 0;
  if (j0 < 0) j0 = 0;
  if (i1 > fb->W - 1) i1 = fb->W - 1;
  if (j1 > fb->H - 1) j1 = fb->H - 1;
  const int tl0 = top_left(v1.X, v1.Y, v2.X, v2.Y), tl1 = top_left(v2.X, v2.Y, v0.X, v0.Y),
            tl2 = top_left(v0.X, v0.Y, v1.X, v1.Y);
  const float fa = (float)area;
  for (int j = j0; j <= j1; ++j)
    for (int i = i0; i <= i1; ++i) {
      const int32_t px = i * 256 + 128, py = j * 256 + 128;
      const int64_t w0 = edge(v1.X, v1.Y, v2.X, v2.Y, px, py);
      const int64_t w1 = edge(v2.X, v2.Y, v0.X, v0.Y, px, py);
      const int64_t w2 = edge(v0.X, v0.Y, v1.X, v1.Y, px, py);
      if (w0 < 0 || w1 < 0 || w2 < 0) continue;
      if ((w0 == 0 && !tl0) || (w1 == 0 && !tl1) || (w2 == 0 && !tl2)) continue;
      const float l0 = (float)w0 / fa, l1 = (float)w1 / fa, l2 = (float)w2 / fa;
      const float z = (l0 * v0.z + l1 * v1.z) + l2 * v2.z;
      if (!(z >= 0.0f && z <= 1.0f)) continue;
      const size_t p = (size_t)j * fb->W + i;
      const uint32_t d = depth24(z);
      if (!(d < fb->depth[p])) continue;
      const float q0 = l0 * v0.iw, q1 = l1 * v1.iw, q2 = l2 * v2.iw;
      const float den = (q0 + q1) + q2;
      float a[8];
      for (int k = 0; k < 8; ++k) a[k] = ((q0 * v0.a[k] + q1 * v1.a[k]) + q2 * v2.a[k]) / den;
      fb->depth[p] = d;
      fn(ctx, fb, p, a);
    }
}

/* Point vertex stage (PointSprites_points_vs.glsl). Returns 0 when clipped. */
typedef struct { float x, y, s, vz; } sprite_t;

static int sprite_setup(const float* pv, const float* view, const aq_draw_command* dc, float tan_half, const float* p,
                        sprite_t* o) {
  const v4 c = mat_vec(pv, p[0], p[1], p[2]);
  if (!(c.w > 0.0f) || !(c.x >= -c.w && c.x <= c.w && c.y >= -c.w && c.y <= c.w && c.z >= -c.w && c.z <= c.w))
    return 0;
  const v3 cam = V3(dc->camera_position[0], dc->camera_position[1], dc->camera_position[2]);
  const v3 d = sub3(V3(p[0], p[1], p[2]), cam);
  const float dist = sqrtf(dot3(d, d));
  const float half = tan_half * dist;
  float s = ((float)dc->window_height / 2.0f) * dc->point_radius / half;
  if (!(s >= 1.0f)) s = 1.0f;
  if (s > 2048.0f) s = 2048.0f;
  const float hw = 0.5f * (float)dc->window_width, hh = 0.5f * (float)dc->window_height;
  o->x = hw * (c.x / c.w) + hw;
  o->y = hh * (c.y / c.w) + hh;
  o->s = s;
  const v4 pc = mat_vec(view, p[0], p[1], p[2]);
  o->vz = pc.z / pc.w;
  return 1;
}

/* --------------------------------------------------------------- frame */
typedef struct {
  env_t e;
  const float* phase;
  v3 cam;
} fctx_t;

static void frag_container(void* ctx, fb_t* fb, size_t px, const float* a) {  /* Container_face_fs.glsl */
  const fctx_t* c = (const fctx_t*)ctx;
  const v3 dir = normalize3(sub3(V3(a[0], a[1], a[2]), c->cam));
  blend(fb, px, trace_env(&c->e, c->cam, dir));
}

static void frag_mesh(void* ctx, fb_t* fb, size_t px, const float* a) {
  const fctx_t* c = (const fctx_t*)ctx;
  v4 tex = V4(0, 0, 0, 0);
  if (c->phase) {
    const float u = (a[3] + 1.0f) / 2.0f, v = (a[4] + 1.0f) / 2.0f;
    const float fu = floorf(u * (float)fb->W), fv = floorf(v * (float)fb->H);
    int ti = 0, tj = 0;
    if (fu == fu && fabsf(fu) < 1e9f) { ti = (int)fu % fb->W; if (ti < 0) ti += fb->W; }
    if (fv == fv && fabsf(fv) < 1e9f) { tj = (int)fv % fb->H; if (tj < 0) tj += fb->H; }
    const float* t = c->phase + ((size_t)tj * fb->W + ti) * 4;
    tex = V4(t[0], t[1], t[2], t[3]);
  }
  blend(fb, px, shade_mesh(&c->e, V3(a[0], a[1], a[2]), V3(a[5], a[6], a[7]), tex));
}

static void sprite_range(const sprite_t* s, int W, int H, int* i0, int* i1, int* j0, int* j1) {
  const float lx = s->x - s->s * 0.5f, hx = s->x + s->s * 0.5f;
  const float ly = s->y - s->s * 0.5f, hy = s->y + s->s * 0.5f;
  float a = floorf(lx - 0.5f), b = ceilf(hx - 0.5f), c = floorf(ly - 0.5f), d = ceilf(hy - 0.5f);
  a = fmaxf(a, 0.0f); c = fmaxf(c, 0.0f);
  b = fminf(b, (float)(W - 1)); d = fminf(d, (float)(H - 1));
  *i0 = (int)a; *i1 = (int)b; *j0 = (int)c; *j1 = (int)d;
}

/* Sprite coverage + discard; returns 1 and coord2D when the fragment lives. */
static int sprite_frag(const sprite_t* s, int i, int j, float* cx, float* cy) {
  const float px = (float)i + 0.5f, py = (float)j + 0.5f;
  const float lx = s->x - s->s * 0.5f, hx = s->x + s->s * 0.5f;
  const float ly = s->y - s->s * 0.5f, hy = s->y + s->s * 0.5f;
  if (!(px >= lx && px < hx && py >= ly && py < hy)) return 0;
  const float ps = (px - s->x) / s->s + 0.5f, pt = (py - s->y) / s->s + 0.5f;
  const float x = ps * 2.0f - 1.0f, y = pt * 2.0f - 1.0f;
  if (sqrtf(x * x + y * y) >= 1.0f) return 0;
  *cx = x;
  *cy = y;
  return 1;
}

int orc_render_frame(const aq_draw_command* dc, const float* points, int32_t n_points, const float* mesh,
                     int64_t n_vertices, const uint8_t* sky, int32_t face, const uint8_t* logo, int32_t lw,
                     int32_t lh, uint8_t* rgba, float* phase_out) {
  if (!dc || !rgba || dc->window_width <= 0 || dc->window_height <= 0 || n_points < 0 || n_vertices < 0) return -1;
  if (dc->render_mode < 0 || dc->render_mode > AQ_RENDER_NONE || dc->environment_mode < 0 ||
      dc->environment_mode > AQ_ENV_CHESS_BOARD)
    return -1;
  const int W = dc->window_width, H = dc->window_height;
  const size_t npx = (size_t)W * H;
  fb_t fb = {W, H, rgba, (uint32_t*)malloc(npx * sizeof(uint32_t))};
  float* phase = (float*)calloc(npx * 4, sizeof(float));
  if (!fb.depth || !phase) { free(fb.depth); free(phase); return -1; }
  for (size_t p = 0; p < npx; ++p) {
    rgba[p * 4 + 0] = 0; rgba[p * 4 + 1] = 0; rgba[p * 4 + 2] = 0; rgba[p * 4 + 3] = 255;
    fb.depth[p] = 16777215u;
  }
  const int mode = dc->render_mode, env = dc->environment_mode;
  fctx_t ctx = {{dc, sky, face, logo, lw, lh}, NULL,
                V3(dc->camera_position[0], dc->camera_position[1], dc->camera_position[2])};
  const mat4 pv = mat_mul(dc->projection, dc->view);
  if (mode != AQ_RENDER_NONE) {
    /* Skybox::draw: the cube around the camera covers every pixel. */
    if (env == AQ_ENV_SKYBOX) {
      const float* V = dc->view;
      for (int j = 0; j < H; ++j)
        for (int i = 0; i < W; ++i) {
          const float xn = ((float)i + 0.5f) * 2.0f / (float)W - 1.0f;
          const float yn = ((float)j + 0.5f) * 2.0f / (float)H - 1.0f;
          const float dx = xn / dc->projection[0], dy = yn / dc->projection[5], dz = -1.0f;
          const float dir[3] = {(V[0] * dx + V[1] * dy) + V[2] * dz, (V[4] * dx + V[5] * dy) + V[6] * dz,
                                (V[8] * dx + V[9] * dy) + V[10] * dz};
          float c[4];
          orc_sample_cube(sky, face, dir, c);
          blend(&fb, (size_t)j * W + i, V4(c[0], c[1], c[2], 1.0f));
        }
    }
    /* Container::drawFace */
    mat4 model;
    int ntri;
    const float S = dc->container_size;
    if (env == AQ_ENV_CORNELL_BOX) {
      const float pad = (dc->cornell_box_size - S) / 2.0f;
      model = diag_model(S * (dc->cornell_box_size / S), -pad, -pad);
      ntri = 12;
    } else if (env == AQ_ENV_CHESS_BOARD) {
      const float big = S * 100.0f;
      const float pad = (big - S) / 2.0f;
      model = diag_model(S * (big / S), -pad, -pad);
      ntri = 2;
    } else {
      model = diag_model(S, 0.0f, 0.0f);
      ntri = 2;
    }
    const mat4 mvp = mat_mul(pv.m, model.m);
    for (int t = 0; t < ntri; ++t) {
      tv_t v[3];
      int ok = 1;
      for (int k = 0; k < 3; ++k) ok &= tri_vertex(mvp.m, model.m, kCubeTris[t * 3 + k], NULL, W, H, &v[k]);
      if (ok) raster_tri(&fb, v[0], v[1], v[2], frag_container, &ctx);
    }
    if (mode <= AQ_RENDER_PHASE1_MESH) {
      const int multiphase = mode == AQ_RENDER_MULTIPHASE_MESH || mode >= AQ_RENDER_REFRACT_MESH;
      if (multiphase && points) {
        /* drawPhaseThickness: additive, no depth test, its own texture */
        const float tan_half = tanf((dc->fov * 0.01745329251994329576923690768489f) / 2.0f);
        for (int32_t n = 0; n < n_points; ++n) {
          sprite_t s;
          const float* p = points + (size_t)n * 7;
          if (!sprite_setup(pv.m, dc->view, dc, tan_half, p, &s)) continue;
          int i0, i1, j0, j1;
          sprite_range(&s, W, H, &i0, &i1, &j0, &j1);
          for (int j = j0; j <= j1; ++j)
            for (int i = i0; i <= i1; ++i) {
              float cx, cy;
              if (!sprite_frag(&s, i, j, &cx, &cy)) continue;
              float* t = phase + ((size_t)j * W + i) * 4;
              t[0] = t[0] + p[3]; t[1] = t[1] + p[4]; t[2] = t[2] + p[5]; t[3] = t[3] + p[6];
            }
        }
        ctx.phase = phase;
      }
      /* model = identity: the mesh goes through projection * view as is */
      const float ident[16] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1};
      const mat4 mmvp = pv;
      if (mesh)
        for (int64_t t = 0; t + 2 < n_vertices; t += 3) {
          tv_t v[3];
          int ok = 1;
          for (int k = 0; k < 3; ++k) {
            const float* q = mesh + (size_t)(t + k) * 6;
            ok &= tri_vertex(mmvp.m, ident, q, q + 3, W, H, &v[k]);
          }
          if (ok) raster_tri(&fb, v[0], v[1], v[2], frag_mesh, &ctx);
        }
    } else if (mode == AQ_RENDER_PARTICLES && points) {
      /* drawSimple: PointSprites_simple_fs.glsl with depth */
      const float tan_half = tanf((dc->fov * 0.01745329251994329576923690768489f) / 2.0f);
      const float* P = dc->projection;
      for (int32_t n = 0; n < n_points; ++n) {
        sprite_t s;
        const float* p = points + (size_t)n * 7;
        if (!sprite_setup(pv.m, dc->view, dc, tan_half, p, &s)) continue;
        int i0, i1, j0, j1;
        sprite_range(&s, W, H, &i0, &i1, &j0, &j1);
        for (int j = j0; j <= j1; ++j)
          for (int i = i0; i <= i1; ++i) {
            float cx, cy;
            if (!sprite_frag(&s, i, j, &cx, &cy)) continue;
            const float zs = sqrtf((1.0f - cx * cx) - cy * cy);
            float diffuse = gmax(0.0f, (0.0f * cx + 1.0f * cy) + 0.0f * zs);
            diffuse = 0.5f + diffuse / 2.0f;
            const float depth = s.vz + zs * dc->point_radius;
            /* projectZ: projection * vec4(0, 0, depth, 1) */
            const float pz = (P[0 * 4 + 2] * 0.0f + P[1 * 4 + 2] * 0.0f) + (P[2 * 4 + 2] * depth + P[3 * 4 + 2] * 1.0f);
            const float pw = (P[0 * 4 + 3] * 0.0f + P[1 * 4 + 3] * 0.0f) + (P[2 * 4 + 3] * depth + P[3 * 4 + 3] * 1.0f);
            const float fd = clamp01(0.5f * ((1.0f * (pz / pw) + 1.0f) + 0.0f));
            const size_t px = (size_t)j * W + i;
            const uint32_t d = depth24(fd);
            if (!(d < fb.depth[px])) continue;
            fb.depth[px] = d;
            blend(&fb, px, V4(diffuse * 0.0f, diffuse * 0.0f, diffuse * 1.0f, 1.0f));
          }
      }
    }
  }
  if (phase_out) memcpy(phase_out, phase, npx * 4 * sizeof(float));
  free(phase);
  free(fb.depth);
  return 0;
}

/* ---------------------------------------------------------------- camera */
static v3 euler_to_vec(double yaw, double pitch) {  /* camera.h:24-30 */
  const double r = 0.01745329251994329576923690768489;
  v3 v;
  v.x = (float)(-sin(yaw * r) * cos(pitch * r));
  v.y = (float)sin(pitch * r);
  v.z = (float)(-cos(yaw * r) * cos(pitch * r));
  return normalize3(v);
}

static v3 cross3(v3 x, v3 y) {
  return V3(x.y * y.z - y.y * x.z, x.z * y.x - y.z * x.x, x.x * y.y - y.x * x.y);
}

void orc_draw_command_default(aq_draw_command* dc, int32_t width, int32_t height, float domain_size,
                              int32_t size_y) {
  memset(dc, 0, sizeof(*dc));
  const float c = domain_size / 2.0f;
  const v3 center = V3(c, c, c);
  /* Camera(center): global yaw 0, pitch 30, radius 18; lookAtCenter */
  const v3 pos = mul3s(euler_to_vec(0.0, 30.0), 18.0f);
  const v3 front = normalize3(mul3s(pos, -1.0f));
  const v3 right = normalize3(cross3(front, V3(0.0f, 1.0f, 0.0f)));
  const v3 up = normalize3(cross3(right, front));
  const v3 eye = add3(center, pos);
  /* glm::lookAt(eye, eye + front, up) */
  const v3 f = normalize3(sub3(add3(eye, front), eye));
  const v3 s = normalize3(cross3(f, up));
  const v3 u = cross3(s, f);
  float* V = dc->view;
  V[0] = s.x; V[4] = s.y; V[8] = s.z;
  V[1] = u.x; V[5] = u.y; V[9] = u.z;
  V[2] = -f.x; V[6] = -f.y; V[10] = -f.z;
  V[12] = -dot3(s, eye); V[13] = -dot3(u, eye); V[14] = dot3(f, eye);
  V[3] = 0.0f; V[7] = 0.0f; V[11] = 0.0f; V[15] = 1.0f;
  /* glm::perspective(45, w/h, 0.1, 1000) */
  const float fovy = 45.0f, aspect = (float)width / (float)height, zn = 0.1f, zf = 1000.0f;
  const float th = tanf(fovy / 2.0f);
  float* P = dc->projection;
  P[0] = 1.0f / (aspect * th);
  P[5] = 1.0f / th;
  P[10] = -(zf + zn) / (zf - zn);
  P[11] = -1.0f;
  P[14] = -(2.0f * zf * zn) / (zf - zn);
  dc->camera_position[0] = eye.x; dc->camera_position[1] = eye.y; dc->camera_position[2] = eye.z;
  dc->window_width = width;
  dc->window_height = height;
  dc->fov = 45.0f;
  dc->near_plane = zn;
  dc->far_plane = zf;
  dc->render_mode = AQ_RENDER_MULTIPHASE_MESH;
  dc->environment_mode = AQ_ENV_SKYBOX;
  dc->light_position[0] = c; dc->light_position[1] = 15.0f; dc->light_position[2] = c;
  dc->container_size = domain_size;
  dc->cornell_box_size = domain_size * 4.0f;
  dc->point_radius = domain_size / (float)size_y;
  dc->phase_count = 2;
  const float pcol[2][4] = {{0, 0, 1, 0.2f}, {1, 0, 0, 1}};
  memcpy(dc->phase_colors, pcol, sizeof(pcol));
}
