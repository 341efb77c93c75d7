// Headless frame kernels (aq_renderer_draw in include/aquarius_b200.h).
//
// One frame of the reference's renderer (main.cu:111-145 and
// Fluid/Fluid_3D_FLIP.cu:396-430) without a graphics API.  GL draws primitive
// by primitive; here the screen is cut into 16x16-pixel tiles, every point
// sprite and triangle is listed under the tiles its footprint touches, the
// lists are sorted stably by tile (so each list keeps submission order), and
// one CTA per tile walks its lists with one thread per pixel.  Each pixel
// sees the same fragments in the same order as under GL, so depth tests,
// blending and the additive phase-thickness sums come out the same.  The
// framebuffer of a tile lives in registers for the whole pass.
//
// Fixed-function rules, shared with the CPU oracle (all float arithmetic
// rounded as written — the _rn intrinsics below keep nvcc from fusing):
//  - vertices: clip = M (p, 1) with rows summed (a0+a1)+(a2+a3) (glm's
//    mat4 * vec4); window x = (W/2) ndc.x + W/2, y likewise, z = ndc.z/2 + 1/2;
//  - triangles: dropped whole when a vertex has w <= 0, z < -w or
//    |ndc.x|, |ndc.y| > 16; window x, y snapped to 1/256 pixel; integer edge
//    functions with a top-left rule; no culling; depth linear in window
//    space, kept in [0,1]; varyings perspective-correct;
//  - points: dropped when outside the clip volume; size in [1, 2048]; a
//    pixel is covered when its centre is in [x - s/2, x + s/2) on both axes;
//  - 24-bit depth, GL_LESS; RGBA8 framebuffer, source clamped to [0,1],
//    blended SRC_ALPHA / ONE_MINUS_SRC_ALPHA, rounded to the nearest 1/255.
// The shading is the arithmetic of resources/Shaders/RayTraceEnvironment.glsl,
// Container_face_fs.glsl, FluidMeshRenderer_fs.glsl, PointSprites_*.glsl.
#include <algorithm>
#include <cstdint>

#include "aq_kernels.cuh"

namespace aqb {

namespace {

constexpr int kT = kRenderTile;  // tile edge in pixels
static_assert(kT == 16, "a CTA of 8 warps covers a 16x16 region as 8x4 blocks");

// Container::bottomData (Rendering/Renderer3D/Container.h:41-90): the unit
// cube's six faces as 12 triangles, floor first.
__constant__ float kRenderCube[108] = {
    0, 0, 0, 0, 0, 1, 1, 0, 0, 1, 0, 0, 0, 0, 1, 1, 0, 1,
    0, 1, 0, 0, 0, 0, 1, 0, 0, 1, 0, 0, 1, 1, 0, 0, 1, 0,
    0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 1, 0, 0, 1, 1, 0, 0, 1,
    1, 0, 0, 1, 0, 1, 1, 1, 1, 1, 1, 1, 1, 1, 0, 1, 0, 0,
    0, 0, 1, 0, 1, 1, 1, 1, 1, 1, 1, 1, 1, 0, 1, 0, 0, 1,
    0, 1, 0, 1, 1, 0, 1, 1, 1, 1, 1, 1, 0, 1, 1, 0, 1, 0,
};

__device__ __forceinline__ float fm(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fa(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fs(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fd(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ float fsq(float a) { return __fsqrt_rn(a); }

struct v3 { float x, y, z; };
struct v4 { float x, y, z, w; };
__device__ __forceinline__ v3 mk3(float x, float y, float z) { return v3{x, y, z}; }
__device__ __forceinline__ v4 mk4(float x, float y, float z, float w) { return v4{x, y, z, w}; }
__device__ __forceinline__ v3 add3(v3 a, v3 b) { return mk3(fa(a.x, b.x), fa(a.y, b.y), fa(a.z, b.z)); }
__device__ __forceinline__ v3 sub3(v3 a, v3 b) { return mk3(fs(a.x, b.x), fs(a.y, b.y), fs(a.z, b.z)); }
__device__ __forceinline__ v3 mul3s(v3 a, float s) { return mk3(fm(a.x, s), fm(a.y, s), fm(a.z, s)); }
__device__ __forceinline__ v3 mul3(v3 a, v3 b) { return mk3(fm(a.x, b.x), fm(a.y, b.y), fm(a.z, b.z)); }
__device__ __forceinline__ float dot3(v3 a, v3 b) { return fa(fa(fm(a.x, b.x), fm(a.y, b.y)), fm(a.z, b.z)); }
__device__ __forceinline__ v3 normalize3(v3 v) { return mul3s(v, fd(1.0f, fsq(dot3(v, v)))); }
__device__ __forceinline__ v3 reflect3(v3 i, v3 n) { return sub3(i, mul3s(mul3s(n, dot3(n, i)), 2.0f)); }
__device__ __forceinline__ float gmin(float x, float y) { return y < x ? y : x; }
__device__ __forceinline__ float gmax(float x, float y) { return x < y ? y : x; }
__device__ __forceinline__ v4 mul4s(v4 a, float s) { return mk4(fm(a.x, s), fm(a.y, s), fm(a.z, s), fm(a.w, s)); }
__device__ __forceinline__ v4 add4(v4 a, v4 b) { return mk4(fa(a.x, b.x), fa(a.y, b.y), fa(a.z, b.z), fa(a.w, b.w)); }
__device__ __forceinline__ v4 mix4(v4 x, v4 y, float a) { return add4(mul4s(x, fs(1.0f, a)), mul4s(y, a)); }

// GLSL int(float): truncation, saturating, NaN -> 0 (cvt.rzi).
__device__ __forceinline__ int f2i_trunc(float v) { return __float2int_rz(v); }

__device__ __forceinline__ v4 mat_vec(const float* m, float x, float y, float z) {
  float o[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) o[k] = fa(fa(fm(m[k], x), fm(m[4 + k], y)), fa(fm(m[8 + k], z), fm(m[12 + k], 1.0f)));
  return mk4(o[0], o[1], o[2], o[3]);
}

// ------------------------------------------------------------- samplers
__device__ __forceinline__ float texel(const uint8_t* img, int w, int h, int x, int y, int c) {
  x = x < 0 ? 0 : (x > w - 1 ? w - 1 : x);
  y = y < 0 ? 0 : (y > h - 1 ? h - 1 : y);
  return fd((float)__ldg(img + ((size_t)y * w + x) * 3 + c), 255.0f);
}

__device__ v3 sample_2d(const uint8_t* img, int w, int h, float s, float t) {
  if (!img || w <= 0 || h <= 0 || !(s == s) || !(t == t)) return mk3(0.f, 0.f, 0.f);
  const float u = fs(fm(s, (float)w), 0.5f), v = fs(fm(t, (float)h), 0.5f);
  const float fu = floorf(u), fv = floorf(v);
  const float a = fs(u, fu), b = fs(v, fv);
  const int x0 = f2i_trunc(fu), y0 = f2i_trunc(fv);
  const int x1 = x0 == 2147483647 ? x0 : x0 + 1, y1 = y0 == 2147483647 ? y0 : y0 + 1;
  float r[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const float c00 = texel(img, w, h, x0, y0, c), c10 = texel(img, w, h, x1, y0, c);
    const float c01 = texel(img, w, h, x0, y1, c), c11 = texel(img, w, h, x1, y1, c);
    r[c] = fa(fm(fa(fm(c00, fs(1.0f, a)), fm(c10, a)), fs(1.0f, b)), fm(fa(fm(c01, fs(1.0f, a)), fm(c11, a)), b));
  }
  return mk3(r[0], r[1], r[2]);
}

__device__ v3 sample_cube(const uint8_t* sky, int face, v3 d) {
  const float ax = fabsf(d.x), ay = fabsf(d.y), az = fabsf(d.z);
  int f;
  float sc, tc, ma;
  if (ax >= ay && ax >= az) {
    ma = ax;
    if (d.x >= 0.0f) { f = 0; sc = -d.z; tc = -d.y; } else { f = 1; sc = d.z; tc = -d.y; }
  } else if (ay >= az) {
    ma = ay;
    if (d.y >= 0.0f) { f = 2; sc = d.x; tc = d.z; } else { f = 3; sc = d.x; tc = -d.z; }
  } else {
    ma = az;
    if (d.z >= 0.0f) { f = 4; sc = d.x; tc = -d.y; } else { f = 5; sc = -d.x; tc = -d.y; }
  }
  const float s = fm(fa(fd(sc, ma), 1.0f), 0.5f), t = fm(fa(fd(tc, ma), 1.0f), 0.5f);
  return sample_2d(sky ? sky + (size_t)f * face * face * 3 : nullptr, face, face, s, t);
}

// ------------------------------------------------ RayTraceEnvironment.glsl
__device__ __forceinline__ v3 chess_board(float x, float z) {
  const int xi = f2i_trunc(fa(x, 100.0f)), zi = f2i_trunc(fa(z, 100.0f));
  if ((((unsigned)xi + (unsigned)zi) & 1u) == 0u) return mk3(0.5f, 0.5f, 0.5f);
  return mk3(0.8f, 0.8f, 0.8f);
}

__device__ v3 cornell_color(const RenderParams& P, v3 pos, v3 bmin, v3 bmax) {
  if (fabsf(fs(pos.z, bmax.z)) < 1e-3f) {
    const float fsx = fs(bmax.x, bmin.x), fsy = fs(bmax.y, bmin.y);
    const float lsx = fm(0.3f, fsx), lsy = fm(0.3f, fsy);
    const float lcx = fa(fm(0.5f, fsx), bmin.x), lcy = fa(fm(0.3f, fsy), bmin.y);
    const float lminx = fs(lcx, fd(lsx, 2.0f)), lminy = fs(lcy, fd(lsy, 2.0f));
    float lx = fs(pos.x, lminx), ly = fs(pos.y, lminy);
    lx = fd(lx, lsx);
    ly = fd(ly, lsy);
    lx = fs(1.0f, lx);
    ly = fs(1.0f, ly);
    if (lx >= 0.0f && lx <= 1.0f && ly >= 0.0f && ly <= 1.0f) return sample_2d(P.logo, P.lw, P.lh, lx, ly);
  }
  if (fabsf(fs(pos.y, bmin.y)) < 1e-3f) return chess_board(pos.x, pos.z);
  return mk3(0.8f, 0.8f, 0.8f);
}

__device__ __forceinline__ v3 cornell_normal(v3 pos, v3 bmin, v3 bmax) {
  if (fabsf(fs(pos.x, bmin.x)) < 1e-3f) return mk3(1, 0, 0);
  if (fabsf(fs(pos.x, bmax.x)) < 1e-3f) return mk3(-1, 0, 0);
  if (fabsf(fs(pos.y, bmin.y)) < 1e-3f) return mk3(0, 1, 0);
  if (fabsf(fs(pos.y, bmax.y)) < 1e-3f) return mk3(0, -1, 0);
  if (fabsf(fs(pos.z, bmin.z)) < 1e-3f) return mk3(0, 0, 1);
  if (fabsf(fs(pos.z, bmax.z)) < 1e-3f) return mk3(0, 0, -1);
  return mk3(0, 0, 0);
}

__device__ v4 trace_env(const RenderParams& P, v3 o, v3 d) {
  const v3 light = mk3(P.light[0], P.light[1], P.light[2]);
  if (P.env == AQ_ENV_CORNELL_BOX) {
    const float pad = fd(fs(P.cornell, P.container), 2.0f);
    const v3 bmin = mul3s(mk3(-1.0f, 0.0f, -1.0f), pad);
    const v3 bmax = add3(bmin, mk3(P.cornell, P.cornell, P.cornell));
    const v3 inv = mk3(fd(1.0f, d.x), fd(1.0f, d.y), fd(1.0f, d.z));
    const v3 tbot = mul3(inv, sub3(bmin, o)), ttop = mul3(inv, sub3(bmax, o));
    const v3 tmin = mk3(gmin(ttop.x, tbot.x), gmin(ttop.y, tbot.y), gmin(ttop.z, tbot.z));
    const v3 tmax = mk3(gmax(ttop.x, tbot.x), gmax(ttop.y, tbot.y), gmax(ttop.z, tbot.z));
    const float t0 = gmax(tmin.x, gmax(tmin.y, tmin.z));
    const float t1 = gmin(tmax.x, gmin(tmax.y, tmax.z));
    if (t0 >= t1) return mk4(0, 0, 0, 0);
    if (t1 < 0.0f) return mk4(0, 0, 0, 0);
    const float t = t0 < 0.0f ? t1 : t0;
    const v3 hit = add3(o, mul3s(d, t));
    const v3 base = cornell_color(P, hit, bmin, bmax);
    const v3 n = cornell_normal(hit, bmin, bmax);
    const v3 tl = normalize3(sub3(light, hit));
    const v3 r = mul3s(base, fa(0.1f, fm(0.5f, gmax(0.0f, dot3(n, tl)))));
    return mk4(r.x, r.y, r.z, 1.0f);
  }
  const float tg = fd(o.y, -d.y);
  const v3 hit = add3(o, mul3s(d, tg));
  if (P.env == AQ_ENV_SKYBOX) {
    if (tg > 0.0f && hit.x >= 0.0f && hit.x <= P.container && hit.z >= 0.0f && hit.z <= P.container) {
      const v3 c = chess_board(hit.x, hit.z);
      return mk4(c.x, c.y, c.z, 1.0f);
    }
    const v3 c = sample_cube(P.sky, P.face, d);
    return mk4(c.x, c.y, c.z, 1.0f);
  }
  if (tg > 0.0f) {
    const v3 tl = normalize3(sub3(light, hit));
    const v3 c = chess_board(hit.x, hit.z);
    return mul4s(mk4(c.x, c.y, c.z, 1.0f), fa(0.1f, fm(0.5f, dot3(mk3(0.0f, 1.0f, 0.0f), tl))));
  }
  return mk4(0, 0, 0, 1);
}

// ------------------------------------------------ FluidMeshRenderer_fs.glsl
__device__ v4 shade_mesh(const RenderParams& P, v3 fpos, v3 fnormal, v4 texel) {
  const int mode = P.mode;
  const v3 light = mk3(P.light[0], P.light[1], P.light[2]);
  const v3 cam = mk3(P.cam[0], P.cam[1], P.cam[2]);
  const v3 normal = normalize3(fnormal);
  if (mode == AQ_RENDER_FLAT_MESH) {
    const v3 tl = normalize3(sub3(light, fpos));
    const float l = fa(0.3f, fm(0.5f, dot3(normal, tl)));
    return mk4(l, l, l, 1.0f);
  }
  if (mode == AQ_RENDER_NORMAL_MESH) return mk4(normal.x, normal.y, normal.z, 1.0f);
  const v3 incident = normalize3(sub3(fpos, cam));
  const v3 refl = reflect3(incident, normal);
  v4 rc = trace_env(P, fpos, refl);
  {
    const v3 tl = normalize3(sub3(light, fpos));
    if (P.env == AQ_ENV_CHESS_BOARD || P.env == AQ_ENV_CORNELL_BOX) {
      const float r = 0.3f;
      rc = mul4s(rc, fa(fs(1.0f, r), fm(r, dot3(normal, tl))));
    }
  }
  if (mode == AQ_RENDER_MIRROR_MESH) return rc;
  const float n = fd(1.0f, 1.333f);
  const float w = fm(n, dot3(normal, mul3s(incident, -1.0f)));
  const float k = fsq(fa(1.0f, fm(fs(w, n), fa(w, n))));
  const v3 refr = normalize3(add3(mul3s(normal, fs(w, k)), mul3s(incident, n)));
  v4 fc;
  const bool multiphase = mode == AQ_RENDER_MULTIPHASE_MESH || (mode >= AQ_RENDER_REFRACT_MESH && mode <= AQ_RENDER_PHASE1_MESH);
  if (multiphase) {
    const v4 pt = mul4s(texel, 0.1f);
    const float thickness = fa(fa(fa(pt.x, pt.y), pt.z), pt.w);
    const float fr[4] = {fd(pt.x, thickness), fd(pt.y, thickness), fd(pt.z, thickness), fd(pt.w, thickness)};
    const float ptv[4] = {pt.x, pt.y, pt.z, pt.w};
    v4 tint = mk4(0, 0, 0, 0);
    const float ct = fa(fa(fa(fm(pt.x, P.phase_colors[3]), fm(pt.y, P.phase_colors[7])), fm(pt.z, P.phase_colors[11])),
                        fm(pt.w, P.phase_colors[15]));
    if (ct > 0.0f) {
      float cf[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) cf[i] = fd(fm(ptv[i], P.phase_colors[i * 4 + 3]), ct);
      const int pc = P.phase_count < 4 ? P.phase_count : 4;
      for (int i = 0; i < pc; ++i) {
        tint.x = fa(tint.x, fm(cf[i], P.phase_colors[i * 4 + 0]));
        tint.y = fa(tint.y, fm(cf[i], P.phase_colors[i * 4 + 1]));
        tint.z = fa(tint.z, fm(cf[i], P.phase_colors[i * 4 + 2]));
        tint.w = fa(tint.w, fm(fr[i], P.phase_colors[i * 4 + 3]));
      }
    }
    const float att = gmax(expf(fm(0.2f, -ct)), 0.2f);
    fc = mix4(tint, trace_env(P, fpos, refr), att);
    if (mode == AQ_RENDER_REFRACT_MESH) return fc;
    if (mode == AQ_RENDER_PHASE0_MESH) { const float v = fd(pt.x, 50.0f); return mk4(v, v, v, 1.0f); }
    if (mode == AQ_RENDER_PHASE1_MESH) { const float v = fd(pt.y, 50.0f); return mk4(v, v, v, 1.0f); }
  } else {
    const v4 tint = mk4(6.0f / 256.0f, 105.0f / 256.0f, 217.0f / 256.0f, 1.0f);
    fc = mix4(tint, trace_env(P, fpos, refr), 0.5f);
  }
  const float f0a = fd(fs(1.333f, 1.0f), fa(1.333f, 1.0f));
  const float f0 = fm(f0a, f0a);
  const float F = fa(f0, fm(fs(1.0f, f0), fs(1.0f, dot3(normal, mul3s(incident, -1.0f)))));
  v4 c = mix4(fc, rc, F);
  c.w = 1.0f;
  return c;
}

// ----------------------------------------------------------- framebuffer
__device__ __forceinline__ float clamp01(float v) { return fminf(fmaxf(v, 0.0f), 1.0f); }

// One RGBA8 pixel packed in a register (r in the low byte).
__device__ __forceinline__ uint32_t blend(uint32_t dst, v4 c) {
  const float src[4] = {clamp01(c.x), clamp01(c.y), clamp01(c.z), clamp01(c.w)};
  const float sa = src[3];
  uint32_t out = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const float d = fd((float)((dst >> (8 * k)) & 0xffu), 255.0f);
    const float v = fa(fm(src[k], sa), fm(d, fs(1.0f, sa)));
    out |= (uint32_t)__float2uint_rn(fm(v, 255.0f)) << (8 * k);
  }
  return out;
}

__device__ __forceinline__ uint32_t depth24(float z) { return __double2uint_rn(__dmul_rn((double)z, 16777215.0)); }

__device__ __forceinline__ long long edge(int ax, int ay, int bx, int by, int px, int py) {
  return (long long)(bx - ax) * (long long)(py - ay) - (long long)(by - ay) * (long long)(px - ax);
}

__device__ __forceinline__ bool top_left(int ax, int ay, int bx, int by) {
  const int dx = bx - ax, dy = by - ay;
  return dy < 0 || (dy == 0 && dx < 0);
}

// Vertex -> window space; false when the triangle is dropped.
__device__ bool tri_vertex(const float* mvp, const float* model, const float* p, const float* nrm, int W, int H,
                           int& X, int& Y, float& z, float& iw, float* a) {
  const v4 c = mat_vec(mvp, p[0], p[1], p[2]);
  if (!(c.w > 0.0f) || c.z < -c.w) return false;
  const float nx = fd(c.x, c.w), ny = fd(c.y, c.w), nz = fd(c.z, c.w);
  if (!(fabsf(nx) <= 16.0f) || !(fabsf(ny) <= 16.0f)) return false;
  const float hw = fm(0.5f, (float)W), hh = fm(0.5f, (float)H);
  const float xw = fa(fm(hw, nx), hw), yw = fa(fm(hh, ny), hh);
  X = __float2int_rn(fm(xw, 256.0f));
  Y = __float2int_rn(fm(yw, 256.0f));
  z = fa(fm(nz, 0.5f), 0.5f);
  iw = fd(1.0f, c.w);
  const v4 wp = mat_vec(model, p[0], p[1], p[2]);
  a[0] = fd(wp.x, wp.w); a[1] = fd(wp.y, wp.w); a[2] = fd(wp.z, wp.w);
  a[3] = nx; a[4] = ny;
  a[5] = nrm ? nrm[0] : 0.0f; a[6] = nrm ? nrm[1] : 0.0f; a[7] = nrm ? nrm[2] : 0.0f;
  return true;
}

// Builds a triangle record; false when dropped or of zero area.
__device__ bool tri_setup(const float* mvp, const float* model, const float* p0, const float* p1, const float* p2,
                          const float* n0, const float* n1, const float* n2, int W, int H, RenderTri& t) {
  int X[3], Y[3];
  float z[3], iw[3], a[3][8];
  if (!tri_vertex(mvp, model, p0, n0, W, H, X[0], Y[0], z[0], iw[0], a[0])) return false;
  if (!tri_vertex(mvp, model, p1, n1, W, H, X[1], Y[1], z[1], iw[1], a[1])) return false;
  if (!tri_vertex(mvp, model, p2, n2, W, H, X[2], Y[2], z[2], iw[2], a[2])) return false;
  long long area = edge(X[0], Y[0], X[1], Y[1], X[2], Y[2]);
  if (area == 0) return false;
  int o[3] = {0, 1, 2};
  if (area < 0) { o[1] = 2; o[2] = 1; area = -area; }
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    t.X[k] = X[o[k]]; t.Y[k] = Y[o[k]]; t.z[k] = z[o[k]]; t.iw[k] = iw[o[k]];
#pragma unroll
    for (int q = 0; q < 8; ++q) t.a[k][q] = a[o[k]][q];
  }
  t.area = area;
  t.tl = (top_left(t.X[1], t.Y[1], t.X[2], t.Y[2]) ? 1 : 0) | (top_left(t.X[2], t.Y[2], t.X[0], t.Y[0]) ? 2 : 0) |
         (top_left(t.X[0], t.Y[0], t.X[1], t.Y[1]) ? 4 : 0);
  return true;
}

// Pixel range a triangle can cover (conservative, clamped); false if empty.
__device__ bool tri_pixels(const RenderTri& t, int W, int H, int& i0, int& i1, int& j0, int& j1) {
  const int xmin = min(t.X[0], min(t.X[1], t.X[2])), xmax = max(t.X[0], max(t.X[1], t.X[2]));
  const int ymin = min(t.Y[0], min(t.Y[1], t.Y[2])), ymax = max(t.Y[0], max(t.Y[1], t.Y[2]));
  i0 = max((xmin - 128) >> 8, 0);
  i1 = min((xmax - 128 + 255) >> 8, W - 1);
  j0 = max((ymin - 128) >> 8, 0);
  j1 = min((ymax - 128 + 255) >> 8, H - 1);
  return i0 <= i1 && j0 <= j1;
}

// Coverage, depth and the interpolated varyings of pixel (i, j); false when
// the pixel is outside, on a non-top-left edge, or its depth out of range.
__device__ __forceinline__ bool tri_fragment(const RenderTri& t, int i, int j, float& z, float* a, bool want_a) {
  const int px = i * 256 + 128, py = j * 256 + 128;
  const long long w0 = edge(t.X[1], t.Y[1], t.X[2], t.Y[2], px, py);
  const long long w1 = edge(t.X[2], t.Y[2], t.X[0], t.Y[0], px, py);
  const long long w2 = edge(t.X[0], t.Y[0], t.X[1], t.Y[1], px, py);
  if (w0 < 0 || w1 < 0 || w2 < 0) return false;
  if ((w0 == 0 && !(t.tl & 1)) || (w1 == 0 && !(t.tl & 2)) || (w2 == 0 && !(t.tl & 4))) return false;
  const float area = __ll2float_rn(t.area);
  const float l0 = fd(__ll2float_rn(w0), area), l1 = fd(__ll2float_rn(w1), area), l2 = fd(__ll2float_rn(w2), area);
  z = fa(fa(fm(l0, t.z[0]), fm(l1, t.z[1])), fm(l2, t.z[2]));
  if (!(z >= 0.0f && z <= 1.0f)) return false;
  if (want_a) {
    const float q0 = fm(l0, t.iw[0]), q1 = fm(l1, t.iw[1]), q2 = fm(l2, t.iw[2]);
    const float den = fa(fa(q0, q1), q2);
#pragma unroll
    for (int k = 0; k < 8; ++k) a[k] = fd(fa(fa(fm(q0, t.a[0][k]), fm(q1, t.a[1][k])), fm(q2, t.a[2][k])), den);
  }
  return true;
}

// --------------------------------------------------------------- sprites
// Vertex stage of PointSprites_points_vs.glsl; false when the point is clipped.
__device__ bool sprite_setup(const RenderParams& P, const float* p, float4& s) {
  const v4 c = mat_vec(P.pv, p[0], p[1], p[2]);
  if (!(c.w > 0.0f) || !(c.x >= -c.w && c.x <= c.w && c.y >= -c.w && c.y <= c.w && c.z >= -c.w && c.z <= c.w))
    return false;
  const v3 d = sub3(mk3(p[0], p[1], p[2]), mk3(P.cam[0], P.cam[1], P.cam[2]));
  const float dist = fsq(dot3(d, d));
  const float half = fm(P.tan_half, dist);
  float sz = fd(fm(fd((float)P.H, 2.0f), P.radius), half);
  if (!(sz >= 1.0f)) sz = 1.0f;
  if (sz > 2048.0f) sz = 2048.0f;
  const float hw = fm(0.5f, (float)P.W), hh = fm(0.5f, (float)P.H);
  const v4 pc = mat_vec(P.view, p[0], p[1], p[2]);
  s = make_float4(fa(fm(hw, fd(c.x, c.w)), hw), fa(fm(hh, fd(c.y, c.w)), hh), sz, fd(pc.z, pc.w));
  return true;
}

__device__ __forceinline__ bool sprite_pixels(const float4& s, int W, int H, int& i0, int& i1, int& j0, int& j1) {
  const float h = fm(s.z, 0.5f);
  const float lx = fs(s.x, h), hx = fa(s.x, h), ly = fs(s.y, h), hy = fa(s.y, h);
  i0 = (int)fmaxf(floorf(fs(lx, 0.5f)), 0.0f);
  i1 = (int)fminf(ceilf(fs(hx, 0.5f)), (float)(W - 1));
  j0 = (int)fmaxf(floorf(fs(ly, 0.5f)), 0.0f);
  j1 = (int)fminf(ceilf(fs(hy, 0.5f)), (float)(H - 1));
  return i0 <= i1 && j0 <= j1;
}

// Coverage + the disc discard; coord2D out.
__device__ __forceinline__ bool sprite_fragment(const float4& s, float px, float py, float& cx, float& cy) {
  const float h = fm(s.z, 0.5f);
  if (!(px >= fs(s.x, h) && px < fa(s.x, h) && py >= fs(s.y, h) && py < fa(s.y, h))) return false;
  const float ps = fa(fd(fs(px, s.x), s.z), 0.5f), pt = fa(fd(fs(py, s.y), s.z), 0.5f);
  const float x = fs(fm(ps, 2.0f), 1.0f), y = fs(fm(pt, 2.0f), 1.0f);
  if (fsq(fa(fm(x, x), fm(y, y))) >= 1.0f) return false;
  cx = x;
  cy = y;
  return true;
}

template <int T>
__device__ __forceinline__ int tiles_of(int i0, int i1, int j0, int j1) {
  return (i1 / T - i0 / T + 1) * (j1 / T - j0 / T + 1);
}

constexpr int kS = kSpriteTile;
static_assert(kT == 2 * kS, "a 16x16 CTA region holds 2x2 sprite tiles, one per pair of 8x4 warp blocks");

// The 8x4 pixel block of warp w in the 16x16 region of CTA tile (tx, ty).
__device__ __forceinline__ int block_x(int tx, int warp) { return tx * kT + (warp & 1) * 8; }
__device__ __forceinline__ int block_y(int ty, int warp) { return ty * kT + (warp >> 1) * 4; }

// ---------------------------------------------------------------- kernels
__global__ void __launch_bounds__(256) k_sprite_setup(RenderParams P, const float* __restrict__ pts, int n,
                                                      float4* __restrict__ spr, float4* __restrict__ frac,
                                                      int* __restrict__ cnt, unsigned long long* __restrict__ total) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  int c = 0;
  if (i < n) {
    const float* p = pts + (size_t)i * 7;
    float4 s;
    int i0, i1, j0, j1;
    if (sprite_setup(P, p, s) && sprite_pixels(s, P.W, P.H, i0, i1, j0, j1)) {
      c = tiles_of<kS>(i0, i1, j0, j1);
      spr[i] = s;
      frac[i] = make_float4(p[3], p[4], p[5], p[6]);
    }
    cnt[i] = c;
  }
  unsigned long long v = (unsigned long long)c;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0 && v) atomicAdd(total, v);
}

__global__ void __launch_bounds__(256) k_sprite_emit(RenderParams P, const float4* __restrict__ spr,
                                                     const int* __restrict__ off, int n, unsigned* __restrict__ keys,
                                                     int* __restrict__ vals) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int base = off[i], c = off[i + 1] - base;
  if (c <= 0) return;
  int i0, i1, j0, j1;
  sprite_pixels(spr[i], P.W, P.H, i0, i1, j0, j1);
  int k = 0;
  for (int ty = j0 / kS; ty <= j1 / kS; ++ty)
    for (int tx = i0 / kS; tx <= i1 / kS; ++tx) {
      keys[base + k] = (unsigned)(ty * P.stiles_x + tx);
      vals[base + k] = i;
      ++k;
    }
}

__global__ void __launch_bounds__(256) k_tri_setup(RenderParams P, const float* __restrict__ mesh, int ntri,
                                                   RenderTri* __restrict__ tris, int* __restrict__ cnt,
                                                   unsigned long long* __restrict__ total) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  int c = 0;
  if (t < ntri) {
    const float* q = mesh + (size_t)t * 18;
    const float ident[16] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1};
    RenderTri tr;
    int i0, i1, j0, j1;
    if (tri_setup(P.pv, ident, q, q + 6, q + 12, q + 3, q + 9, q + 15, P.W, P.H, tr) &&
        tri_pixels(tr, P.W, P.H, i0, i1, j0, j1)) {
      c = tiles_of<kT>(i0, i1, j0, j1);
      tris[t] = tr;
    }
    cnt[t] = c;
  }
  unsigned long long v = (unsigned long long)c;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0 && v) atomicAdd(total, v);
}

__global__ void __launch_bounds__(256) k_tri_emit(RenderParams P, const RenderTri* __restrict__ tris,
                                                  const int* __restrict__ off, int ntri, unsigned* __restrict__ keys,
                                                  int* __restrict__ vals) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ntri) return;
  const int base = off[t], c = off[t + 1] - base;
  if (c <= 0) return;
  int i0, i1, j0, j1;
  tri_pixels(tris[t], P.W, P.H, i0, i1, j0, j1);
  int k = 0;
  for (int ty = j0 / kT; ty <= j1 / kT; ++ty)
    for (int tx = i0 / kT; tx <= i1 / kT; ++tx) {
      keys[base + k] = (unsigned)(ty * P.tiles_x + tx);
      vals[base + k] = t;
      ++k;
    }
}

// Container faces (Container::drawFace): at most 12 triangles, set up once.
__global__ void k_container_setup(RenderParams P, RenderTri* __restrict__ tris, int* __restrict__ live) {
  const int t = threadIdx.x;
  if (t >= P.ntri_container) return;
  RenderTri tr;
  const float* q = kRenderCube + t * 9;
  live[t] = tri_setup(P.cmvp, P.model, q, q + 3, q + 6, nullptr, nullptr, nullptr, P.W, P.H, tr) ? 1 : 0;
  tris[t] = tr;
}

__global__ void __launch_bounds__(1024) k_tile_ranges(const unsigned* __restrict__ keys, int n,
                                                      int2* __restrict__ range) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const unsigned k = keys[i];
    if (i == 0 || keys[i - 1] != k) range[k].x = i;
    if (i == n - 1 || keys[i + 1] != k) range[k].y = i + 1;
  }
}

// drawPhaseThickness: per tile, the sprites in submission order, summed.
// Each warp owns an 8x4 pixel block of the 16x16 tile; per batch of 32
// sprites it ballots which reach its block (the coverage test's own bounds)
// and visits only those, lowest index first, so every pixel still sums in
// submission order.  Inside a sprite's square, the disc test
// sqrt(cx^2 + cy^2) >= 1 of PointSprites_phase_fs.glsl is decided from the
// squared distance to the centre when that lies outside a +-2e-5 relative
// band around the radius (the rounding of the exact path is below 1e-6
// relative there), and by the exact gl_PointCoord arithmetic inside it: the
// same fragments survive as in sprite_fragment.
__global__ void __launch_bounds__(64) k_phase(RenderParams P, const int2* __restrict__ range,
                                              const int* __restrict__ order, const int* __restrict__ vals,
                                              const float4* __restrict__ spr, const float4* __restrict__ frac,
                                              float4* __restrict__ phase) {
  // One CTA of two warps per 8x8 sprite tile, the tiles taken longest list
  // first (order).  The warps run independently, each staging 32 sprites at
  // a time in its own shared slice: the square [lx, hx) x [ly, hy), centre,
  // squared-radius band, size and the fractions of the sprites that reach
  // its 8x4 block.
  __shared__ float4 s_box[2][32], s_ctr[2][32], s_frac[2][32];
  __shared__ float s_size[2][32];
  const int st = order[blockIdx.x];
  const int sx = st % P.stiles_x, sy = st / P.stiles_x;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int bx = sx * kS, by = sy * kS + warp * 4;  // the warp's 8x4 block
  const int i = bx + (lane & 7), j = by + (lane >> 3);
  const float px = fa((float)i, 0.5f), py = fa((float)j, 0.5f);
  const float bx0 = fa((float)bx, 0.5f), bx1 = fa((float)(bx + 7), 0.5f);
  const float by0 = fa((float)by, 0.5f), by1 = fa((float)(by + 3), 0.5f);
  float4* box = s_box[warp];
  float4* ctr = s_ctr[warp];
  float4* fr = s_frac[warp];
  float* sz = s_size[warp];
  const int2 r = range[st];
  float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
  for (int b = r.x; b < r.y; b += 32) {
    const int k = b + lane;
    bool hit = false;
    __syncwarp();
    if (k < r.y) {
      const int id = __ldg(vals + k);
      const float4 sp = __ldg(spr + id);
      const float h = fm(sp.z, 0.5f), R2 = fm(h, h);
      const float4 bk = make_float4(fs(sp.x, h), fa(sp.x, h), fs(sp.y, h), fa(sp.y, h));
      hit = bx1 >= bk.x && bx0 < bk.y && by1 >= bk.z && by0 < bk.w;
      if (hit) {
        box[lane] = bk;
        ctr[lane] = make_float4(sp.x, sp.y, fm(R2, 0.99998f), fm(R2, 1.00002f));
        sz[lane] = sp.z;
        fr[lane] = __ldg(frac + id);
      }
    }
    unsigned mask = __ballot_sync(0xffffffffu, hit);
    __syncwarp();
    while (mask) {
      const int q = __ffs(mask) - 1;
      mask &= mask - 1;
      const float4 bq = box[q];
      if (!(px >= bq.x && px < bq.y && py >= bq.z && py < bq.w)) continue;
      const float4 c = ctr[q];
      const float dx = fs(px, c.x), dy = fs(py, c.y);
      const float r2 = fa(fm(dx, dx), fm(dy, dy));
      if (r2 > c.w) continue;
      if (!(r2 < c.z)) {  // the band: the exact gl_PointCoord arithmetic
        const float S = sz[q];
        const float ps = fa(fd(dx, S), 0.5f), pt = fa(fd(dy, S), 0.5f);
        const float x = fs(fm(ps, 2.0f), 1.0f), y = fs(fm(pt, 2.0f), 1.0f);
        if (!(fsq(fa(fm(x, x), fm(y, y))) < 1.0f)) continue;
      }
      const float4 f = fr[q];
      acc.x = fa(acc.x, f.x); acc.y = fa(acc.y, f.y); acc.z = fa(acc.z, f.z); acc.w = fa(acc.w, f.w);
    }
  }
  if (i < P.W && j < P.H) phase[(size_t)j * P.W + i] = acc;
}

// Sprite-tile list lengths (sort keys for the longest-first order) and tile ids.
__global__ void __launch_bounds__(256) k_tile_load(const int2* __restrict__ range, int n, unsigned* __restrict__ load,
                                                   int* __restrict__ ids) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int2 r = range[t];
  load[t] = (unsigned)(r.y - r.x);
  ids[t] = t;
}

// The frame: background, container faces, then the mesh or the shaded sprites.
__global__ void __launch_bounds__(kT * kT) k_frame(RenderParams P, const RenderTri* __restrict__ ctris,
                                                   const int* __restrict__ clive, const int2* __restrict__ trange,
                                                   const int* __restrict__ tvals, const RenderTri* __restrict__ tris,
                                                   const int2* __restrict__ srange, const int* __restrict__ svals,
                                                   const float4* __restrict__ spr, const float4* __restrict__ phase,
                                                   uchar4* __restrict__ rgba) {
  __shared__ float4 s_spr[8][32];
  const int tile = blockIdx.x;
  const int tx = tile % P.tiles_x, ty = tile / P.tiles_x;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int bx = block_x(tx, warp), by = block_y(ty, warp);  // the warp's 8x4 block
  const int i = bx + (lane & 7), j = by + (lane >> 3);
  const bool inside = i < P.W && j < P.H;
  uint32_t color = 0xff000000u;  // (0,0,0,1)
  uint32_t depth = 16777215u;
  const v3 cam = mk3(P.cam[0], P.cam[1], P.cam[2]);
  if (P.mode != AQ_RENDER_NONE) {
    if (P.env == AQ_ENV_SKYBOX && inside) {
      const float xn = fs(fd(fm(fa((float)i, 0.5f), 2.0f), (float)P.W), 1.0f);
      const float yn = fs(fd(fm(fa((float)j, 0.5f), 2.0f), (float)P.H), 1.0f);
      const float dx = fd(xn, P.proj[0]), dy = fd(yn, P.proj[5]), dz = -1.0f;
      const float* V = P.view;
      const v3 dir = mk3(fa(fa(fm(V[0], dx), fm(V[1], dy)), fm(V[2], dz)), fa(fa(fm(V[4], dx), fm(V[5], dy)), fm(V[6], dz)),
                         fa(fa(fm(V[8], dx), fm(V[9], dy)), fm(V[10], dz)));
      const v3 c = sample_cube(P.sky, P.face, dir);
      color = blend(color, mk4(c.x, c.y, c.z, 1.0f));
    }
    if (inside)
      for (int t = 0; t < P.ntri_container; ++t) {
        if (!clive[t]) continue;
        const RenderTri& tr = ctris[t];
        float z, a[8];
        if (!tri_fragment(tr, i, j, z, a, true)) continue;
        const uint32_t d = depth24(z);
        if (!(d < depth)) continue;
        depth = d;
        const v3 dir = normalize3(sub3(mk3(a[0], a[1], a[2]), cam));
        color = blend(color, trace_env(P, cam, dir));
      }
    if (P.mode <= AQ_RENDER_PHASE1_MESH) {
      const int2 r = trange[tile];
      if (inside)
        for (int k = r.x; k < r.y; ++k) {
          const RenderTri& tr = tris[__ldg(tvals + k)];
          float z, a[8];
          if (!tri_fragment(tr, i, j, z, a, false)) continue;
          const uint32_t d = depth24(z);
          if (!(d < depth)) continue;
          tri_fragment(tr, i, j, z, a, true);
          depth = d;
          v4 tex = mk4(0.f, 0.f, 0.f, 0.f);
          if (P.use_phase) {
            const float u = fd(fa(a[3], 1.0f), 2.0f), v = fd(fa(a[4], 1.0f), 2.0f);
            const float fu = floorf(fm(u, (float)P.W)), fv = floorf(fm(v, (float)P.H));
            int ti = 0, tj = 0;
            if (fu == fu && fabsf(fu) < 1e9f) { ti = (int)fu % P.W; if (ti < 0) ti += P.W; }
            if (fv == fv && fabsf(fv) < 1e9f) { tj = (int)fv % P.H; if (tj < 0) tj += P.H; }
            const float4 t4 = phase[(size_t)tj * P.W + ti];
            tex = mk4(t4.x, t4.y, t4.z, t4.w);
          }
          color = blend(color, shade_mesh(P, mk3(a[0], a[1], a[2]), mk3(a[5], a[6], a[7]), tex));
        }
    } else if (P.mode == AQ_RENDER_PARTICLES) {
      // the warp walks its sprite tile's list, 32 sprites at a time, visiting
      // those that reach its block lowest index first
      const int sx = bx / kS, sy = by / kS;
      const int2 r = (sx < P.stiles_x && sy < P.stiles_y) ? srange[sy * P.stiles_x + sx] : make_int2(0, 0);
      const float px = fa((float)i, 0.5f), py = fa((float)j, 0.5f);
      const float bx0 = fa((float)bx, 0.5f), bx1 = fa((float)(bx + 7), 0.5f);
      const float by0 = fa((float)by, 0.5f), by1 = fa((float)(by + 3), 0.5f);
      const float* Pm = P.proj;
      float4* ws = s_spr[warp];
      for (int b = r.x; b < r.y; b += 32) {
        const int kk = b + lane;
        bool hit = false;
        __syncwarp();
        if (kk < r.y) {
          const float4 sk = __ldg(spr + __ldg(svals + kk));
          const float h = fm(sk.z, 0.5f);
          hit = bx1 >= fs(sk.x, h) && bx0 < fa(sk.x, h) && by1 >= fs(sk.y, h) && by0 < fa(sk.y, h);
          if (hit) ws[lane] = sk;
        }
        unsigned mask = __ballot_sync(0xffffffffu, hit);
        __syncwarp();
        if (!inside) continue;
        while (mask) {
          const int q = __ffs(mask) - 1;
          mask &= mask - 1;
          float cx, cy;
          const float4 s = ws[q];
          if (!sprite_fragment(s, px, py, cx, cy)) continue;
          const float zs = fsq(fs(fs(1.0f, fm(cx, cx)), fm(cy, cy)));
          float diffuse = gmax(0.0f, fa(fa(fm(0.0f, cx), fm(1.0f, cy)), fm(0.0f, zs)));
          diffuse = fa(0.5f, fd(diffuse, 2.0f));
          const float dep = fa(s.w, fm(zs, P.radius));
          const float pz = fa(fa(fm(Pm[2], 0.0f), fm(Pm[6], 0.0f)), fa(fm(Pm[10], dep), fm(Pm[14], 1.0f)));
          const float pw = fa(fa(fm(Pm[3], 0.0f), fm(Pm[7], 0.0f)), fa(fm(Pm[11], dep), fm(Pm[15], 1.0f)));
          const float fdp = clamp01(fm(0.5f, fa(fa(fm(1.0f, fd(pz, pw)), 1.0f), 0.0f)));
          const uint32_t d = depth24(fdp);
          if (!(d < depth)) continue;
          depth = d;
          color = blend(color, mk4(fm(diffuse, 0.0f), fm(diffuse, 0.0f), fm(diffuse, 1.0f), 1.0f));
        }
      }
    }
  }
  if (inside)
    rgba[(size_t)j * P.W + i] = make_uchar4(color & 0xffu, (color >> 8) & 0xffu, (color >> 16) & 0xffu, color >> 24);
}

__global__ void __launch_bounds__(256) k_points_vbo(Particles cur, int n, int phase, float* __restrict__ vbo) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float* o = vbo + (size_t)i * 7;
  o[0] = cur.px[i]; o[1] = cur.py[i]; o[2] = cur.pz[i];
  float4 f = make_float4(phase == 0 ? 1.f : 0.f, phase == 1 ? 1.f : 0.f, phase == 2 ? 1.f : 0.f, phase == 3 ? 1.f : 0.f);
  if (cur.frac) f = cur.frac[i];
  o[3] = f.x; o[4] = f.y; o[5] = f.z; o[6] = f.w;
}

}  // namespace

cudaError_t launch_sprite_setup(cudaStream_t st, const RenderParams& P, const float* pts, int n, float4* spr,
                                float4* frac, int* cnt, unsigned long long* total) {
  if (n <= 0) return cudaSuccess;
  k_sprite_setup<<<(n + 255) / 256, 256, 0, st>>>(P, pts, n, spr, frac, cnt, total);
  return cudaGetLastError();
}

cudaError_t launch_sprite_emit(cudaStream_t st, const RenderParams& P, const float4* spr, const int* off, int n,
                               unsigned* keys, int* vals) {
  if (n <= 0) return cudaSuccess;
  k_sprite_emit<<<(n + 255) / 256, 256, 0, st>>>(P, spr, off, n, keys, vals);
  return cudaGetLastError();
}

cudaError_t launch_tri_setup(cudaStream_t st, const RenderParams& P, const float* mesh, int ntri, RenderTri* tris,
                             int* cnt, unsigned long long* total) {
  if (ntri <= 0) return cudaSuccess;
  k_tri_setup<<<(ntri + 255) / 256, 256, 0, st>>>(P, mesh, ntri, tris, cnt, total);
  return cudaGetLastError();
}

cudaError_t launch_tri_emit(cudaStream_t st, const RenderParams& P, const RenderTri* tris, const int* off, int ntri,
                            unsigned* keys, int* vals) {
  if (ntri <= 0) return cudaSuccess;
  k_tri_emit<<<(ntri + 255) / 256, 256, 0, st>>>(P, tris, off, ntri, keys, vals);
  return cudaGetLastError();
}

cudaError_t launch_container_setup(cudaStream_t st, const RenderParams& P, RenderTri* tris, int* live) {
  k_container_setup<<<1, 32, 0, st>>>(P, tris, live);
  return cudaGetLastError();
}

cudaError_t launch_tile_ranges(cudaStream_t st, const unsigned* keys, int n, int2* range) {
  if (n <= 0) return cudaSuccess;
  k_tile_ranges<<<std::min((n + 1023) / 1024, 148 * 8), 1024, 0, st>>>(keys, n, range);
  return cudaGetLastError();
}

cudaError_t launch_phase(cudaStream_t st, const RenderParams& P, const int2* range, const int* order,
                         const int* vals, const float4* spr, const float4* frac, float4* phase) {
  k_phase<<<P.stiles_x * P.stiles_y, 64, 0, st>>>(P, range, order, vals, spr, frac, phase);
  return cudaGetLastError();
}

cudaError_t launch_tile_load(cudaStream_t st, const int2* range, int n, unsigned* load, int* ids) {
  if (n <= 0) return cudaSuccess;
  k_tile_load<<<(n + 255) / 256, 256, 0, st>>>(range, n, load, ids);
  return cudaGetLastError();
}

cudaError_t launch_frame(cudaStream_t st, const RenderParams& P, const RenderTri* ctris, const int* clive,
                         const int2* trange, const int* tvals, const RenderTri* tris, const int2* srange,
                         const int* svals, const float4* spr, const float4* phase, uchar4* rgba) {
  k_frame<<<P.tiles_x * P.tiles_y, kT * kT, 0, st>>>(P, ctris, clive, trange, tvals, tris, srange, svals, spr, phase,
                                                      rgba);
  return cudaGetLastError();
}

cudaError_t launch_points_vbo(cudaStream_t st, Particles cur, int n, int phase, float* vbo) {
  if (n <= 0) return cudaSuccess;
  k_points_vbo<<<(n + 255) / 256, 256, 0, st>>>(cur, n, phase, vbo);
  return cudaGetLastError();
}

}  // namespace aqb
