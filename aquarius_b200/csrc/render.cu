// Host side of the headless frame (aq_renderer_* and aq_draw_command_default
// in include/aquarius_b200.h).
//
// Reference: the frame of main.cu:111-145 — DrawCommand (Rendering/
// DrawCommand.h:37-59) built from Camera (Rendering/Renderer3D/camera.h), then
// Skybox::draw, Container::drawFace and Fluid::draw (Fluid/Fluid_3D_FLIP.cu:
// 396-430), which feeds the point-sprite VBO (updatePositionsAndPhasesVBO,
// Fluid/Fluid_3D_kernels.cuh:69-91) and the mesher's VBO to PointSprites and
// FluidMeshRenderer.  The GL draw calls become: per-primitive setup kernels,
// a stable sort of (tile, primitive) pairs by tile, and two per-tile kernels
// (phase thickness, then the frame).

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/aquarius_b200.h"
#include "fluid_impl.cuh"

using namespace aqb;

#define AQR_CUDA(call)                                                                           \
  do {                                                                                           \
    cudaError_t e_ = (call);                                                                     \
    if (e_ != cudaSuccess)                                                                       \
      return fail(e_ == cudaErrorMemoryAllocation ? AQ_ERR_OUT_OF_MEMORY : AQ_ERR_CUDA,          \
                  std::string(#call) + ": " + cudaGetErrorString(e_));                           \
  } while (0)

#define AQR_TRY(expr)             \
  do {                            \
    aq_status s_ = (expr);        \
    if (s_ != AQ_OK) return s_;   \
  } while (0)

namespace {

// A grow-only device buffer.
template <typename T>
struct DevBuf {
  T* p = nullptr;
  size_t cap = 0;
  aq_status ensure(size_t n) {
    if (n <= cap && p) return AQ_OK;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    const size_t want = std::max<size_t>(n + n / 4, 16);
    AQR_CUDA(cudaMalloc(&p, want * sizeof(T)));
    cap = want;
    return AQ_OK;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
  }
};

// glm's mat4 * mat4 (column-major, each entry ((a0 b0 + a1 b1) + a2 b2) + a3 b3).
void mat_mul(const float* a, const float* b, float* r) {
  for (int c = 0; c < 4; ++c)
    for (int k = 0; k < 4; ++k)
      r[c * 4 + k] = ((a[0 * 4 + k] * b[c * 4 + 0] + a[1 * 4 + k] * b[c * 4 + 1]) + a[2 * 4 + k] * b[c * 4 + 2]) +
                     a[3 * 4 + k] * b[c * 4 + 3];
}

// scale(s) with the translation (tx, 0, tz): Container's model matrices
// (Container.cu:79-112; glm::translate(I, t) * glm::scale(scale(I, S), v)).
void diag_model(float s, float tx, float tz, float* m) {
  std::memset(m, 0, 16 * sizeof(float));
  m[0] = s; m[5] = s; m[10] = s; m[15] = 1.0f;
  m[12] = tx; m[14] = tz;
}

struct V3 { float x, y, z; };
V3 v3(float x, float y, float z) { return V3{x, y, z}; }
V3 operator+(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
V3 operator-(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
V3 operator*(V3 a, float s) { return v3(a.x * s, a.y * s, a.z * s); }
float dot(V3 a, V3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
V3 normalize(V3 v) { return v * (1.0f / std::sqrt(dot(v, v))); }
V3 cross(V3 x, V3 y) { return v3(x.y * y.z - y.y * x.z, x.z * y.x - y.z * x.x, x.x * y.y - y.x * x.y); }

// eulerToVec (camera.h:24-30): double trigonometry, float vector, normalised.
V3 euler_to_vec(double yaw, double pitch) {
  const double r = 0.01745329251994329576923690768489;
  V3 v;
  v.x = (float)(-std::sin(yaw * r) * std::cos(pitch * r));
  v.y = (float)std::sin(pitch * r);
  v.z = (float)(-std::cos(yaw * r) * std::cos(pitch * r));
  return normalize(v);
}

int key_bits(int ntiles) {
  int b = 1;
  while (b < 31 && (1 << b) < ntiles) ++b;
  return b;
}

}  // namespace

struct aq_renderer {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  uint8_t* sky = nullptr;
  int face = 0;
  uint8_t* logo = nullptr;
  int lw = 0, lh = 0;
  DevBuf<float4> spr, frac, phase;
  DevBuf<int> scnt, soff, sscan, tcnt, toff, tscan;
  DevBuf<RenderTri> tris, ctris;
  DevBuf<int> clive;
  DevBuf<unsigned> skeys, skeys2, tkeys, tkeys2;
  DevBuf<int> svals, svals2, tvals, tvals2;
  DevBuf<int2> srange, trange;
  DevBuf<unsigned> tload, tload2;  // sprite-tile list lengths (longest-first order)
  DevBuf<int> tids, torder;
  DevBuf<unsigned long long> totals;
  DevBuf<int> sort_tmp;
  DevBuf<uchar4> image;          // the image when the caller passes none
  DevBuf<float> points_vbo, mesh_vbo;  // aq_fluid_draw's VBOs
  const uint8_t* last_image = nullptr;
  unsigned long long* totals_host = nullptr;
  int launches = 0;
  int last_w = 0, last_h = 0;

  ~aq_renderer() {
    if (device >= 0) cudaSetDevice(device);
    if (stream) cudaStreamSynchronize(stream);
    for (auto* b : {&spr, &frac, &phase}) b->release();
    for (auto* b : {&scnt, &soff, &sscan, &tcnt, &toff, &tscan, &clive, &svals, &svals2, &tvals, &tvals2}) b->release();
    tris.release();
    ctris.release();
    skeys.release(); skeys2.release(); tkeys.release(); tkeys2.release();
    srange.release(); trange.release(); totals.release(); sort_tmp.release();
    image.release(); points_vbo.release(); mesh_vbo.release();
    tload.release(); tload2.release(); tids.release(); torder.release();
    if (sky) cudaFree(sky);
    if (logo) cudaFree(logo);
    if (totals_host) cudaFreeHost(totals_host);
    if (own_stream && stream) cudaStreamDestroy(stream);
  }

  // Stable sort of n (key, value) pairs by key into keys2/vals2, then the
  // per-tile ranges.
  aq_status sort_pairs(DevBuf<unsigned>& keys, DevBuf<unsigned>& keys2, DevBuf<int>& vals, DevBuf<int>& vals2,
                       int n, int ntiles, DevBuf<int2>& range) {
    const int bits = key_bits(ntiles);
    AQR_TRY(sort_tmp.ensure(radix_sort_temp_ints(n)));
    AQR_CUDA(radix_sort_pairs(stream, keys.p, vals.p, keys2.p, vals2.p, n, bits, false, sort_tmp.p));
    AQR_CUDA(launch_tile_ranges(stream, keys2.p, n, range.p));
    ++launches;
    return AQ_OK;
  }
};

extern "C" {

aq_status aq_draw_command_default(aq_draw_command* dc, int32_t width, int32_t height, float domain_size,
                                  int32_t size_y) {
  if (!dc || width <= 0 || height <= 0 || !(domain_size > 0.0f) || size_y <= 0)
    return fail(AQ_ERR_INVALID_ARGUMENT, "aq_draw_command_default: bad argument");
  std::memset(dc, 0, sizeof(*dc));
  const float c = domain_size / 2.0f;  // Fluid::getCenter (Fluid/Fluid_3D_FLIP.cu:728-730)
  const V3 center = v3(c, c, c);
  // Camera(center): globalYaw 0, globalPitch 30, globalRadius 18, lookAtCenter
  const V3 pos = euler_to_vec(0.0, 30.0) * 18.0f;
  const V3 front = normalize(pos * -1.0f);
  const V3 right = normalize(cross(front, v3(0.0f, 1.0f, 0.0f)));
  const V3 up = normalize(cross(right, front));
  const V3 eye = center + pos;  // getActualPosition
  // glm::lookAt(eye, eye + front, up) (right-handed)
  const V3 f = normalize((eye + front) - eye);
  const V3 s = normalize(cross(f, up));
  const V3 u = cross(s, f);
  float* V = dc->view;
  V[0] = s.x; V[4] = s.y; V[8] = s.z;
  V[1] = u.x; V[5] = u.y; V[9] = u.z;
  V[2] = -f.x; V[6] = -f.y; V[10] = -f.z;
  V[12] = -dot(s, eye); V[13] = -dot(u, eye); V[14] = dot(f, eye);
  V[15] = 1.0f;
  // glm::perspective(Camera::FOV = 45, width/height, 0.1, 1000), fovy in radians
  const float fovy = 45.0f, aspect = (float)width / (float)height, zn = 0.1f, zf = 1000.0f;
  const float th = std::tan(fovy / 2.0f);
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
  dc->light_position[0] = c; dc->light_position[1] = 15.0f; dc->light_position[2] = c;  // main.cu:124
  dc->container_size = domain_size;                  // Fluid::getContainerSize
  dc->cornell_box_size = domain_size * 4.0f;         // Container::Container (Container.cu:14)
  dc->point_radius = domain_size / (float)size_y;    // cellPhysicalSize
  dc->phase_count = 2;                               // FluidConfig (Fluid/FluidConfig.cuh:79-95)
  const float pcol[2][4] = {{0, 0, 1, 0.2f}, {1, 0, 0, 1}};
  std::memcpy(dc->phase_colors, pcol, sizeof(pcol));
  return AQ_OK;
}

aq_status aq_fluid_points_vbo(aq_fluid* f, float* vbo) {
  if (!f || !vbo) return fail(AQ_ERR_INVALID_ARGUMENT, "aq_fluid_points_vbo: bad argument");
  cudaSetDevice(f->device);
  AQR_CUDA(launch_points_vbo(f->stream, f->cur, f->n, f->multiphase ? -1 : f->phase, vbo));
  return AQ_OK;
}

aq_status aq_renderer_create(int32_t device, void* stream, aq_renderer** out) {
  if (!out) return fail(AQ_ERR_INVALID_ARGUMENT, "aq_renderer_create: out is NULL");
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0)
    return fail(AQ_ERR_NO_DEVICE, "aq_renderer_create: no CUDA device");
  if (device < 0 || device >= ndev) return fail(AQ_ERR_INVALID_ARGUMENT, "aq_renderer_create: bad device");
  AQR_CUDA(cudaSetDevice(device));
  aq_renderer* r = new aq_renderer();
  r->device = device;
  if (stream) {
    r->stream = (cudaStream_t)stream;
  } else {
    if (cudaStreamCreateWithFlags(&r->stream, cudaStreamNonBlocking) != cudaSuccess) {
      delete r;
      return fail(AQ_ERR_CUDA, "aq_renderer_create: stream");
    }
    r->own_stream = true;
  }
  if (cudaMallocHost(&r->totals_host, 2 * sizeof(unsigned long long)) != cudaSuccess) {
    delete r;
    return fail(AQ_ERR_OUT_OF_MEMORY, "aq_renderer_create: pinned memory");
  }
  *out = r;
  return AQ_OK;
}

void aq_renderer_destroy(aq_renderer* r) { delete r; }

aq_status aq_renderer_set_skybox(aq_renderer* r, const uint8_t* faces_rgb, int32_t face_size) {
  if (!r || (faces_rgb && face_size <= 0)) return fail(AQ_ERR_INVALID_ARGUMENT, "aq_renderer_set_skybox: bad argument");
  cudaSetDevice(r->device);
  AQR_CUDA(cudaStreamSynchronize(r->stream));
  if (r->sky) cudaFree(r->sky);
  r->sky = nullptr;
  r->face = 0;
  if (!faces_rgb) return AQ_OK;
  const size_t bytes = (size_t)6 * face_size * face_size * 3;
  AQR_CUDA(cudaMalloc(&r->sky, bytes));
  AQR_CUDA(cudaMemcpy(r->sky, faces_rgb, bytes, cudaMemcpyHostToDevice));
  r->face = face_size;
  return AQ_OK;
}

aq_status aq_renderer_set_logo(aq_renderer* r, const uint8_t* rgb, int32_t width, int32_t height) {
  if (!r || (rgb && (width <= 0 || height <= 0)))
    return fail(AQ_ERR_INVALID_ARGUMENT, "aq_renderer_set_logo: bad argument");
  cudaSetDevice(r->device);
  AQR_CUDA(cudaStreamSynchronize(r->stream));
  if (r->logo) cudaFree(r->logo);
  r->logo = nullptr;
  r->lw = r->lh = 0;
  if (!rgb) return AQ_OK;
  const size_t bytes = (size_t)width * height * 3;
  AQR_CUDA(cudaMalloc(&r->logo, bytes));
  AQR_CUDA(cudaMemcpy(r->logo, rgb, bytes, cudaMemcpyHostToDevice));
  r->lw = width;
  r->lh = height;
  return AQ_OK;
}

aq_status aq_renderer_draw(aq_renderer* r, const aq_draw_command* dc, const float* points, int32_t n_points,
                           const float* mesh, int64_t n_vertices, uint8_t* rgba) {
  if (!r || !dc || n_points < 0 || n_vertices < 0 || (n_points > 0 && !points) ||
      (n_vertices > 0 && !mesh))
    return fail(AQ_ERR_INVALID_ARGUMENT, "aq_renderer_draw: bad argument");
  if (dc->window_width <= 0 || dc->window_height <= 0 || dc->window_width > 16384 || dc->window_height > 16384)
    return fail(AQ_ERR_INVALID_ARGUMENT, "aq_renderer_draw: window size out of range (1..16384)");
  if (dc->render_mode < 0 || dc->render_mode > AQ_RENDER_NONE || dc->environment_mode < 0 ||
      dc->environment_mode > AQ_ENV_CHESS_BOARD)
    return fail(AQ_ERR_INVALID_ARGUMENT, "aq_renderer_draw: bad render or environment mode");
  if (n_vertices / 3 > INT_MAX) return fail(AQ_ERR_INVALID_ARGUMENT, "aq_renderer_draw: too many vertices");
  cudaSetDevice(r->device);
  cudaStream_t st = r->stream;
  r->launches = 0;

  RenderParams P{};
  P.W = dc->window_width;
  P.H = dc->window_height;
  P.tiles_x = (P.W + kRenderTile - 1) / kRenderTile;
  P.tiles_y = (P.H + kRenderTile - 1) / kRenderTile;
  P.stiles_x = (P.W + kSpriteTile - 1) / kSpriteTile;
  P.stiles_y = (P.H + kSpriteTile - 1) / kSpriteTile;
  P.mode = dc->render_mode;
  P.env = dc->environment_mode;
  mat_mul(dc->projection, dc->view, P.pv);
  std::memcpy(P.view, dc->view, sizeof(P.view));
  std::memcpy(P.proj, dc->projection, sizeof(P.proj));
  const float S = dc->container_size;
  if (P.env == AQ_ENV_CORNELL_BOX) {
    const float pad = (dc->cornell_box_size - S) / 2.0f;
    diag_model(S * (dc->cornell_box_size / S), -pad, -pad, P.model);
    P.ntri_container = 12;
  } else if (P.env == AQ_ENV_CHESS_BOARD) {
    const float big = S * 100.0f;  // Container::bigChessBoardSize
    const float pad = (big - S) / 2.0f;
    diag_model(S * (big / S), -pad, -pad, P.model);
    P.ntri_container = 2;
  } else {
    diag_model(S, 0.0f, 0.0f, P.model);
    P.ntri_container = 2;
  }
  mat_mul(P.pv, P.model, P.cmvp);
  for (int k = 0; k < 3; ++k) {
    P.cam[k] = dc->camera_position[k];
    P.light[k] = dc->light_position[k];
  }
  P.container = S;
  P.cornell = dc->cornell_box_size;
  P.radius = dc->point_radius;
  // tanHalfFOV uniform: tan(glm::radians(FOV) / 2) (Rendering/Shader.cpp:141-142)
  P.tan_half = std::tan((dc->fov * 0.01745329251994329576923690768489f) / 2.0f);
  P.phase_count = dc->phase_count;
  std::memcpy(P.phase_colors, dc->phase_colors, sizeof(P.phase_colors));
  P.sky = r->sky;
  P.face = r->face;
  P.logo = r->logo;
  P.lw = r->lw;
  P.lh = r->lh;
  const bool mesh_mode = P.mode <= AQ_RENDER_PHASE1_MESH;
  const bool multiphase = P.mode == AQ_RENDER_MULTIPHASE_MESH ||
                          (P.mode >= AQ_RENDER_REFRACT_MESH && P.mode <= AQ_RENDER_PHASE1_MESH);
  const bool need_spr = n_points > 0 && ((mesh_mode && multiphase) || P.mode == AQ_RENDER_PARTICLES);
  const int ntri = mesh_mode ? (int)(n_vertices / 3) : 0;
  const bool need_tri = ntri > 0;
  P.use_phase = (mesh_mode && multiphase && n_points > 0) ? 1 : 0;

  const int ntiles = P.tiles_x * P.tiles_y, nstiles = P.stiles_x * P.stiles_y;
  const size_t npx = (size_t)P.W * P.H;
  if (!rgba) {
    AQR_TRY(r->image.ensure(npx));
    rgba = reinterpret_cast<uint8_t*>(r->image.p);
  }
  AQR_TRY(r->phase.ensure(npx));
  AQR_TRY(r->srange.ensure((size_t)nstiles));
  AQR_TRY(r->trange.ensure((size_t)ntiles));
  AQR_TRY(r->ctris.ensure(12));
  AQR_TRY(r->clive.ensure(12));
  AQR_TRY(r->totals.ensure(2));
  AQR_CUDA(cudaMemsetAsync(r->totals.p, 0, 2 * sizeof(unsigned long long), st));
  AQR_CUDA(cudaMemsetAsync(r->srange.p, 0, sizeof(int2) * nstiles, st));
  AQR_CUDA(cudaMemsetAsync(r->trange.p, 0, sizeof(int2) * ntiles, st));
  if (need_spr) {
    const size_t n = (size_t)n_points;
    AQR_TRY(r->spr.ensure(n));
    AQR_TRY(r->frac.ensure(n));
    AQR_TRY(r->scnt.ensure(n + 1));
    AQR_TRY(r->soff.ensure(n + 1));
    AQR_TRY(r->sscan.ensure(cell_scan_tiles(n_points)));
    AQR_CUDA(cudaMemsetAsync(r->scnt.p + n, 0, sizeof(int), st));
    AQR_CUDA(launch_sprite_setup(st, P, points, n_points, r->spr.p, r->frac.p, r->scnt.p, r->totals.p));
    AQR_CUDA(launch_cell_scan(st, n_points, r->scnt.p, r->soff.p, r->sscan.p));
    r->launches += 4;
  }
  if (need_tri) {
    const size_t n = (size_t)ntri;
    AQR_TRY(r->tris.ensure(n));
    AQR_TRY(r->tcnt.ensure(n + 1));
    AQR_TRY(r->toff.ensure(n + 1));
    AQR_TRY(r->tscan.ensure(cell_scan_tiles(ntri)));
    AQR_CUDA(cudaMemsetAsync(r->tcnt.p + n, 0, sizeof(int), st));
    AQR_CUDA(launch_tri_setup(st, P, mesh, ntri, r->tris.p, r->tcnt.p, r->totals.p + 1));
    AQR_CUDA(launch_cell_scan(st, ntri, r->tcnt.p, r->toff.p, r->tscan.p));
    r->launches += 4;
  }
  if (P.mode != AQ_RENDER_NONE) {
    AQR_CUDA(launch_container_setup(st, P, r->ctris.p, r->clive.p));
    ++r->launches;
  } else {
    AQR_CUDA(cudaMemsetAsync(r->clive.p, 0, sizeof(int) * 12, st));
  }
  if (need_spr || need_tri) {
    AQR_CUDA(cudaMemcpyAsync(r->totals_host, r->totals.p, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
    AQR_CUDA(cudaStreamSynchronize(st));
    if (r->totals_host[0] > (unsigned long long)INT_MAX || r->totals_host[1] > (unsigned long long)INT_MAX)
      return fail(AQ_ERR_INVALID_ARGUMENT, "aq_renderer_draw: more than 2^31 primitive-tile pairs");
  }
  if (need_spr && r->totals_host[0] > 0) {
    const int np = (int)r->totals_host[0];
    AQR_TRY(r->skeys.ensure(np)); AQR_TRY(r->skeys2.ensure(np));
    AQR_TRY(r->svals.ensure(np)); AQR_TRY(r->svals2.ensure(np));
    AQR_CUDA(launch_sprite_emit(st, P, r->spr.p, r->soff.p, n_points, r->skeys.p, r->svals.p));
    ++r->launches;
    AQR_TRY(r->sort_pairs(r->skeys, r->skeys2, r->svals, r->svals2, np, nstiles, r->srange));
  }
  if (need_tri && r->totals_host[1] > 0) {
    const int np = (int)r->totals_host[1];
    AQR_TRY(r->tkeys.ensure(np)); AQR_TRY(r->tkeys2.ensure(np));
    AQR_TRY(r->tvals.ensure(np)); AQR_TRY(r->tvals2.ensure(np));
    AQR_CUDA(launch_tri_emit(st, P, r->tris.p, r->toff.p, ntri, r->tkeys.p, r->tvals.p));
    ++r->launches;
    AQR_TRY(r->sort_pairs(r->tkeys, r->tkeys2, r->tvals, r->tvals2, np, ntiles, r->trange));
  }
  if (P.use_phase) {
    // sprite tiles longest list first, so the heaviest start in the first wave
    AQR_TRY(r->tload.ensure(nstiles)); AQR_TRY(r->tload2.ensure(nstiles));
    AQR_TRY(r->tids.ensure(nstiles)); AQR_TRY(r->torder.ensure(nstiles));
    AQR_CUDA(launch_tile_load(st, r->srange.p, nstiles, r->tload.p, r->tids.p));
    AQR_TRY(r->sort_tmp.ensure(radix_sort_temp_ints(nstiles)));
    AQR_CUDA(radix_sort_pairs(st, r->tload.p, r->tids.p, r->tload2.p, r->torder.p, nstiles, 32, true, r->sort_tmp.p));
    AQR_CUDA(launch_phase(st, P, r->srange.p, r->torder.p, r->svals2.p, r->spr.p, r->frac.p, r->phase.p));
    r->launches += 2;
  } else {
    AQR_CUDA(cudaMemsetAsync(r->phase.p, 0, sizeof(float4) * npx, st));
  }
  AQR_TRY(r->ctris.ensure(12));
  AQR_CUDA(launch_frame(st, P, r->ctris.p, r->clive.p, r->trange.p, r->tvals2.p, r->tris.p, r->srange.p, r->svals2.p,
                        r->spr.p, r->phase.p, reinterpret_cast<uchar4*>(rgba)));
  ++r->launches;
  r->last_w = P.W;
  r->last_h = P.H;
  r->last_image = rgba;
  return AQ_OK;
}

aq_status aq_fluid_draw(aq_fluid* f, aq_renderer* r, const aq_draw_command* dc, uint8_t* rgba) {
  if (!f || !r || !dc) return fail(AQ_ERR_INVALID_ARGUMENT, "aq_fluid_draw: bad argument");
  if (dc->render_mode < 0 || dc->render_mode > AQ_RENDER_NONE)
    return fail(AQ_ERR_INVALID_ARGUMENT, "aq_fluid_draw: bad render mode");
  if (f->device != r->device) return fail(AQ_ERR_INVALID_ARGUMENT, "aq_fluid_draw: fluid and renderer on different devices");
  cudaSetDevice(f->device);
  const bool mesh_mode = dc->render_mode <= AQ_RENDER_PHASE1_MESH;
  const bool points_needed = dc->render_mode != AQ_RENDER_NONE;
  int64_t records = 0;
  if (mesh_mode) {
    // the mesher's VBO: one 90-float record per occupied cube, grown to fit
    AQR_TRY(r->mesh_vbo.ensure((size_t)90 * 4096));
    long long cap = (long long)(r->mesh_vbo.cap / 90);
    int32_t cubes = 0;
    AQR_TRY(aq_fluid_mesh(f, r->mesh_vbo.p, cap, &cubes));
    if (cubes > cap) {
      AQR_CUDA(cudaStreamSynchronize(f->stream));
      AQR_TRY(r->mesh_vbo.ensure((size_t)std::max(cubes, 1) * 90));
      cap = (long long)(r->mesh_vbo.cap / 90);
      AQR_TRY(aq_fluid_mesh(f, r->mesh_vbo.p, cap, &cubes));
    }
    records = std::min<long long>(cubes, cap);
  }
  if (points_needed && f->n > 0) {
    AQR_TRY(r->points_vbo.ensure((size_t)f->n * 7));
    AQR_CUDA(launch_points_vbo(f->stream, f->cur, f->n, f->multiphase ? -1 : f->phase, r->points_vbo.p));
  }
  AQR_CUDA(cudaStreamSynchronize(f->stream));
  return aq_renderer_draw(r, dc, points_needed ? r->points_vbo.p : nullptr, points_needed ? f->n : 0,
                          mesh_mode ? r->mesh_vbo.p : nullptr, records * 15, rgba);
}

aq_status aq_renderer_download_image(aq_renderer* r, uint8_t* host) {
  if (!r || !host) return fail(AQ_ERR_INVALID_ARGUMENT, "aq_renderer_download_image: bad argument");
  if (!r->last_image) return fail(AQ_ERR_INVALID_ARGUMENT, "aq_renderer_download_image: no frame yet");
  cudaSetDevice(r->device);
  AQR_CUDA(cudaMemcpyAsync(host, r->last_image, (size_t)r->last_w * r->last_h * 4, cudaMemcpyDeviceToHost, r->stream));
  AQR_CUDA(cudaStreamSynchronize(r->stream));
  return AQ_OK;
}

aq_status aq_renderer_synchronize(aq_renderer* r) {
  if (!r) return fail(AQ_ERR_INVALID_ARGUMENT, "aq_renderer_synchronize: NULL");
  cudaSetDevice(r->device);
  AQR_CUDA(cudaStreamSynchronize(r->stream));
  return AQ_OK;
}

aq_status aq_renderer_download_phase_thickness(aq_renderer* r, float* host) {
  if (!r || !host) return fail(AQ_ERR_INVALID_ARGUMENT, "aq_renderer_download_phase_thickness: bad argument");
  if (r->last_w <= 0) return fail(AQ_ERR_INVALID_ARGUMENT, "aq_renderer_download_phase_thickness: no frame yet");
  cudaSetDevice(r->device);
  AQR_CUDA(cudaMemcpyAsync(host, r->phase.p, sizeof(float4) * (size_t)r->last_w * r->last_h, cudaMemcpyDeviceToHost,
                           r->stream));
  AQR_CUDA(cudaStreamSynchronize(r->stream));
  return AQ_OK;
}

aq_status aq_renderer_launches(const aq_renderer* r, int32_t* launches) {
  if (!r || !launches) return fail(AQ_ERR_INVALID_ARGUMENT, "aq_renderer_launches: bad argument");
  *launches = r->launches;
  return AQ_OK;
}

}  // extern "C"
