// Host side of the particle-only solvers (aq_sph_* in include/aquarius_b200.h):
// position-based fluids and PCISPH.
//
// Reference: Fluid_3D_PBF::Fluid (Fluid/Fluid_3D_PBF.cu:270-532) and
// Fluid_3D_PCISPH::Fluid (Fluid/Fluid_3D_PCISPH.cu:236-468): init (spacing
// from the particle budget, seeding with glibc rand(), spatial hash, rest
// densities) and simulationStep.  A step is captured once as a CUDA graph
// (one per parity of the sorted/unsorted array sets) and replayed.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/aquarius_b200.h"
#include "fluid_impl.cuh"

using namespace aqb;

#define AQS_CUDA(call)                                                                           \
  do {                                                                                           \
    cudaError_t e_ = (call);                                                                     \
    if (e_ != cudaSuccess)                                                                       \
      return fail(e_ == cudaErrorMemoryAllocation ? AQ_ERR_OUT_OF_MEMORY : AQ_ERR_CUDA,          \
                  std::string(#call) + ": " + cudaGetErrorString(e_));                           \
  } while (0)

#define AQS_TRY(expr)             \
  do {                            \
    aq_status s_ = (expr);        \
    if (s_ != AQ_OK) return s_;   \
  } while (0)

namespace {

constexpr float kSize = 10.f;  // gridPhysicalSize (Fluid_3D_PBF.cuh:63, Fluid_3D_PCISPH.cuh:59)
constexpr float kPiHost = 3.14159265358979323846f;

// The array roles of k_sph.cu.
enum { A_P = 0, A_V = 1, A_Q = 2, A_L = 3, A_W = 3, A_F = 4, A_R = 5 };

// cubic_spline_kernel (Fluid/WeightKernels.cuh:196-206), host arithmetic.
float cubic_spline(float r, float radius, float radius3) {
  const float q = 2.0f * r / radius;
  if (q > 2.0f) return 0.0f;
  const float a = 0.25f / (kPiHost * radius3);
  return a * ((q > 1.0f) ? (2.0f - q) * (2.0f - q) * (2.0f - q) : ((3.0f * q - 6.0f) * q * q + 4.0f));
}

inline float clampf(float v, float lo, float hi) { return std::fmin(hi, std::fmax(lo, v)); }

}  // namespace

struct aq_sph {
  aq_sph_config cfg{};
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int method = 0, n = 0;
  float spacing = 0, kr = 0;
  int cells = 0;
  SphParams sp{};
  double time = 0.0;
  float4* arr[2][kSphArrays] = {};  // two sets; cur is the live one
  int cur = 0;
  int *key = nullptr, *slot = nullptr, *count = nullptr, *off = nullptr, *tiles = nullptr, *perm = nullptr;
  cudaGraphExec_t exec[2] = {nullptr, nullptr};
  std::vector<void*> allocs;

  ~aq_sph() {
    cudaSetDevice(device);
    if (stream) cudaStreamSynchronize(stream);
    for (auto& e : exec)
      if (e) cudaGraphExecDestroy(e);
    for (void* p : allocs) cudaFree(p);
    if (own_stream && stream) cudaStreamDestroy(stream);
  }
  int narrays() const { return method == AQ_SPH_PBF ? 4 : 6; }
  float4* A(int role) const { return arr[cur][role]; }
  template <typename T>
  aq_status alloc(T** p, size_t count_) {
    void* q = nullptr;
    AQS_CUDA(cudaMalloc(&q, std::max<size_t>(count_ * sizeof(T), 16)));
    allocs.push_back(q);
    *p = (T*)q;
    AQS_CUDA(cudaMemsetAsync(q, 0, std::max<size_t>(count_ * sizeof(T), 16), stream));
    return AQ_OK;
  }
  void invalidate() {
    for (auto& e : exec)
      if (e) { cudaGraphExecDestroy(e); e = nullptr; }
  }

  // performSpatialHashing2 on the kernel-radius grid: keys and slots, cell
  // offsets, stable placement and the gather of every array into the other
  // set, which becomes the live one.
  aq_status enq_sort() {
    AQS_CUDA(launch_sph_keys(stream, sp, A(A_P), key, slot, count, n));
    AQS_CUDA(launch_cell_scan(stream, cells, count, off, tiles));
    AQS_CUDA(launch_scatter(stream, key, slot, off, perm, n));
    SphArrays src{}, dst{};
    for (int a = 0; a < kSphArrays; ++a) {
      src.a[a] = a < narrays() ? arr[cur][a] : nullptr;
      dst.a[a] = a < narrays() ? arr[1 - cur][a] : nullptr;
    }
    AQS_CUDA(launch_sph_gather(stream, key, off, perm, src, dst, n));
    cur = 1 - cur;
    return AQ_OK;
  }

  // Fluid::simulationStep (Fluid_3D_PBF.cu:489-517, Fluid_3D_PCISPH.cu:424-448)
  aq_status enq_step() {
    if (method == AQ_SPH_PBF) {
      AQS_TRY(enq_sort());
      for (int s = 0; s < cfg.substeps; ++s) {
        AQS_CUDA(launch_pbf_predict(stream, sp, A(A_P), A(A_L), A(A_V), n));
        AQS_TRY(enq_sort());
        for (int it = 0; it < cfg.iterations; ++it) {
          AQS_CUDA(launch_pbf_lambda(stream, sp, off, A(A_P), A(A_V), A(A_Q), false, n));
          AQS_CUDA(launch_pbf_delta(stream, sp, off, A(A_Q), A(A_P), n));
        }
        AQS_CUDA(launch_pbf_update(stream, sp, A(A_P), A(A_L), A(A_V), n));
      }
    } else {
      for (int s = 0; s < cfg.substeps; ++s) {
        AQS_TRY(enq_sort());
        AQS_CUDA(launch_pci_init(stream, A(A_W), A(A_F), n));
        for (int it = 0; it < cfg.iterations; ++it) {
          AQS_CUDA(launch_pci_predict(stream, sp, A(A_P), A(A_V), A(A_Q), A(A_W), A(A_F), false, n));
          AQS_CUDA(launch_pci_density(stream, sp, off, A(A_P), A(A_V), A(A_Q), A(A_W), A(A_R), false, n));
          AQS_CUDA(launch_pci_force(stream, sp, off, A(A_P), A(A_R), A(A_F), n));
        }
        AQS_CUDA(launch_pci_predict(stream, sp, A(A_P), A(A_V), A(A_Q), A(A_W), A(A_F), true, n));
      }
    }
    return AQ_OK;
  }

  int launches_per_step() const {
    const int sorts = method == AQ_SPH_PBF ? 1 + cfg.substeps : cfg.substeps;
    const int per_sub = method == AQ_SPH_PBF ? 2 + 2 * cfg.iterations : 2 + 3 * cfg.iterations;
    return sorts * 6 + cfg.substeps * per_sub;  // a sort: keys, 3 scan kernels, scatter, gather
  }

  aq_status step(int nsteps) {
    for (int i = 0; i < nsteps; ++i) {
      const int parity = cur;
      if (!exec[parity]) {
        cudaGraph_t g = nullptr;
        AQS_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
        aq_status st = enq_step();
        cudaError_t e = cudaStreamEndCapture(stream, &g);
        if (st != AQ_OK) {
          if (g) cudaGraphDestroy(g);
          cur = parity;
          return st;
        }
        if (e != cudaSuccess) return fail(AQ_ERR_CUDA, std::string("capture: ") + cudaGetErrorString(e));
        e = cudaGraphInstantiate(&exec[parity], g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) {
          exec[parity] = nullptr;
          return fail(AQ_ERR_CUDA, std::string("instantiate: ") + cudaGetErrorString(e));
        }
        // capturing only recorded the launches: the array sets swapped on the
        // host as they will on the device, so undo that before replaying
        cur = parity;
      }
      AQS_CUDA(cudaGraphLaunch(exec[parity], stream));
      const int sorts = method == AQ_SPH_PBF ? 1 + cfg.substeps : cfg.substeps;
      cur = (parity + sorts) & 1;
      time += (double)cfg.timestep;
    }
    return AQ_OK;
  }
};

namespace {

aq_status validate(const aq_sph_config* c) {
  if (!c) return fail(AQ_ERR_INVALID_ARGUMENT, "config is NULL");
  if (c->method != AQ_SPH_PBF && c->method != AQ_SPH_PCISPH) return fail(AQ_ERR_INVALID_CONFIG, "unknown method");
  if (c->volume_count < 0 || c->volume_count > AQ_MAX_VOLUMES) return fail(AQ_ERR_INVALID_CONFIG, "volume_count");
  if (c->substeps < 1 || c->iterations < 0) return fail(AQ_ERR_INVALID_CONFIG, "substeps >= 1, iterations >= 0");
  if (c->max_particle_count < 1) return fail(AQ_ERR_INVALID_CONFIG, "max_particle_count >= 1");
  if (!(c->timestep > 0.f) || !std::isfinite(c->timestep)) return fail(AQ_ERR_INVALID_CONFIG, "timestep > 0");
  for (int k = 0; k < 3; ++k)
    if (!std::isfinite(c->gravity[k])) return fail(AQ_ERR_INVALID_CONFIG, "gravity");
  if (c->method == AQ_SPH_PBF && !std::isfinite(c->particle_jitter)) return fail(AQ_ERR_INVALID_CONFIG, "jitter");
  return AQ_OK;
}

// createSquareFluid / createSphereFluid (Fluid_3D_PBF.cu:397-472,
// Fluid_3D_PCISPH.cu:254-323), loops x, y, z.
void seed(const aq_sph_config& c, int method, float sp, HostRand& rng, std::vector<float>& pos) {
  const float S = kSize;
  for (int vi = 0; vi < c.volume_count; ++vi) {
    const aq_volume& v = c.volumes[vi];
    if (v.shape == AQ_SHAPE_SQUARE) {
      const float md = sp / 2.f;
      const float shrink = (float)((double)md - 1e-3);
      const float x0 = v.box_min[0] * S + md, y0 = v.box_min[1] * S + md, z0 = v.box_min[2] * S + md;
      const float x1 = v.box_max[0] * S - shrink, y1 = v.box_max[1] * S - shrink, z1 = v.box_max[2] * S - shrink;
      const float mag = method == AQ_SPH_PBF ? sp * c.particle_jitter : sp / 2.f;
      for (float x = x0; x <= x1; x += sp)
        for (float y = y0; y <= y1; y += sp)
          for (float z = z0; z <= z1; z += sp) {
            float jx = (float)((double)rng.random0to1() - 0.5);
            float jy = (float)((double)rng.random0to1() - 0.5);
            float jz = (float)((double)rng.random0to1() - 0.5);
            jx *= mag; jy *= mag; jz *= mag;
            pos.push_back(clampf(x + jx, md, S - md));
            pos.push_back(clampf(y + jy, md, S - md));
            pos.push_back(clampf(z + jz, md, S - md));
          }
    } else if (v.shape == AQ_SHAPE_SPHERE) {
      // PBF adds (r - 0.5) * spacing * 0.5; PCISPH draws (scale 0.01) and
      // never adds it
      const float lo = sp * 0.5f, hi = S - sp * 0.5f;
      const float cx = v.ball_center[0] * S, cy = v.ball_center[1] * S, cz = v.ball_center[2] * S;
      const float R = v.ball_radius * S;
      const double scale = method == AQ_SPH_PBF ? 0.5 : 0.01;
      for (float x = lo; x < hi; x += sp)
        for (float y = lo; y < hi; y += sp)
          for (float z = lo; z < hi; z += sp) {
            float px = x, py = y, pz = z;
            const float jx = (float)(((double)rng.random0to1() - 0.5) * sp * scale);
            const float jy = (float)(((double)rng.random0to1() - 0.5) * sp * scale);
            const float jz = (float)(((double)rng.random0to1() - 0.5) * sp * scale);
            if (method == AQ_SPH_PBF) { px += jx; py += jy; pz += jz; }
            const float ex = px - cx, ey = py - cy, ez = pz - cz;
            if (std::sqrt(ex * ex + ey * ey + ez * ez) < R) {
              pos.push_back(px);
              pos.push_back(py);
              pos.push_back(pz);
            }
          }
    }
  }
}

}  // namespace

extern "C" {

aq_status aq_sph_config_default(int32_t method, aq_sph_config* c) {
  if (!c) return fail(AQ_ERR_INVALID_ARGUMENT, "config is NULL");
  if (method != AQ_SPH_PBF && method != AQ_SPH_PCISPH) return fail(AQ_ERR_INVALID_ARGUMENT, "unknown method");
  memset(c, 0, sizeof(*c));
  c->method = method;
  c->volume_count = 2;
  c->volumes[0].shape = AQ_SHAPE_SQUARE;
  c->volumes[1].shape = AQ_SHAPE_SPHERE;
  for (int i = 0; i < 2; ++i) {
    aq_volume& v = c->volumes[i];
    v.box_max[0] = 1; v.box_max[1] = 0.1875f; v.box_max[2] = 1;
    v.ball_center[0] = 0.5f; v.ball_center[1] = 0.75f; v.ball_center[2] = 0.5f;
    v.ball_radius = 0.125f;
  }
  c->gravity[1] = -9.8f;
  if (method == AQ_SPH_PBF) {  // ConfigPBF (Fluid/FluidConfig.cuh:52-58)
    c->timestep = 0.033f; c->substeps = 4; c->iterations = 2;
  } else {  // ConfigPCISPH (Fluid/FluidConfig.cuh:60-66)
    c->timestep = 0.005f; c->substeps = 1; c->iterations = 4;
  }
  c->max_particle_count = 300000;
  c->particle_jitter = 0.05f;
  c->stiffness = 15.f;
  c->seed = 1;
  return AQ_OK;
}

aq_status aq_sph_create(const aq_sph_config* cfg, aq_sph** out) {
  if (!out) return fail(AQ_ERR_INVALID_ARGUMENT, "out is NULL");
  *out = nullptr;
  AQS_TRY(validate(cfg));
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return fail(AQ_ERR_NO_DEVICE, "no CUDA device");
  }
  if (cfg->device < 0 || cfg->device >= ndev) return fail(AQ_ERR_INVALID_CONFIG, "device ordinal out of range");
  aq_sph* s = new aq_sph();
  s->cfg = *cfg;
  s->device = cfg->device;
  s->method = cfg->method;
  auto bail = [&](aq_status st) { delete s; return st; };
  if (cudaSetDevice(s->device) != cudaSuccess) return bail(fail(AQ_ERR_CUDA, "cudaSetDevice"));
  if (cfg->stream) {
    s->stream = (cudaStream_t)cfg->stream;
  } else {
    if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess)
      return bail(fail(AQ_ERR_CUDA, "cudaStreamCreate"));
    s->own_stream = true;
  }
  // init (Fluid_3D_PBF.cu:275-300, Fluid_3D_PCISPH.cu:325-340)
  const float full = (float)cfg->max_particle_count;
  float sp = (float)std::pow((double)(kSize * kSize * kSize / full), 1.0 / 3.0);
  sp = kSize / std::ceil(kSize / sp);
  const float kr = sp * (s->method == AQ_SPH_PBF ? 2.01f : 2.f);
  const float kr2 = kr * kr, kr3 = kr2 * kr;
  s->spacing = sp;
  s->kr = kr;
  SphParams& p = s->sp;
  p.dt = cfg->timestep / (float)cfg->substeps;
  p.g = make_float3(cfg->gravity[0], cfg->gravity[1], cfg->gravity[2]);
  p.md = sp / 2.f;
  p.size = kSize;
  p.kr = kr;
  p.kr2 = kr2;
  p.kr6 = kr2 * kr2 * kr2;
  p.kr9 = p.kr6 * kr2 * kr;
  p.gx = p.gy = p.gz = (int)std::ceil(kSize / kr);
  p.s_corr_den = cubic_spline(0, kr, kr3);
  p.s_corr_k = 1e-6f;
  p.leave = (float)((double)p.md / ((double)p.dt * 1e2));
  {
    // the largest r^2 whose IEEE square root is still <= kernelRadius
    float x = kr2;
    while (std::sqrt(std::nextafter(x, INFINITY)) <= kr) x = std::nextafter(x, INFINITY);
    while (std::sqrt(x) > kr) x = std::nextafter(x, -INFINITY);
    p.skip_r2 = std::fmax(kr2, x);
  }
  if ((long long)p.gx * p.gy * p.gz >= (1ll << 31)) return bail(fail(AQ_ERR_INVALID_CONFIG, "hash grid too large"));
  s->cells = p.gx * p.gy * p.gz;
  HostRand rng(cfg->seed);
  std::vector<float> pos;
  seed(*cfg, s->method, sp, rng, pos);
  if (pos.size() / 3 >= (size_t)INT32_MAX) return bail(fail(AQ_ERR_INVALID_CONFIG, "too many particles"));
  const int n = (int)(pos.size() / 3);
  s->n = n;
  aq_status st = AQ_OK;
  for (int set = 0; set < 2 && st == AQ_OK; ++set)
    for (int a = 0; a < s->narrays() && st == AQ_OK; ++a) st = s->alloc(&s->arr[set][a], (size_t)n);
  if (st == AQ_OK) st = s->alloc(&s->key, (size_t)n);
  if (st == AQ_OK) st = s->alloc(&s->slot, (size_t)n);
  if (st == AQ_OK) st = s->alloc(&s->perm, (size_t)n);
  if (st == AQ_OK) st = s->alloc(&s->count, (size_t)s->cells + 1);
  if (st == AQ_OK) st = s->alloc(&s->off, (size_t)s->cells + 1);
  if (st == AQ_OK) st = s->alloc(&s->tiles, cell_scan_tiles(s->cells));
  if (st != AQ_OK) return bail(st);
  // Particle(float3): position = lastPosition = predictedPosition, velocity 0
  std::vector<float4> h4((size_t)n);
  for (int i = 0; i < n; ++i) h4[i] = make_float4(pos[3 * (size_t)i], pos[3 * (size_t)i + 1], pos[3 * (size_t)i + 2], 0.f);
  const int copies[2] = {A_P, s->method == AQ_SPH_PBF ? (int)A_L : (int)A_Q};
  for (int c : copies)
    if (n && cudaMemcpyAsync(s->arr[0][c], h4.data(), sizeof(float4) * n, cudaMemcpyHostToDevice, s->stream) != cudaSuccess)
      return bail(fail(AQ_ERR_CUDA, "upload"));
  // computeRestDensity: the hash, then the density pass that sets rest densities
  st = s->enq_sort();
  if (st == AQ_OK) {
    cudaError_t e = s->method == AQ_SPH_PBF
                        ? launch_pbf_lambda(s->stream, p, s->off, s->A(A_P), s->A(A_V), s->A(A_Q), true, n)
                        : launch_pci_density(s->stream, p, s->off, s->A(A_P), s->A(A_V), s->A(A_Q), s->A(A_W),
                                             s->A(A_R), true, n);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    if (e != cudaSuccess) st = fail(AQ_ERR_CUDA, std::string("init: ") + cudaGetErrorString(e));
  }
  if (st != AQ_OK) return bail(st);
  *out = s;
  return AQ_OK;
}

void aq_sph_destroy(aq_sph* s) { delete s; }

aq_status aq_sph_info_get(const aq_sph* s, aq_sph_info* info) {
  if (!s || !info) return fail(AQ_ERR_INVALID_ARGUMENT, "bad argument");
  info->particle_count = s->n;
  info->particle_spacing = s->spacing;
  info->kernel_radius = s->kr;
  info->grid_size[0] = s->sp.gx; info->grid_size[1] = s->sp.gy; info->grid_size[2] = s->sp.gz;
  info->container_size = kSize;
  return AQ_OK;
}

aq_status aq_sph_step(aq_sph* s, int32_t nsteps) {
  if (!s || nsteps < 0) return fail(AQ_ERR_INVALID_ARGUMENT, "bad argument");
  cudaSetDevice(s->device);
  return s->step(nsteps);
}

aq_status aq_sph_synchronize(aq_sph* s) {
  if (!s) return fail(AQ_ERR_INVALID_ARGUMENT, "bad argument");
  cudaSetDevice(s->device);
  AQS_CUDA(cudaStreamSynchronize(s->stream));
  return AQ_OK;
}

aq_status aq_sph_launches_per_step(const aq_sph* s, int32_t* launches) {
  if (!s || !launches) return fail(AQ_ERR_INVALID_ARGUMENT, "bad argument");
  *launches = s->launches_per_step();
  return AQ_OK;
}

aq_status aq_sph_download_state(aq_sph* s, aq_sph_state* st) {
  if (!s || !st) return fail(AQ_ERR_INVALID_ARGUMENT, "bad argument");
  if (st->particle_count != s->n) return fail(AQ_ERR_INVALID_ARGUMENT, "particle count does not match");
  cudaSetDevice(s->device);
  AQS_CUDA(cudaStreamSynchronize(s->stream));
  const size_t n = (size_t)s->n;
  st->physical_time = s->time;
  std::vector<float4> h(n);
  auto get = [&](int role) -> aq_status {
    if (n) AQS_CUDA(cudaMemcpy(h.data(), s->A(role), sizeof(float4) * n, cudaMemcpyDeviceToHost));
    return AQ_OK;
  };
  auto xyz = [&](float* dst) {
    if (!dst) return;
    for (size_t i = 0; i < n; ++i) { dst[i] = h[i].x; dst[n + i] = h[i].y; dst[2 * n + i] = h[i].z; }
  };
  auto w = [&](float* dst) {
    if (!dst) return;
    for (size_t i = 0; i < n; ++i) dst[i] = h[i].w;
  };
  AQS_TRY(get(A_P)); xyz(st->position); w(st->rest_density);
  AQS_TRY(get(A_V)); xyz(st->velocity); w(st->density);
  if (s->method == AQ_SPH_PBF) {
    AQS_TRY(get(A_L)); xyz(st->last_position);
    AQS_TRY(get(A_Q)); w(st->lambda);
  } else {
    AQS_TRY(get(A_Q)); xyz(st->predicted_position);
    AQS_TRY(get(A_W)); xyz(st->predicted_velocity); w(st->pressure);
    AQS_TRY(get(A_F)); xyz(st->pressure_force);
  }
  return AQ_OK;
}

aq_status aq_sph_upload_state(aq_sph* s, const aq_sph_state* st) {
  if (!s || !st) return fail(AQ_ERR_INVALID_ARGUMENT, "bad argument");
  if (st->particle_count != s->n) return fail(AQ_ERR_INVALID_ARGUMENT, "particle count does not match");
  const size_t n = (size_t)s->n;
  for (const float* pp : {st->position, st->last_position, st->predicted_position}) {
    if (!pp) continue;
    for (size_t i = 0; i < 3 * n; ++i)
      if (!(pp[i] >= 0.f && pp[i] <= kSize)) return fail(AQ_ERR_INVALID_ARGUMENT, "position outside the container");
  }
  cudaSetDevice(s->device);
  AQS_CUDA(cudaStreamSynchronize(s->stream));
  s->time = st->physical_time;
  std::vector<float4> h(n);
  auto edit = [&](int role, const float* x3, const float* w1) -> aq_status {
    if (!x3 && !w1) return AQ_OK;
    if (!n) return AQ_OK;
    AQS_CUDA(cudaMemcpy(h.data(), s->A(role), sizeof(float4) * n, cudaMemcpyDeviceToHost));
    for (size_t i = 0; i < n; ++i) {
      if (x3) { h[i].x = x3[i]; h[i].y = x3[n + i]; h[i].z = x3[2 * n + i]; }
      if (w1) h[i].w = w1[i];
    }
    AQS_CUDA(cudaMemcpy(s->A(role), h.data(), sizeof(float4) * n, cudaMemcpyHostToDevice));
    return AQ_OK;
  };
  AQS_TRY(edit(A_P, st->position, st->rest_density));
  AQS_TRY(edit(A_V, st->velocity, st->density));
  if (s->method == AQ_SPH_PBF) {
    AQS_TRY(edit(A_L, st->last_position, nullptr));
    AQS_TRY(edit(A_Q, nullptr, st->lambda));
  } else {
    AQS_TRY(edit(A_Q, st->predicted_position, nullptr));
    AQS_TRY(edit(A_W, st->predicted_velocity, st->pressure));
    AQS_TRY(edit(A_F, st->pressure_force, nullptr));
  }
  return AQ_OK;
}

}  // extern "C"
