/*
 * Headless harness around the reference's own particle-only solvers — TEST
 * INFRASTRUCTURE ONLY.  Built by oracle/Makefile (target `sph`) into
 * oracle/_ref/libaqsph.so from Fluid/Fluid_3D_PBF.cu and
 * Fluid/Fluid_3D_PCISPH.cu where they lie, with the same headless render
 * stand-ins as the FLIP harness.  It drives Fluid_3D_PBF::Fluid and
 * Fluid_3D_PCISPH::Fluid through init / simulationStep (main.cu:158-170)
 * and copies their Particle arrays to and from the aq_sph_state layout.
 */
#include <cstdlib>
#include <cstring>
#include <vector>

#include "Common/GpuCommons.h"

// Fluid_3D_PBF::simulationStep times its iterations with GLFW's clock and
// discards the values; headless there is no GLFW.
static inline double glfwGetTime() { return 0.0; }

#include "Fluid/Fluid_3D_common.cu"
#include "Fluid/Fluid_3D_kernels.cu"
#include "Fluid/MAC_Grid_3D.cu"
#include "Fluid/Fluid_3D_PBF.cu"
#include "Fluid/Fluid_3D_PCISPH.cu"

#include "../include/aquarius_b200.h"

cudaError_t aqref_first_error = cudaSuccess;

namespace {

struct SphRun {
  int method = 0;
  Fluid_3D_PBF::Fluid* pbf = nullptr;
  Fluid_3D_PCISPH::Fluid* pci = nullptr;
  int n() const { return pbf ? pbf->particleCount : pci->particleCount; }
};

FluidConfig to_fluid_config(const aq_sph_config* c) {
  FluidConfig fc;
  fc.method = c->method == AQ_SPH_PBF ? "PBF" : "PCISPH";
  fc.initialVolumes.clear();
  for (int i = 0; i < c->volume_count; ++i) {
    const aq_volume& v = c->volumes[i];
    InitializationVolume iv(v.shape == AQ_SHAPE_SPHERE ? ShapeType::Sphere : ShapeType::Square);
    iv.boxMin = make_float3(v.box_min[0], v.box_min[1], v.box_min[2]);
    iv.boxMax = make_float3(v.box_max[0], v.box_max[1], v.box_max[2]);
    iv.ballCenter = make_float3(v.ball_center[0], v.ball_center[1], v.ball_center[2]);
    iv.ballRadius = v.ball_radius;
    fc.initialVolumes.push_back(iv);
  }
  fc.gravity = make_float3(c->gravity[0], c->gravity[1], c->gravity[2]);
  fc.PBF.timestep = c->timestep;
  fc.PBF.substeps = c->substeps;
  fc.PBF.iterations = c->iterations;
  fc.PBF.maxParticleCount = c->max_particle_count;
  fc.PBF.particleJitter = c->particle_jitter;
  fc.PCISPH.timestep = c->timestep;
  fc.PCISPH.substeps = c->substeps;
  fc.PCISPH.iterations = c->iterations;
  fc.PCISPH.maxParticleCount = c->max_particle_count;
  fc.PCISPH.stiffness = c->stiffness;
  return fc;
}

template <typename P>
void to_planes(const std::vector<P>& ps, float* dst, float3 P::*m) {
  if (!dst) return;
  const size_t n = ps.size();
  for (size_t i = 0; i < n; ++i) {
    dst[i] = (ps[i].*m).x;
    dst[n + i] = (ps[i].*m).y;
    dst[2 * n + i] = (ps[i].*m).z;
  }
}

template <typename P>
void from_planes(std::vector<P>& ps, const float* src, float3 P::*m) {
  if (!src) return;
  const size_t n = ps.size();
  for (size_t i = 0; i < n; ++i) ps[i].*m = make_float3(src[i], src[n + i], src[2 * n + i]);
}

template <typename P>
void to_scalar(const std::vector<P>& ps, float* dst, float P::*m) {
  if (!dst) return;
  for (size_t i = 0; i < ps.size(); ++i) dst[i] = ps[i].*m;
}

template <typename P>
void from_scalar(std::vector<P>& ps, const float* src, float P::*m) {
  if (!src) return;
  for (size_t i = 0; i < ps.size(); ++i) ps[i].*m = src[i];
}

}  // namespace

extern "C" {

/* srand(seed), then Fluid::init. */
void* aqsph_create(const aq_sph_config* cfg) {
  aqref_first_error = cudaSuccess;
  SphRun* r = new SphRun();
  r->method = cfg->method;
  srand(cfg->seed);
  if (cfg->method == AQ_SPH_PBF) {
    r->pbf = new Fluid_3D_PBF::Fluid();
    r->pbf->init(to_fluid_config(cfg));
  } else {
    r->pci = new Fluid_3D_PCISPH::Fluid();
    r->pci->init(to_fluid_config(cfg));
  }
  cudaDeviceSynchronize();
  if (aqref_first_error != cudaSuccess) return nullptr;
  return r;
}

void aqsph_destroy(void* h) {
  SphRun* r = (SphRun*)h;
  if (!r) return;
  delete r->pbf;
  delete r->pci;
  delete r;
}

int aqsph_count(void* h) { return ((SphRun*)h)->n(); }

int aqsph_error(void) { return (int)aqref_first_error; }

int aqsph_step(void* h, int n) {
  SphRun* r = (SphRun*)h;
  for (int i = 0; i < n; ++i) {
    if (r->pbf) r->pbf->simulationStep();
    else r->pci->simulationStep();
  }
  cudaDeviceSynchronize();
  aqref_record(cudaGetLastError(), "step", __FILE__, __LINE__);
  return (int)aqref_first_error;
}

int aqsph_get(void* h, aq_sph_state* s) {
  SphRun* r = (SphRun*)h;
  const int n = r->n();
  if (s->particle_count != n) return -2;
  cudaDeviceSynchronize();
  if (r->pbf) {
    using P = Fluid_3D_PBF::Particle;
    std::vector<P> ps(n);
    aqref_record(cudaMemcpy(ps.data(), r->pbf->particles, sizeof(P) * n, cudaMemcpyDeviceToHost), "get", __FILE__,
                 __LINE__);
    s->physical_time = r->pbf->physicalTime;
    to_planes(ps, s->position, &P::position);
    to_planes(ps, s->velocity, &P::velosity);
    to_planes(ps, s->last_position, &P::lastPosition);
    to_scalar(ps, s->density, &P::density);
    to_scalar(ps, s->rest_density, &P::restDensity);
    to_scalar(ps, s->lambda, &P::lambda);
  } else {
    using P = Fluid_3D_PCISPH::Particle;
    std::vector<P> ps(n);
    aqref_record(cudaMemcpy(ps.data(), r->pci->particles, sizeof(P) * n, cudaMemcpyDeviceToHost), "get", __FILE__,
                 __LINE__);
    s->physical_time = r->pci->physicalTime;
    to_planes(ps, s->position, &P::position);
    to_planes(ps, s->velocity, &P::velosity);
    to_planes(ps, s->pressure_force, &P::pressureForces);
    to_planes(ps, s->predicted_position, &P::predictedPosition);
    to_planes(ps, s->predicted_velocity, &P::predictedVelocity);
    to_scalar(ps, s->density, &P::density);
    to_scalar(ps, s->rest_density, &P::restDensity);
    to_scalar(ps, s->pressure, &P::pressure);
  }
  return (int)aqref_first_error;
}

int aqsph_set(void* h, const aq_sph_state* s) {
  SphRun* r = (SphRun*)h;
  const int n = r->n();
  if (s->particle_count != n) return -2;
  cudaDeviceSynchronize();
  if (r->pbf) {
    using P = Fluid_3D_PBF::Particle;
    std::vector<P> ps(n);
    aqref_record(cudaMemcpy(ps.data(), r->pbf->particles, sizeof(P) * n, cudaMemcpyDeviceToHost), "set", __FILE__,
                 __LINE__);
    r->pbf->physicalTime = (float)s->physical_time;
    from_planes(ps, s->position, &P::position);
    from_planes(ps, s->velocity, &P::velosity);
    from_planes(ps, s->last_position, &P::lastPosition);
    from_scalar(ps, s->density, &P::density);
    from_scalar(ps, s->rest_density, &P::restDensity);
    from_scalar(ps, s->lambda, &P::lambda);
    aqref_record(cudaMemcpy(r->pbf->particles, ps.data(), sizeof(P) * n, cudaMemcpyHostToDevice), "set", __FILE__,
                 __LINE__);
  } else {
    using P = Fluid_3D_PCISPH::Particle;
    std::vector<P> ps(n);
    aqref_record(cudaMemcpy(ps.data(), r->pci->particles, sizeof(P) * n, cudaMemcpyDeviceToHost), "set", __FILE__,
                 __LINE__);
    r->pci->physicalTime = (float)s->physical_time;
    from_planes(ps, s->position, &P::position);
    from_planes(ps, s->velocity, &P::velosity);
    from_planes(ps, s->pressure_force, &P::pressureForces);
    from_planes(ps, s->predicted_position, &P::predictedPosition);
    from_planes(ps, s->predicted_velocity, &P::predictedVelocity);
    from_scalar(ps, s->density, &P::density);
    from_scalar(ps, s->rest_density, &P::restDensity);
    from_scalar(ps, s->pressure, &P::pressure);
    aqref_record(cudaMemcpy(r->pci->particles, ps.data(), sizeof(P) * n, cudaMemcpyHostToDevice), "set", __FILE__,
                 __LINE__);
  }
  cudaDeviceSynchronize();
  return (int)aqref_first_error;
}

/* particleSpacing, kernelRadius, gridSize. */
void aqsph_info(void* h, float* spacing, float* kernel_radius, int* grid) {
  SphRun* r = (SphRun*)h;
  if (r->pbf) {
    *spacing = r->pbf->particleSpacing;
    *kernel_radius = r->pbf->kernelRadius;
    grid[0] = r->pbf->gridSize.x; grid[1] = r->pbf->gridSize.y; grid[2] = r->pbf->gridSize.z;
  } else {
    *spacing = r->pci->particleSpacing;
    *kernel_radius = r->pci->kernelRadius;
    grid[0] = r->pci->gridSize.x; grid[1] = r->pci->gridSize.y; grid[2] = r->pci->gridSize.z;
  }
}

}  // extern "C"
