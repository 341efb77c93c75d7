/*
 * Headless harness around the reference's own FLIP kernels — TEST
 * INFRASTRUCTURE ONLY.  Built by oracle/Makefile into oracle/_ref/libaqref.so
 * from the reference sources where they lie (a tree of file symlinks points
 * at them; the GL-bound headers resolve to oracle/ref_shim).  It drives
 * Fluid_3D_FLIP::Fluid through its public members, exactly as main.cu does
 * (main.cu:158-170, :134), and adds state dump/injection via cudaMemcpy3D on
 * the reference's cudaArrays, so the CPU oracle can be pinned against the
 * reference kernels running on the GPU.
 */
#include <cstdlib>
#include <cstring>
#include <vector>

#include "Fluid/Fluid_3D_common.cu"
#include "Fluid/Fluid_3D_kernels.cu"
#include "Fluid/MAC_Grid_3D.cu"
#include "Fluid/Fluid_3D_FLIP.cu"

#include "../include/aquarius_b200.h"

cudaError_t aqref_first_error = cudaSuccess;

namespace {

using Fluid_3D_FLIP::Particle;

struct RefFluid {
  Fluid_3D_FLIP::Fluid* f = nullptr;
  bool ink = false; /* initInkRenderer ran: inkParticles is allocated */
};

template <typename T>
void array_to_host(cudaArray* arr, int w, int h, int d, std::vector<T>& out) {
  out.resize((size_t)w * h * d);
  cudaMemcpy3DParms p;
  memset(&p, 0, sizeof(p));
  p.srcArray = arr;
  p.dstPtr = make_cudaPitchedPtr(out.data(), (size_t)w * sizeof(T), (size_t)w, (size_t)h);
  p.extent = make_cudaExtent((size_t)w, (size_t)h, (size_t)d);
  p.kind = cudaMemcpyDeviceToHost;
  aqref_record(cudaMemcpy3D(&p), "array_to_host", __FILE__, __LINE__);
}

template <typename T>
void host_to_array(cudaArray* arr, int w, int h, int d, const std::vector<T>& in) {
  cudaMemcpy3DParms p;
  memset(&p, 0, sizeof(p));
  p.dstArray = arr;
  p.srcPtr = make_cudaPitchedPtr((void*)in.data(), (size_t)w * sizeof(T), (size_t)w, (size_t)h);
  p.extent = make_cudaExtent((size_t)w, (size_t)h, (size_t)d);
  p.kind = cudaMemcpyHostToDevice;
  aqref_record(cudaMemcpy3D(&p), "host_to_array", __FILE__, __LINE__);
}

/* cudaArray element (x,y,z) sits at (z*h + y)*w + x; the canonical layout is
 * (x*h + y)*d + z.  Scalar fields. */
template <typename T>
void get_scalar(cudaArray* arr, int w, int h, int d, T* dst) {
  if (!dst) return;
  std::vector<T> tmp;
  array_to_host(arr, w, h, d, tmp);
  for (int x = 0; x < w; ++x)
    for (int y = 0; y < h; ++y)
      for (int z = 0; z < d; ++z) dst[((size_t)x * h + y) * d + z] = tmp[((size_t)z * h + y) * w + x];
}
template <typename T>
void set_scalar(cudaArray* arr, int w, int h, int d, const T* src) {
  if (!src) return;
  std::vector<T> tmp((size_t)w * h * d);
  for (int x = 0; x < w; ++x)
    for (int y = 0; y < h; ++y)
      for (int z = 0; z < d; ++z) tmp[((size_t)z * h + y) * w + x] = src[((size_t)x * h + y) * d + z];
  host_to_array(arr, w, h, d, tmp);
}
/* 4-component fields: `comps` planar components are exchanged, the rest are 0 on upload. */
template <typename V, typename S>
void get_vec4(cudaArray* arr, int w, int h, int d, int comps, S* dst) {
  if (!dst) return;
  std::vector<V> tmp;
  array_to_host(arr, w, h, d, tmp);
  size_t cnt = (size_t)w * h * d;
  for (int x = 0; x < w; ++x)
    for (int y = 0; y < h; ++y)
      for (int z = 0; z < d; ++z) {
        const V& v = tmp[((size_t)z * h + y) * w + x];
        size_t c = ((size_t)x * h + y) * d + z;
        const S e[4] = {(S)v.x, (S)v.y, (S)v.z, (S)v.w};
        for (int k = 0; k < comps; ++k) dst[k * cnt + c] = e[k];
      }
}
template <typename V, typename S>
void set_vec4(cudaArray* arr, int w, int h, int d, int comps, const S* src) {
  if (!src) return;
  size_t cnt = (size_t)w * h * d;
  std::vector<V> tmp(cnt);
  for (int x = 0; x < w; ++x)
    for (int y = 0; y < h; ++y)
      for (int z = 0; z < d; ++z) {
        size_t c = ((size_t)x * h + y) * d + z;
        S e[4] = {0, 0, 0, 0};
        for (int k = 0; k < comps; ++k) e[k] = src[k * cnt + c];
        V v;
        v.x = e[0]; v.y = e[1]; v.z = e[2]; v.w = e[3];
        tmp[((size_t)z * h + y) * w + x] = v;
      }
  host_to_array(arr, w, h, d, tmp);
}

FluidConfig to_fluid_config(const aq_config* c) {
  FluidConfig fc;
  fc.method = "FLIP";
  fc.initialVolumes.clear();
  for (int i = 0; i < c->volume_count; ++i) {
    const aq_volume& v = c->volumes[i];
    InitializationVolume iv(v.shape == AQ_SHAPE_SPHERE ? ShapeType::Sphere : ShapeType::Square);
    iv.boxMin = make_float3(v.box_min[0], v.box_min[1], v.box_min[2]);
    iv.boxMax = make_float3(v.box_max[0], v.box_max[1], v.box_max[2]);
    iv.ballCenter = make_float3(v.ball_center[0], v.ball_center[1], v.ball_center[2]);
    iv.ballRadius = v.ball_radius;
    iv.phase = v.phase;
    fc.initialVolumes.push_back(iv);
  }
  fc.gravity = make_float3(c->gravity[0], c->gravity[1], c->gravity[2]);
  fc.phaseCount = c->phase_count;
  fc.phaseDensities = make_float4(c->phase_densities[0], c->phase_densities[1], c->phase_densities[2],
                                  c->phase_densities[3]);
  fc.diffusionCoeff = c->diffusion_coeff;
  fc.FLIP.sizeX = c->size_x;
  fc.FLIP.sizeY = c->size_y;
  fc.FLIP.sizeZ = c->size_z;
  fc.FLIP.pressureIterations = c->pressure_iterations;
  fc.FLIP.diffusionIterations = c->diffusion_iterations;
  fc.FLIP.timestep = c->timestep;
  fc.FLIP.FLIPcoeff = c->flip_coeff;
  fc.FLIP.particleJitter = c->particle_jitter;
  return fc;
}

__global__ void probe_fill(VolumeData v, int w, int h, int d) {
  int x = blockIdx.x * blockDim.x + threadIdx.x;
  int y = blockIdx.y * blockDim.y + threadIdx.y;
  int z = blockIdx.z * blockDim.z + threadIdx.z;
  if (x >= w || y >= h || z >= d) return;
  v.writeSurface<float>((float)(x + 100 * y + 10000 * z), x, y, z);
}

__global__ void probe_read(VolumeData v, const float* coords, float* out, int n) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  out[i] = v.readTexture<float>(coords[3 * i], coords[3 * i + 1], coords[3 * i + 2]);
}

}  // namespace

extern "C" {

/* Creates and initialises the reference solver (Fluid::init).  srand(seed)
 * first: the reference never seeds, which equals seed 1. */
void* aqref_create(const aq_config* cfg) {
  aqref_first_error = cudaSuccess;
  RefFluid* r = new RefFluid();
  r->f = new Fluid_3D_FLIP::Fluid();
  r->f->gridPhysicalSize = cfg->domain_size;
  srand(cfg->seed);
  r->f->init(to_fluid_config(cfg));
  cudaDeviceSynchronize();
  if (aqref_first_error != cudaSuccess) {
    delete r->f;
    delete r;
    return nullptr;
  }
  return r;
}

void aqref_destroy(void* h) {
  RefFluid* r = (RefFluid*)h;
  if (!r) return;
  if (r->ink) cudaFree(r->f->inkParticles);
  delete r->f;
  delete r;
}

int aqref_particle_count(void* h) { return ((RefFluid*)h)->f->particleCount; }

int aqref_error(void) { return (int)aqref_first_error; }

int aqref_step(void* h, int n) {
  RefFluid* r = (RefFluid*)h;
  for (int i = 0; i < n; ++i) r->f->simulationStep();
  cudaDeviceSynchronize();
  return (int)aqref_first_error;
}

/* Times n simulationStep()s with CUDA events on the legacy default stream,
 * the stream every reference kernel is launched on.  The reference
 * synchronises the device inside a step (HANDLE_ERROR / CHECK_CUDA_ERROR,
 * Common/GpuCommons.h:118-142); those waits are part of its behaviour and of
 * the measured time. */
int aqref_time_steps(void* h, int n, float* ms) {
  RefFluid* r = (RefFluid*)h;
  cudaEvent_t a, b;
  aqref_record(cudaEventCreate(&a), "event", __FILE__, __LINE__);
  aqref_record(cudaEventCreate(&b), "event", __FILE__, __LINE__);
  cudaDeviceSynchronize();
  cudaEventRecord(a, 0);
  for (int i = 0; i < n; ++i) r->f->simulationStep();
  cudaEventRecord(b, 0);
  cudaEventSynchronize(b);
  float t = 0.f;
  aqref_record(cudaEventElapsedTime(&t, a, b), "elapsed", __FILE__, __LINE__);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  if (ms) *ms = t;
  return (int)aqref_first_error;
}

/* One sub-stage, with the exact calls simulationStep / transferToGrid make. */
int aqref_stage(void* h, int stage) {
  Fluid_3D_FLIP::Fluid* f = ((RefFluid*)h)->f;
  MAC_Grid_3D& g = *f->grid;
  switch (stage) {
    case AQ_STAGE_G2P_ADVECT:
      f->transferToParticles();
      f->moveParticles(f->timestep);
      break;
    case AQ_STAGE_SORT:
      performSpatialHashing2(f->particleIndices, f->particleHashes, f->particles, f->particlesCopy,
                             f->particleCount, f->cellPhysicalSize, f->sizeX, f->sizeY, f->sizeZ,
                             f->numBlocksParticle, f->numThreadsParticle, f->cellStart, f->cellEnd,
                             f->cellCount);
      break;
    case AQ_STAGE_P2G:
      Fluid_3D_FLIP::resetCellImpl<<<g.cudaGridSize, g.cudaBlockSize>>>(g.volumes, f->sizeX, f->sizeY,
                                                                       f->sizeZ, CONTENT_AIR);
      cudaDeviceSynchronize();
      Fluid_3D_FLIP::transferToCellAccumPhase<<<g.cudaGridSize, g.cudaBlockSize>>>(
          g.volumes, f->sizeX, f->sizeY, f->sizeZ, f->cellPhysicalSize, f->cellStart, f->cellEnd,
          f->particles, f->particleCount);
      Fluid_3D_FLIP::transferToCellDividePhase<<<g.cudaGridSize, g.cudaBlockSize>>>(
          g.volumes, f->sizeX, f->sizeY, f->sizeZ, f->cellPhysicalSize, f->cellStart, f->cellEnd,
          f->particles, f->particleCount);
      Fluid_3D_FLIP::transferVolumeFractionsToCell<<<g.cudaGridSize, g.cudaBlockSize>>>(
          g.volumes, f->sizeX, f->sizeY, f->sizeZ, f->cellPhysicalSize, f->cellStart, f->cellEnd,
          f->particles, f->particleCount, f->config.phaseDensities);
      applyGravity(f->timestep, g, f->config.gravity);
      fixBoundary(g);
      break;
    case AQ_STAGE_DIVERGENCE:
      f->countParticlesInCells();
      computeDivergence(g, f->particlesPerCell);
      break;
    case AQ_STAGE_PRESSURE:
      solvePressureJacobi(f->timestep, g, f->config.FLIP.pressureIterations);
      break;
    case AQ_STAGE_PROJECT:
      updateVelocityWithPressure(f->timestep, g);
      break;
    case AQ_STAGE_EXTRAPOLATE:
      extrapolateVelocity(f->timestep, g);
      break;
    case AQ_STAGE_DIFFUSE:
      solveDiffusionJacobi(f->timestep, g, f->config.FLIP.diffusionIterations, f->config.diffusionCoeff,
                           f->cellPhysicalSize);
      f->physicalTime += f->timestep;
      break;
    default:
      return -1;
  }
  cudaDeviceSynchronize();
  aqref_record(cudaGetLastError(), "stage", __FILE__, __LINE__);
  return (int)aqref_first_error;
}

int aqref_get_state(void* h, aq_host_state* s) {
  Fluid_3D_FLIP::Fluid* f = ((RefFluid*)h)->f;
  const int sx = f->sizeX, sy = f->sizeY, sz = f->sizeZ, n = f->particleCount;
  if (s->size_x != sx || s->size_y != sy || s->size_z != sz || s->particle_count != n) return -2;
  cudaDeviceSynchronize();
  VolumeCollection& v = f->grid->volumes;
  s->physical_time = f->physicalTime;
  get_scalar<int>(v.content.array, sx + 1, sy + 1, sz + 1, s->content);
  get_vec4<float4, float>(v.velocity.array, sx + 1, sy + 1, sz + 1, 3, s->velocity);
  get_vec4<float4, float>(v.newVelocity.array, sx + 1, sy + 1, sz + 1, 3, s->new_velocity);
  get_scalar<float>(v.pressure.array, sx, sy, sz, s->pressure);
  get_scalar<float>(v.divergence.array, sx, sy, sz, s->divergence);
  get_scalar<int>(v.particleCount.array, sx, sy, sz, s->particle_count_cell);
  get_vec4<int4, int32_t>(v.hasVelocity.array, sx, sy, sz, 3, s->has_velocity);
  get_vec4<float4, float>(v.volumeFractions.array, sx, sy, sz, 4, s->volume_fractions);
  get_vec4<float4, float>(v.newVolumeFractions.array, sx, sy, sz, 4, s->new_volume_fractions);
  get_scalar<float>(v.density.array, sx, sy, sz, s->density);
  const int C = sx * sy * sz;
  if (s->cell_start) aqref_record(cudaMemcpy(s->cell_start, f->cellStart, sizeof(int) * C, cudaMemcpyDeviceToHost), "cs", __FILE__, __LINE__);
  if (s->cell_end) aqref_record(cudaMemcpy(s->cell_end, f->cellEnd, sizeof(int) * C, cudaMemcpyDeviceToHost), "ce", __FILE__, __LINE__);
  if (s->particle_hash) aqref_record(cudaMemcpy(s->particle_hash, f->particleHashes, sizeof(int) * n, cudaMemcpyDeviceToHost), "ph", __FILE__, __LINE__);
  if (s->sort_index) aqref_record(cudaMemcpy(s->sort_index, f->particleIndices, sizeof(int) * n, cudaMemcpyDeviceToHost), "pi", __FILE__, __LINE__);
  if (s->position || s->velocity_p || s->fractions) {
    std::vector<Particle> ps(n);
    aqref_record(cudaMemcpy(ps.data(), f->particles, sizeof(Particle) * n, cudaMemcpyDeviceToHost), "p", __FILE__, __LINE__);
    for (int i = 0; i < n; ++i) {
      if (s->position) { s->position[i] = ps[i].position.x; s->position[n + i] = ps[i].position.y; s->position[2 * n + i] = ps[i].position.z; }
      if (s->velocity_p) { s->velocity_p[i] = ps[i].velocity.x; s->velocity_p[n + i] = ps[i].velocity.y; s->velocity_p[2 * n + i] = ps[i].velocity.z; }
      if (s->fractions) {
        s->fractions[i] = ps[i].volumeFractions.x; s->fractions[n + i] = ps[i].volumeFractions.y;
        s->fractions[2 * n + i] = ps[i].volumeFractions.z; s->fractions[3 * n + i] = ps[i].volumeFractions.w;
      }
    }
  }
  cudaDeviceSynchronize();
  return (int)aqref_first_error;
}

int aqref_set_state(void* h, const aq_host_state* s) {
  Fluid_3D_FLIP::Fluid* f = ((RefFluid*)h)->f;
  const int sx = f->sizeX, sy = f->sizeY, sz = f->sizeZ, n = f->particleCount;
  if (s->size_x != sx || s->size_y != sy || s->size_z != sz || s->particle_count != n) return -2;
  cudaDeviceSynchronize();
  VolumeCollection& v = f->grid->volumes;
  f->physicalTime = (float)s->physical_time;
  set_scalar<int>(v.content.array, sx + 1, sy + 1, sz + 1, s->content);
  set_vec4<float4, float>(v.velocity.array, sx + 1, sy + 1, sz + 1, 3, s->velocity);
  set_vec4<float4, float>(v.newVelocity.array, sx + 1, sy + 1, sz + 1, 3, s->new_velocity);
  set_scalar<float>(v.pressure.array, sx, sy, sz, s->pressure);
  set_scalar<float>(v.divergence.array, sx, sy, sz, s->divergence);
  set_scalar<int>(v.particleCount.array, sx, sy, sz, s->particle_count_cell);
  set_vec4<int4, int32_t>(v.hasVelocity.array, sx, sy, sz, 3, s->has_velocity);
  set_vec4<float4, float>(v.volumeFractions.array, sx, sy, sz, 4, s->volume_fractions);
  set_vec4<float4, float>(v.newVolumeFractions.array, sx, sy, sz, 4, s->new_volume_fractions);
  set_scalar<float>(v.density.array, sx, sy, sz, s->density);
  const int C = sx * sy * sz;
  if (s->cell_start) aqref_record(cudaMemcpy(f->cellStart, s->cell_start, sizeof(int) * C, cudaMemcpyHostToDevice), "cs", __FILE__, __LINE__);
  if (s->cell_end) aqref_record(cudaMemcpy(f->cellEnd, s->cell_end, sizeof(int) * C, cudaMemcpyHostToDevice), "ce", __FILE__, __LINE__);
  if (s->particle_hash) aqref_record(cudaMemcpy(f->particleHashes, s->particle_hash, sizeof(int) * n, cudaMemcpyHostToDevice), "ph", __FILE__, __LINE__);
  if (s->sort_index) aqref_record(cudaMemcpy(f->particleIndices, s->sort_index, sizeof(int) * n, cudaMemcpyHostToDevice), "pi", __FILE__, __LINE__);
  if (s->position || s->velocity_p || s->fractions) {
    std::vector<Particle> ps(n);
    aqref_record(cudaMemcpy(ps.data(), f->particles, sizeof(Particle) * n, cudaMemcpyDeviceToHost), "p", __FILE__, __LINE__);
    for (int i = 0; i < n; ++i) {
      if (s->position) ps[i].position = make_float3(s->position[i], s->position[n + i], s->position[2 * n + i]);
      if (s->velocity_p) ps[i].velocity = make_float3(s->velocity_p[i], s->velocity_p[n + i], s->velocity_p[2 * n + i]);
      if (s->fractions) ps[i].volumeFractions = make_float4(s->fractions[i], s->fractions[n + i], s->fractions[2 * n + i], s->fractions[3 * n + i]);
    }
    aqref_record(cudaMemcpy(f->particles, ps.data(), sizeof(Particle) * n, cudaMemcpyHostToDevice), "p", __FILE__, __LINE__);
  }
  cudaDeviceSynchronize();
  return (int)aqref_first_error;
}

/* Ink particles, the calls the reference leaves commented out: Fluid::init
 * would run initInkRenderer after seeding (Fluid_3D_FLIP.cu:498), so it
 * continues the same rand() sequence when called right after aqref_create;
 * simulationStep would end with transferToInkParticles + moveInkParticles
 * (Fluid_3D_FLIP.cu:349-350).  Returns the ink count, or -1 on error. */
int aqref_ink_init(void* h) {
  RefFluid* r = (RefFluid*)h;
  if (!r->ink) {
    r->f->initInkRenderer();
    cudaDeviceSynchronize();
    r->ink = true;
  }
  return aqref_first_error == cudaSuccess ? r->f->inkParticleCount : -1;
}

int aqref_ink_step(void* h) {
  RefFluid* r = (RefFluid*)h;
  if (!r->ink) return -1;
  r->f->transferToInkParticles();
  r->f->moveInkParticles(r->f->timestep);
  cudaDeviceSynchronize();
  aqref_record(cudaGetLastError(), "ink", __FILE__, __LINE__);
  return (int)aqref_first_error;
}

/* Ink positions / velocities as [3][n] planes (either may be NULL). */
int aqref_ink_get(void* h, float* pos, float* vel) {
  RefFluid* r = (RefFluid*)h;
  if (!r->ink) return -1;
  const int n = r->f->inkParticleCount;
  std::vector<Fluid_3D_FLIP::Particle> ps(n);
  aqref_record(cudaMemcpy(ps.data(), r->f->inkParticles, sizeof(Fluid_3D_FLIP::Particle) * n,
                          cudaMemcpyDeviceToHost), "ink", __FILE__, __LINE__);
  for (int i = 0; i < n; ++i) {
    if (pos) { pos[i] = ps[i].position.x; pos[n + i] = ps[i].position.y; pos[2 * n + i] = ps[i].position.z; }
    if (vel) { vel[i] = ps[i].velocity.x; vel[n + i] = ps[i].velocity.y; vel[2 * n + i] = ps[i].velocity.z; }
  }
  return (int)aqref_first_error;
}

int aqref_ink_set(void* h, const float* pos, const float* vel) {
  RefFluid* r = (RefFluid*)h;
  if (!r->ink) return -1;
  const int n = r->f->inkParticleCount;
  std::vector<Fluid_3D_FLIP::Particle> ps(n);
  aqref_record(cudaMemcpy(ps.data(), r->f->inkParticles, sizeof(Fluid_3D_FLIP::Particle) * n,
                          cudaMemcpyDeviceToHost), "ink", __FILE__, __LINE__);
  for (int i = 0; i < n; ++i) {
    if (pos) ps[i].position = make_float3(pos[i], pos[n + i], pos[2 * n + i]);
    if (vel) ps[i].velocity = make_float3(vel[i], vel[n + i], vel[2 * n + i]);
  }
  aqref_record(cudaMemcpy(r->f->inkParticles, ps.data(), sizeof(Fluid_3D_FLIP::Particle) * n,
                          cudaMemcpyHostToDevice), "ink", __FILE__, __LINE__);
  return (int)aqref_first_error;
}

/* Texture address probe: createField3D (VolumeData.cuh:44-76) sets only
 * addressMode[0]; this reads a w*h*d float field filled with x+100y+10000z
 * through the reference's own readTexture at the given coordinates. */
int aqref_probe_texture(int w, int h, int d, const float* coords, float* out, int n) {
  dim3 block(8, 8, 8);
  dim3 grid(divUp(w + 1, 8), divUp(h + 1, 8), divUp(d + 1, 8));
  VolumeData v = createField3D<float>(w, h, d, grid, block, 0.f, false);
  probe_fill<<<grid, block>>>(v, w, h, d);
  float *dc = nullptr, *dout = nullptr;
  cudaMalloc(&dc, sizeof(float) * 3 * n);
  cudaMalloc(&dout, sizeof(float) * n);
  cudaMemcpy(dc, coords, sizeof(float) * 3 * n, cudaMemcpyHostToDevice);
  probe_read<<<divUp(n, 128), 128>>>(v, dc, dout, n);
  cudaMemcpy(out, dout, sizeof(float) * n, cudaMemcpyDeviceToHost);
  cudaFree(dc);
  cudaFree(dout);
  releaseField3D(v);
  cudaDeviceSynchronize();
  aqref_record(cudaGetLastError(), "probe", __FILE__, __LINE__);
  return (int)aqref_first_error;
}

}  // extern "C"
