/*
 * Headless harness around the reference's own surface mesher — TEST
 * INFRASTRUCTURE ONLY.  Built by oracle/Makefile (target `mesh`) into
 * oracle/_ref/libaqmesh.so from the reference sources where they lie: the
 * real Rendering/Renderer3D/Mesher.cuh / Mesher.cu (the FLIP harness keeps
 * its stub, because Fluid::init would otherwise re-sort the particles by
 * the mesher's grid, Fluid/Fluid_3D_FLIP.cu:502).
 *
 * It constructs Mesher exactly as Fluid::init does
 * (Fluid/Fluid_3D_FLIP.cu:481-482, :495: container = size * h, particle
 * spacing h/2) and runs Mesher::mesh on particles given from the host,
 * returning the output buffer's occupied records, the SDF grid and the
 * order mesh() leaves the particles in.  It also probes the texture
 * filtering createField3D(..., filter = true, cudaAddressModeBorder) sets up
 * (Fluid/VolumeData.cuh:44-76), which marching cubes samples through.
 */
#include <cstdlib>
#include <cstring>
#include <vector>

#include "Fluid/Fluid_3D_common.cu"
#include "Fluid/Fluid_3D_kernels.cu"
#include "Fluid/MAC_Grid_3D.cu"
#include "Fluid/Fluid_3D_FLIP.cuh"
#include "Rendering/Renderer3D/Mesher.cu"

cudaError_t aqref_first_error = cudaSuccess;

namespace {

using Fluid_3D_FLIP::Particle;

struct MeshRun {
  Mesher* m = nullptr;
  int n = 0;
  Particle* particles = nullptr;
  Particle* copy = nullptr;
  int* hashes = nullptr;
  int* indices = nullptr;
  float* output = nullptr;
  size_t output_floats = 0;
};

__global__ void probe_fill_values(VolumeData v, const float* vals, int w, int h, int d) {
  int x = blockIdx.x * blockDim.x + threadIdx.x;
  int y = blockIdx.y * blockDim.y + threadIdx.y;
  int z = blockIdx.z * blockDim.z + threadIdx.z;
  if (x >= w || y >= h || z >= d) return;
  v.writeSurface<float>(vals[((size_t)z * h + y) * w + x], x, y, z);
}

__global__ void probe_read_values(VolumeData v, const float* coords, float* out, int n) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  out[i] = v.readTexture<float>(coords[3 * i], coords[3 * i + 1], coords[3 * i + 2]);
}

}  // namespace

extern "C" {

/* Mesher(make_float3(sx, sy, sz) * h, h / 2, n, ...) as Fluid::init builds it. */
void* aqmesh_create(int sx, int sy, int sz, float h, int n) {
  aqref_first_error = cudaSuccess;
  MeshRun* r = new MeshRun();
  r->n = n;
  const int threads = min(512, n);
  const int blocks = divUp(n, threads);
  r->m = new Mesher(make_float3(sx, sy, sz) * h, h / 2, n, blocks, threads);
  cudaMalloc(&r->particles, sizeof(Particle) * n);
  cudaMalloc(&r->copy, sizeof(Particle) * n);
  cudaMalloc(&r->hashes, sizeof(int) * n);
  cudaMalloc(&r->indices, sizeof(int) * n);
  r->output_floats = (size_t)r->m->triangleCount * 3 * 6;
  cudaMalloc(&r->output, sizeof(float) * r->output_floats);
  cudaDeviceSynchronize();
  aqref_record(cudaGetLastError(), "mesh create", __FILE__, __LINE__);
  if (aqref_first_error != cudaSuccess) return nullptr;
  return r;
}

void aqmesh_destroy(void* h) {
  MeshRun* r = (MeshRun*)h;
  if (!r) return;
  cudaFree(r->particles);
  cudaFree(r->copy);
  cudaFree(r->hashes);
  cudaFree(r->indices);
  cudaFree(r->output);
  delete r->m;
  delete r;
}

/* SDF grid extent, mesh grid extent, SDF and mesh cell sizes. */
void aqmesh_sizes(void* h, int* sdf, int* mesh, float* cell) {
  Mesher* m = ((MeshRun*)h)->m;
  sdf[0] = m->sizeX_SDF; sdf[1] = m->sizeY_SDF; sdf[2] = m->sizeZ_SDF;
  mesh[0] = m->sizeX_mesh; mesh[1] = m->sizeY_mesh; mesh[2] = m->sizeZ_mesh;
  cell[0] = m->cellPhysicalSize_SDF; cell[1] = m->cellPhysicalSize_mesh;
}

/* Loads particles (positions [3][n]; velocity 0, phase 0), runs mesh(), and
 * copies back: the occupied-cube count, up to `capacity` floats of the output
 * buffer, the SDF grid (x fastest, may be NULL), the particles' positions
 * in the order mesh() left them ([3][n], may be NULL) and the time mesh()
 * took between CUDA events on either side of it (may be NULL). */
int aqmesh_run(void* h, const float* pos, float* out, long long capacity, int* cubes, float* sdf,
               float* pos_after, float* ms) {
  MeshRun* r = (MeshRun*)h;
  const int n = r->n;
  std::vector<Particle> ps(n);
  for (int i = 0; i < n; ++i) ps[i] = Particle(make_float3(pos[i], pos[n + i], pos[2 * n + i]), 0);
  aqref_record(cudaMemcpy(r->particles, ps.data(), sizeof(Particle) * n, cudaMemcpyHostToDevice), "p", __FILE__,
               __LINE__);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaDeviceSynchronize();
  cudaEventRecord(e0);
  r->m->mesh(r->particles, r->copy, r->hashes, r->indices, r->output);
  cudaEventRecord(e1);
  cudaEventSynchronize(e1);
  if (ms) cudaEventElapsedTime(ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaDeviceSynchronize();
  unsigned int count = 0;
  aqref_record(cudaMemcpy(&count, r->m->occupiedCellIndex, sizeof(count), cudaMemcpyDeviceToHost), "count",
               __FILE__, __LINE__);
  *cubes = (int)count;
  size_t want = (size_t)count * 90;
  if ((long long)want > capacity) want = (size_t)capacity;
  if (want > r->output_floats) want = r->output_floats;
  if (out && want)
    aqref_record(cudaMemcpy(out, r->output, sizeof(float) * want, cudaMemcpyDeviceToHost), "out", __FILE__,
                 __LINE__);
  Mesher* m = r->m;
  if (sdf) {
    cudaMemcpy3DParms p = {0};
    p.srcArray = m->SDF.array;
    p.dstPtr = make_cudaPitchedPtr(sdf, sizeof(float) * m->sizeX_SDF, m->sizeX_SDF, m->sizeY_SDF);
    p.extent = make_cudaExtent(m->sizeX_SDF, m->sizeY_SDF, m->sizeZ_SDF);
    p.kind = cudaMemcpyDeviceToHost;
    aqref_record(cudaMemcpy3D(&p), "sdf", __FILE__, __LINE__);
  }
  if (pos_after) {
    aqref_record(cudaMemcpy(ps.data(), r->particles, sizeof(Particle) * n, cudaMemcpyDeviceToHost), "p2",
                 __FILE__, __LINE__);
    for (int i = 0; i < n; ++i) {
      pos_after[i] = ps[i].position.x;
      pos_after[n + i] = ps[i].position.y;
      pos_after[2 * n + i] = ps[i].position.z;
    }
  }
  cudaDeviceSynchronize();
  aqref_record(cudaGetLastError(), "mesh", __FILE__, __LINE__);
  return (int)aqref_first_error;
}

/* Texture filtering probe: a w*h*d float field (x fastest) in
 * createField3D<float>(..., filter = true, cudaAddressModeBorder), the SDF's
 * settings (Rendering/Renderer3D/Mesher.cu:627), read through readTexture at
 * the given coordinates. */
int aqmesh_probe_linear(int w, int h, int d, const float* values, const float* coords, float* out, int n) {
  dim3 block(8, 8, 8);
  dim3 grid(divUp(w, 8), divUp(h, 8), divUp(d, 8));
  VolumeData v = createField3D<float>(w, h, d, grid, block, 0.f, true, cudaAddressModeBorder);
  float *dv = nullptr, *dc = nullptr, *dout = nullptr;
  cudaMalloc(&dv, sizeof(float) * w * h * d);
  cudaMalloc(&dc, sizeof(float) * 3 * n);
  cudaMalloc(&dout, sizeof(float) * n);
  cudaMemcpy(dv, values, sizeof(float) * w * h * d, cudaMemcpyHostToDevice);
  cudaMemcpy(dc, coords, sizeof(float) * 3 * n, cudaMemcpyHostToDevice);
  probe_fill_values<<<grid, block>>>(v, dv, w, h, d);
  probe_read_values<<<divUp(n, 128), 128>>>(v, dc, dout, n);
  cudaMemcpy(out, dout, sizeof(float) * n, cudaMemcpyDeviceToHost);
  cudaFree(dv);
  cudaFree(dc);
  cudaFree(dout);
  releaseField3D(v);
  cudaDeviceSynchronize();
  aqref_record(cudaGetLastError(), "probe", __FILE__, __LINE__);
  return (int)aqref_first_error;
}

int aqmesh_error(void) { return (int)aqref_first_error; }

}  // extern "C"
