// Host side of the surface mesher (aq_fluid_mesh* in include/aquarius_b200.h).
//
// Reference: Mesher (Rendering/Renderer3D/Mesher.cuh:94-178,
// Rendering/Renderer3D/Mesher.cu:577-630) as Fluid::init constructs it
// (Fluid/Fluid_3D_FLIP.cu:495): container = size * h, particle spacing h/2,
// a 128^3 marching-cubes grid.  Buffers are made on the first call and kept;
// the SDF lives in a cudaArray read through a linear-filtering texture with
// the reference's sampler settings.
#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/aquarius_b200.h"
#include "fluid_impl.cuh"

using namespace aqb;

#define AQM_CUDA(call)                                                                           \
  do {                                                                                           \
    cudaError_t e_ = (call);                                                                     \
    if (e_ != cudaSuccess)                                                                       \
      return fail(e_ == cudaErrorMemoryAllocation ? AQ_ERR_OUT_OF_MEMORY : AQ_ERR_CUDA,          \
                  std::string(#call) + ": " + cudaGetErrorString(e_));                           \
  } while (0)

#define AQM_TRY(expr)             \
  do {                            \
    aq_status s_ = (expr);        \
    if (s_ != AQ_OK) return s_;   \
  } while (0)

namespace aqb {

struct MeshState {
  MeshDims m{};
  int n = 0;
  cudaArray_t sdf = nullptr;
  cudaSurfaceObject_t surf = 0;
  cudaTextureObject_t tex = 0;
  int *skey = nullptr, *scount = nullptr, *soff = nullptr, *stiles = nullptr;
  float4* spos = nullptr;
  float* vv = nullptr;
  uint8_t* ctype = nullptr;
  int *mflag = nullptr, *moff = nullptr, *mtiles = nullptr;
  int *prev = nullptr, *bad = nullptr;
  float* own = nullptr;  // records for aq_fluid_download_mesh
  long long own_cap = 0;
  const float* last_out = nullptr;  // the caller's buffer of the previous call
  long long last_cap = 0;
  std::vector<void*> allocs;

  ~MeshState() {
    if (tex) cudaDestroyTextureObject(tex);
    if (surf) cudaDestroySurfaceObject(surf);
    if (sdf) cudaFreeArray(sdf);
    for (void* p : allocs) cudaFree(p);
    if (own) cudaFree(own);
  }
  template <typename T>
  aq_status alloc(T** p, size_t count) {
    void* q = nullptr;
    AQM_CUDA(cudaMalloc(&q, std::max<size_t>(count * sizeof(T), 16)));
    allocs.push_back(q);
    *p = (T*)q;
    return AQ_OK;
  }
  long long cubes() const { return (long long)m.MX * m.MY * m.MZ; }
  long long hash_cells() const { return (long long)m.HX * m.HY * m.HZ; }
};

void mesh_release(MeshState* s) { delete s; }

}  // namespace aqb

namespace {

// Mesher::Mesher (Rendering/Renderer3D/Mesher.cu:577-603), host float math.
MeshDims mesh_dims(const aq_fluid* f) {
  MeshDims m{};
  const float h = f->d.h;
  const float cx = (float)f->d.sx * h, cy = (float)f->d.sy * h, cz = (float)f->d.sz * h;
  const float spacing = h / 2;
  m.hs = spacing;
  m.radius = spacing;
  m.MX = m.MY = m.MZ = 128;
  m.hm = cx / (float)(m.MX - 2);
  m.SX = (int)(3 + cx / m.hs);
  m.SY = (int)(3 + cy / m.hs);
  m.SZ = (int)(3 + cz / m.hs);
  m.HX = m.SX - 2;
  m.HY = m.SY - 2;
  m.HZ = m.SZ - 2;
  return m;
}

aq_status ensure_state(aq_fluid* f) {
  if (f->mesher) return AQ_OK;
  MeshState* s = new MeshState();
  s->m = mesh_dims(f);
  s->n = f->n;
  const MeshDims& m = s->m;
  if ((long long)m.SX * m.SY * m.SZ >= (1ll << 31)) {
    delete s;
    return fail(AQ_ERR_INVALID_CONFIG, "grid too large for the mesher's SDF");
  }
  auto bail = [&](aq_status st) { delete s; return st; };
  const size_t HC = (size_t)s->hash_cells(), NC = (size_t)s->cubes();
  const size_t NV = (size_t)(m.MX + 1) * (m.MY + 1) * (m.MZ + 1);
  aq_status st = AQ_OK;
  if ((st = s->alloc(&s->skey, (size_t)s->n)) != AQ_OK) return bail(st);
  if ((st = s->alloc(&s->scount, HC + 1)) != AQ_OK) return bail(st);
  if ((st = s->alloc(&s->soff, HC + 1)) != AQ_OK) return bail(st);
  if ((st = s->alloc(&s->stiles, cell_scan_tiles((int)HC))) != AQ_OK) return bail(st);
  if ((st = s->alloc(&s->spos, (size_t)s->n)) != AQ_OK) return bail(st);
  if ((st = s->alloc(&s->vv, NV)) != AQ_OK) return bail(st);
  if ((st = s->alloc(&s->ctype, NC)) != AQ_OK) return bail(st);
  if ((st = s->alloc(&s->mflag, NC + 1)) != AQ_OK) return bail(st);
  if ((st = s->alloc(&s->moff, NC + 1)) != AQ_OK) return bail(st);
  if ((st = s->alloc(&s->mtiles, cell_scan_tiles((int)NC))) != AQ_OK) return bail(st);
  if ((st = s->alloc(&s->prev, 1)) != AQ_OK) return bail(st);
  if ((st = s->alloc(&s->bad, 1)) != AQ_OK) return bail(st);
  cudaError_t e = cudaMemsetAsync(s->scount, 0, sizeof(int) * (HC + 1), f->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(s->mflag, 0, sizeof(int) * (NC + 1), f->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(s->prev, 0, sizeof(int), f->stream);
  // createField3D<float>(..., filter = true, cudaAddressModeBorder)
  // (Rendering/Renderer3D/Mesher.cu:627, Fluid/VolumeData.cuh:44-76).  The
  // reference leaves addressMode[1,2] at 0, which with unnormalised
  // coordinates the texture unit applies as clamp; it is set so here.
  cudaChannelFormatDesc ch = cudaCreateChannelDesc<float>();
  if (e == cudaSuccess)
    e = cudaMalloc3DArray(&s->sdf, &ch, make_cudaExtent(m.SX, m.SY, m.SZ), cudaArraySurfaceLoadStore);
  if (e == cudaSuccess) {
    cudaResourceDesc rd;
    memset(&rd, 0, sizeof(rd));
    rd.resType = cudaResourceTypeArray;
    rd.res.array.array = s->sdf;
    cudaTextureDesc td;
    memset(&td, 0, sizeof(td));
    td.addressMode[0] = cudaAddressModeBorder;
    td.addressMode[1] = cudaAddressModeClamp;
    td.addressMode[2] = cudaAddressModeClamp;
    td.filterMode = cudaFilterModeLinear;
    td.readMode = cudaReadModeElementType;
    td.normalizedCoords = 0;
    e = cudaCreateTextureObject(&s->tex, &rd, &td, nullptr);
    if (e == cudaSuccess) e = cudaCreateSurfaceObject(&s->surf, &rd);
  }
  if (e != cudaSuccess) {
    delete s;
    return fail(e == cudaErrorMemoryAllocation ? AQ_ERR_OUT_OF_MEMORY : AQ_ERR_CUDA,
                std::string("mesher buffers: ") + cudaGetErrorString(e));
  }
  f->mesher = s;
  return AQ_OK;
}

// SDF (keys, stable placement, computeSDF) and the cube classification and
// scan; the occupied-cube count ends in moff[NC].
aq_status mesh_front(aq_fluid* f) {
  MeshState* s = f->mesher;
  const MeshDims& m = s->m;
  cudaStream_t st = f->stream;
  AQM_CUDA(cudaMemsetAsync(s->bad, 0, sizeof(int), st));
  AQM_CUDA(launch_sdf_keys(st, m, f->cur.px, f->cur.py, f->cur.pz, s->skey, s->scount, f->n));
  AQM_CUDA(launch_cell_scan(st, (int)s->hash_cells(), s->scount, s->soff, s->stiles));
  AQM_CUDA(launch_sdf_scatter(st, m, f->d, f->cur.px, f->cur.py, f->cur.pz, f->off, s->skey, s->soff, s->spos, s->bad,
                              f->n));
  AQM_CUDA(launch_sdf(st, m, s->soff, s->spos, s->surf));
  AQM_CUDA(launch_mc_vertices(st, m, s->tex, s->vv));
  AQM_CUDA(launch_mc_flags(st, m, s->vv, s->ctype, s->mflag));
  AQM_CUDA(launch_cell_scan(st, (int)s->cubes(), s->mflag, s->moff, s->mtiles));
  return AQ_OK;
}

aq_status mesh_finish(aq_fluid* f, int32_t* cubes) {
  MeshState* s = f->mesher;
  int h[2] = {0, 0};
  AQM_CUDA(cudaMemcpyAsync(&h[0], s->bad, sizeof(int), cudaMemcpyDeviceToHost, f->stream));
  AQM_CUDA(cudaMemcpyAsync(&h[1], s->moff + s->cubes(), sizeof(int), cudaMemcpyDeviceToHost, f->stream));
  AQM_CUDA(cudaStreamSynchronize(f->stream));
  if (h[0]) return fail(AQ_ERR_INVALID_ARGUMENT, "particles are not sorted by cell (run a step or the sort stage)");
  if (cubes) *cubes = h[1];
  return AQ_OK;
}

}  // namespace

extern "C" {

aq_status aq_fluid_mesh_info(const aq_fluid* f, aq_mesh_info* info) {
  if (!f || !info) return fail(AQ_ERR_INVALID_ARGUMENT, "bad argument");
  const MeshDims m = mesh_dims(f);
  info->sdf_size[0] = m.SX; info->sdf_size[1] = m.SY; info->sdf_size[2] = m.SZ;
  info->mesh_size[0] = m.MX; info->mesh_size[1] = m.MY; info->mesh_size[2] = m.MZ;
  info->sdf_cell = m.hs;
  info->mesh_cell = m.hm;
  info->particle_radius = m.radius;
  return AQ_OK;
}

aq_status aq_fluid_mesh(aq_fluid* f, float* output, int64_t capacity_records, int32_t* cubes) {
  if (!f || !output || capacity_records < 0) return fail(AQ_ERR_INVALID_ARGUMENT, "bad argument");
  cudaSetDevice(f->device);
  AQM_TRY(ensure_state(f));
  MeshState* s = f->mesher;
  cudaStream_t st = f->stream;
  if (output != s->last_out || capacity_records != s->last_cap) {
    // a buffer seen for the first time is cleared whole, as the reference's
    // memset does every call; later calls clear only what shrank
    AQM_CUDA(cudaMemsetAsync(output, 0, sizeof(float) * 90 * (size_t)capacity_records, st));
    AQM_CUDA(cudaMemsetAsync(s->prev, 0, sizeof(int), st));
    s->last_out = output;
    s->last_cap = capacity_records;
  }
  AQM_TRY(mesh_front(f));
  AQM_CUDA(launch_mc_emit(st, s->m, s->tex, s->vv, s->ctype, s->moff, output, capacity_records));
  AQM_CUDA(launch_mc_tail(st, s->moff + s->cubes(), s->prev, output, capacity_records));
  return mesh_finish(f, cubes);
}

aq_status aq_fluid_download_mesh(aq_fluid* f, float* records, int64_t capacity_records, int32_t* cubes) {
  if (!f || capacity_records < 0 || (capacity_records > 0 && !records))
    return fail(AQ_ERR_INVALID_ARGUMENT, "bad argument");
  cudaSetDevice(f->device);
  AQM_TRY(ensure_state(f));
  MeshState* s = f->mesher;
  cudaStream_t st = f->stream;
  AQM_TRY(mesh_front(f));
  int32_t total = 0;
  AQM_TRY(mesh_finish(f, &total));
  const long long want = std::min<long long>(total, capacity_records);
  if (want > s->own_cap) {
    if (s->own) cudaFree(s->own);
    s->own = nullptr;
    s->own_cap = 0;
    AQM_CUDA(cudaMalloc(&s->own, sizeof(float) * 90 * (size_t)want));
    s->own_cap = want;
  }
  if (want > 0) {
    AQM_CUDA(launch_mc_emit(st, s->m, s->tex, s->vv, s->ctype, s->moff, s->own, want));
    AQM_CUDA(cudaMemcpyAsync(records, s->own, sizeof(float) * 90 * (size_t)want, cudaMemcpyDeviceToHost, st));
    AQM_CUDA(cudaStreamSynchronize(st));
  }
  if (cubes) *cubes = total;
  return AQ_OK;
}

aq_status aq_fluid_download_sdf(aq_fluid* f, float* sdf) {
  if (!f || !sdf) return fail(AQ_ERR_INVALID_ARGUMENT, "bad argument");
  if (!f->mesher) return fail(AQ_ERR_INVALID_ARGUMENT, "no mesh has been made yet");
  cudaSetDevice(f->device);
  MeshState* s = f->mesher;
  const MeshDims& m = s->m;
  std::vector<float> xf((size_t)m.SX * m.SY * m.SZ);
  cudaMemcpy3DParms p;
  memset(&p, 0, sizeof(p));
  p.srcArray = s->sdf;
  p.dstPtr = make_cudaPitchedPtr(xf.data(), sizeof(float) * m.SX, m.SX, m.SY);
  p.extent = make_cudaExtent(m.SX, m.SY, m.SZ);
  p.kind = cudaMemcpyDeviceToHost;
  AQM_CUDA(cudaStreamSynchronize(f->stream));
  AQM_CUDA(cudaMemcpy3D(&p));
  for (int x = 0; x < m.SX; ++x)
    for (int y = 0; y < m.SY; ++y)
      for (int z = 0; z < m.SZ; ++z)
        sdf[((size_t)x * m.SY + y) * m.SZ + z] = xf[((size_t)z * m.SY + y) * m.SX + x];
  return AQ_OK;
}

}  // extern "C"
