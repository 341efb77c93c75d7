// Pressure Jacobi sweeps on caller-owned buffers without any allocation.
//
// Some callers cannot allocate device memory while the solver runs: a host
// application that hands the solver a fixed memory pool, code running inside
// a memory-budgeted frame loop, or a plugin loaded into a process whose
// allocator it must not touch.  aq_jacobi_sweeps_noalloc serves them: the
// caller passes the cell types, the right-hand side and the pressure (in and
// out); the second Jacobi buffer and the tile-activity flags the kernels need
// live in file-scope __device__ arrays of fixed size below, so the call makes
// no cudaMalloc, no cudaFree and no allocating library call.
//
// Costs and limits: every GPU that loads this library holds these arrays
// (about 1 MiB) until the process exits; grids above kNoAllocMaxCells cells
// are rejected.  All calls on one device share the arrays and they keep the
// previous call's contents, so each call first rewrites everything it reads;
// two calls whose work overlaps on the GPU (for example on two streams) race
// on them and must be serialised by the caller.
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/aquarius_b200.h"
#include "aq_kernels.cuh"

namespace aqb {
namespace {

constexpr int kNoAllocMaxCells = AQ_NOALLOC_MAX_CELLS;
// every axis is >= 4 cells, so each 8^3 brick holds at least 4^3 cells
constexpr int kNoAllocMaxBricks = kNoAllocMaxCells / 64;

static __device__ __align__(256) float g_noalloc_pressure[kNoAllocMaxCells];
static __device__ __align__(256) uint8_t g_noalloc_bricks[kNoAllocMaxBricks];

// Device addresses of the two arrays, looked up once per device (the host
// symbols are host-side stand-ins, not device addresses).
struct SymbolAddrs {
  float* pressure = nullptr;
  uint8_t* bricks = nullptr;
  bool ready = false;
};
constexpr int kMaxDevices = 64;
SymbolAddrs g_addrs[kMaxDevices];
std::mutex g_addrs_mutex;

// Clears air pressure in the caller's buffer, copies the pressure into the
// scratch buffer (so cells the sweeps skip hold the same values in both) and
// marks the 8^3 bricks that contain fluid.
__global__ void k_noalloc_prepare(Dims d, const int8_t* __restrict__ type, float* __restrict__ p,
                                  float* __restrict__ scratch, uint8_t* __restrict__ bricks) {
  const int z = blockIdx.x * kBrick + threadIdx.x;
  const int y = blockIdx.y * kBrick + threadIdx.y;
  const int x = blockIdx.z * kBrick + threadIdx.z;
  int fl = 0;
  if (x < d.sx && y < d.sy && z < d.sz) {
    const int c = cell_index(d, x, y, z);
    fl = type[c] == kFluid;
    const float v = fl ? p[c] : 0.f;
    p[c] = v;
    scratch[c] = v;
  }
  const int any = __syncthreads_or(fl);
  if (threadIdx.x == 0 && threadIdx.y == 0 && threadIdx.z == 0)
    bricks[(blockIdx.z * d.by + blockIdx.y) * d.bz + blockIdx.x] = any ? 1 : 0;
}

__global__ void k_noalloc_copy(const float* __restrict__ a, float* __restrict__ b, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) b[i] = a[i];
}

}  // namespace
}  // namespace aqb

using namespace aqb;

extern "C" aq_status aq_jacobi_sweeps_noalloc(int32_t sx, int32_t sy, int32_t sz, const int8_t* cell_type,
                                              const float* rhs, float* pressure, int32_t sweeps, void* stream) {
  if (sx < 4 || sy < 4 || sz < 4 || !cell_type || !rhs || !pressure || sweeps < 0)
    return set_last_error(AQ_ERR_INVALID_ARGUMENT, "aq_jacobi_sweeps_noalloc: bad argument");
  const long long cells = (long long)sx * sy * sz;
  if (cells > kNoAllocMaxCells)
    return set_last_error(AQ_ERR_INVALID_ARGUMENT,
                          "aq_jacobi_sweeps_noalloc: grid of " + std::to_string(cells) +
                              " cells exceeds the fixed scratch of " + std::to_string(kNoAllocMaxCells) + " cells");
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
    return set_last_error(AQ_ERR_NO_DEVICE, "aq_jacobi_sweeps_noalloc: no usable CUDA device");
  SymbolAddrs a;
  {
    std::lock_guard<std::mutex> lock(g_addrs_mutex);
    if (!g_addrs[dev].ready) {
      // First call on this device, with it current: resolve the arrays'
      // device addresses.  This call must not happen under stream capture.
      void* pp = nullptr;
      void* pb = nullptr;
      cudaError_t e = cudaGetSymbolAddress(&pp, g_noalloc_pressure);
      if (e == cudaSuccess) e = cudaGetSymbolAddress(&pb, g_noalloc_bricks);
      if (e != cudaSuccess)
        return set_last_error(AQ_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
      g_addrs[dev].pressure = (float*)pp;
      g_addrs[dev].bricks = (uint8_t*)pb;
      g_addrs[dev].ready = true;
    }
    a = g_addrs[dev];
  }
  Dims d;
  memset(&d, 0, sizeof(d));
  d.sx = sx; d.sy = sy; d.sz = sz;
  d.C = (int)cells;
  d.F = (sx + 1) * (sy + 1) * (sz + 1);
  d.nz = sz + 1;
  d.nyz = (sy + 1) * (sz + 1);
  d.bx = (sx + kBrick - 1) / kBrick; d.by = (sy + kBrick - 1) / kBrick; d.bz = (sz + kBrick - 1) / kBrick;
  cudaStream_t st = (cudaStream_t)stream;
  k_noalloc_prepare<<<dim3(d.bz, d.by, d.bx), dim3(kBrick, kBrick, kBrick), 0, st>>>(d, cell_type, pressure,
                                                                                    a.pressure, a.bricks);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_last_error(AQ_ERR_CUDA, cudaGetErrorString(e));
  // Same sweep kernels and order as the fluid's pressure stage, without the
  // residual variant (it writes partial sums this entry point has no room for).
  const JacobiPlan plan = sz % 4 == 0 ? JacobiPlan{1, 0, 1} : JacobiPlan{1, 16, 16};
  float* bufs[2] = {pressure, a.pressure};
  for (int k = 0; k < sweeps; ++k) {
    e = launch_jacobi(st, d, plan, false, bufs[k % 2], bufs[(k + 1) % 2], rhs, cell_type, a.bricks, nullptr,
                      nullptr);
    if (e != cudaSuccess) return set_last_error(AQ_ERR_CUDA, cudaGetErrorString(e));
  }
  if (sweeps % 2 == 1) {
    k_noalloc_copy<<<(d.C + 255) / 256, 256, 0, st>>>(a.pressure, pressure, d.C);
    e = cudaGetLastError();
    if (e != cudaSuccess) return set_last_error(AQ_ERR_CUDA, cudaGetErrorString(e));
  }
  return set_last_error(AQ_OK, "");
}

extern "C" int32_t aq_jacobi_noalloc_max_cells(void) { return kNoAllocMaxCells; }
