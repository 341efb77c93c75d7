// Shared device-side definitions of the B200 FLIP step.
//
// Layout in HBM (all structure-of-arrays, z fastest):
//   cells  [0,s)^3          index (x*sy + y)*sz + z          (C entries)
//   nodes  [0,s]^3          index (x*(sy+1) + y)*(sz+1) + z  (F entries)
//   particles               sorted by cell; px,py,pz,vx,vy,vz float arrays
// Node (x,y,z) of the velocity arrays holds u on the x-face (x, y+1/2, z+1/2)h,
// v on the y-face (x+1/2, y, z+1/2)h and w on the z-face (x+1/2, y+1/2, z)h,
// the staggering of Fluid/MAC_Grid_3D.cuh:100-130 in the reference.
#pragma once

#include <cmath>
#include <cstdint>
#include <cuda_runtime.h>

namespace aqb {

constexpr int kAir = 0;    // CONTENT_AIR   (Fluid/MAC_Grid_3D.cuh:15)
constexpr int kFluid = 1;  // CONTENT_FLUID (Fluid/MAC_Grid_3D.cuh:16)
constexpr int kSolid = 2;  // CONTENT_SOLID (Fluid/MAC_Grid_3D.cuh:17)

// Activity bricks: 8x8x8 cells.  A brick is active when it holds a fluid cell.
constexpr int kBrick = 8;

struct Dims {
  int sx, sy, sz;
  int C, F;          // cells, nodes
  int nyz, nz;       // node strides: (sy+1)*(sz+1), sz+1
  float h, inv_h;    // cellPhysicalSize and its reciprocal
  int bx, by, bz;    // brick counts per axis
  int cov_x, cov_y, cov_z;  // faces each fixBoundary launch covers (see host)
};

__host__ __device__ __forceinline__ int cell_index(const Dims& d, int x, int y, int z) {
  return (x * d.sy + y) * d.sz + z;
}
__host__ __device__ __forceinline__ int node_index(const Dims& d, int x, int y, int z) {
  return x * d.nyz + y * d.nz + z;
}
__host__ __device__ __forceinline__ int brick_index(const Dims& d, int x, int y, int z) {
  return ((x / kBrick) * d.by + (y / kBrick)) * d.bz + (z / kBrick);
}

// fixBoundaryX/Y/Z (Fluid/Fluid_3D_kernels.cu:44-98) are launched with
// ceil(s1*s2/1024)*1024 threads over (s1+1)*(s2+1) faces, so only faces with
// flat index below cov_* are clamped / marked solid.
__host__ __device__ __forceinline__ bool covered_x(const Dims& d, int y, int z) {
  return y * (d.sz + 1) + z < d.cov_x;
}
__host__ __device__ __forceinline__ bool covered_y(const Dims& d, int x, int z) {
  return x * (d.sz + 1) + z < d.cov_y;
}
__host__ __device__ __forceinline__ bool covered_z(const Dims& d, int x, int y) {
  return x * (d.sy + 1) + y < d.cov_z;
}

// Particle arrays (structure of arrays).
struct Particles {
  float *px, *py, *pz;
  float *vx, *vy, *vz;
  float4* frac;  // only in multiphase mode
};

struct StepParams {
  float dt;
  float flip;       // FLIPcoeff
  float gdx, gdy, gdz;  // gravity * dt
  int gx_nz, gy_nz, gz_nz;  // gravity component != 0
  float rho[4];     // phaseDensities
  int phase;        // single-phase mode: the phase every particle carries
  int multiphase;
};

// One scene of a batch: its grid, parameters and offsets into the batch's
// concatenated arrays (particles, cells, nodes, activity bricks, residual
// partial sums).
struct SceneDesc {
  Dims d;
  StepParams sp;
  int p_off, n;  // particles
  int c_off;     // cells (and cell-table keys)
  int f_off;     // nodes
  int br_off;    // 8^3 bricks
  int rp_off;    // flat residual partials
};

// Virtual-block prefix sums per kernel family over the scenes of a batch:
// scene s owns virtual blocks [pre[s], pre[s+1]).
struct BatchIndex {
  const SceneDesc* scenes;
  int n_scenes;
  const int* particles;  // ceil(n/256)
  const int* nodes;      // ceil(sz/32) * ceil(sy/8) * sx
  const int* bricks;     // bx * by * bz
  const int* slayer;     // ceil((F - C)/256)
  const int* flat;       // ceil(sz/128) * ceil(sy/8) * sx
  const int* rows;       // packed-row Jacobi warp items (depends on x planes per item)
};

__device__ __forceinline__ int find_scene(const int* __restrict__ pre, int ns, int vb) {
  int lo = 0, hi = ns;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (__ldg(pre + mid) <= vb) lo = mid;
    else hi = mid;
  }
  return lo;
}

// Device-side record of the pressure solve; read back on demand.
// ||b - A p|| / ||b|| from the squared norms; 0 for an empty system, NaN
// when either norm is not finite (a NaN or Inf in the right-hand side).
__host__ __device__ __forceinline__ double rel_residual_of(double r2, double b2) {
  if (!isfinite(b2) || !isfinite(r2)) return (b2 - b2) + (r2 - r2);  // NaN
  return b2 > 0.0 ? sqrt(r2) / sqrt(b2) : 0.0;
}

struct SolveState {
  int iterations;       // sweeps done in the current/last solve
  int bodies;           // residual-check blocks done
  int converged;
  int nonfinite;
  double rel_residual;  // of the returned iterate; -1 if not computed
  double b2;            // ||b||^2 over fluid cells
  double r2;            // ||b - A p||^2 of the returned iterate
  int fluid_cells;
  int sync_timeout;  // the persistent solve gave up waiting at a grid barrier
  long long total_sweeps;  // cumulative over the fluid's life
  long long total_bodies;
  int warm;                // learned warm start: 1 prediction kept, 2 zero-init fallback, 0 none
  double warm_rel;         // relative residuals after the first 20 sweeps of each start
  double zero_rel;
  // Sticky: a divergence norm or residual of some step since creation (or
  // since the last state upload) was not finite.
  int nonfinite_seen;
};

}  // namespace aqb
