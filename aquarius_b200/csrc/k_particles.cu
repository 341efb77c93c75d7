// Particle kernels: grid-to-particle transfer + RK3 advection, and the
// deterministic counting sort by cell (stages (d) and (a)).
//
// Reference: transferToParticlesImpl / moveParticlesImpl
// (Fluid/Fluid_3D_FLIP.cu:189-285), performSpatialHashing2
// (Fluid/Fluid_3D_common.cuh:27-56), calcHashImpl (Fluid/Fluid_3D_kernels.cuh:8-27),
// findCellStartEndImpl (Fluid/Fluid_kernels.cuh:3-22).
//
// The reference sorts (hash, index) pairs with thrust::sort_by_key, which is
// stable, so particles end up ordered by (cell, previous index).  Here:
//   1. advance kernel: new state into temp arrays in the current order; key =
//      cell; slot = warp-aggregated atomicAdd on the cell's count;
//   2. scan of the counts -> cell offsets (CSR), counts cleared for next step;
//   3. scatter: perm_u[off[key]+slot] = i (order inside a cell is arbitrary);
//   4. rank-gather: rank = #{j in the cell's perm_u segment : j < i}, which is
//      the stable position, and the particle is copied to off[key]+rank.
// The result is bit-identical to a stable sort regardless of atomic order.
#include "aq_kernels.cuh"

namespace aqb {
namespace {

__device__ __forceinline__ float lerpf(float a, float b, float t) { return a + t * (b - a); }

// MAC_Grid_3D::getInterpolatedValueAtPoint (Fluid/MAC_Grid_3D.cuh:66-97):
// clamp to [0, s-1], 8-tap trilinear, lerp along z, then y, then x.
__device__ __forceinline__ float sample_node(const float* __restrict__ f, const Dims& d, float x, float y,
                                             float z) {
  x = fmaxf(fminf(x, (float)d.sx - 1.f), 0.f);
  y = fmaxf(fminf(y, (float)d.sy - 1.f), 0.f);
  z = fmaxf(fminf(z, (float)d.sz - 1.f), 0.f);
  const int i = (int)floorf(x), j = (int)floorf(y), k = (int)floorf(z);
  const float tx = x - (float)i, ty = y - (float)j, tz = z - (float)k;
  const float* b = f + node_index(d, i, j, k);
  const float* c = b + d.nyz;
  const float a000 = __ldg(b), a001 = __ldg(b + 1), a010 = __ldg(b + d.nz), a011 = __ldg(b + d.nz + 1);
  const float a100 = __ldg(c), a101 = __ldg(c + 1), a110 = __ldg(c + d.nz), a111 = __ldg(c + d.nz + 1);
  const float x0y0 = lerpf(a000, a001, tz), x0y1 = lerpf(a010, a011, tz);
  const float x1y0 = lerpf(a100, a101, tz), x1y1 = lerpf(a110, a111, tz);
  return lerpf(lerpf(x0y0, x0y1, ty), lerpf(x1y0, x1y1, ty), tx);
}

// getPointVelocity / getPointNewVelocity (Fluid/MAC_Grid_3D.cuh:100-130).
__device__ __forceinline__ float3 sample_velocity(const float* __restrict__ u, const float* __restrict__ v,
                                                  const float* __restrict__ w, const Dims& d, float px,
                                                  float py, float pz) {
  const float x = __fdiv_rn(px, d.h), y = __fdiv_rn(py, d.h), z = __fdiv_rn(pz, d.h);
  return make_float3(sample_node(u, d, x, y - 0.5f, z - 0.5f), sample_node(v, d, x - 0.5f, y, z - 0.5f),
                     sample_node(w, d, x - 0.5f, y - 0.5f, z));
}

// transferToParticlesImpl's velocity update with FLIP coefficient c
// (Fluid/Fluid_3D_FLIP.cu:189-227), then moveParticlesImpl
// (Fluid/Fluid_3D_FLIP.cu:229-285): Ralston RK3 (2/9, 3/9, 4/9) in
// newVelocity, clamped to [h/4, s*h - h/4] with the velocity component
// reflected.  Shared by the fluid particles and the ink particles.
__device__ __forceinline__ void g2p_move(const Dims& d, float c, float dt, const float* __restrict__ u0,
                                         const float* __restrict__ v0, const float* __restrict__ w0,
                                         const float* __restrict__ un, const float* __restrict__ vn,
                                         const float* __restrict__ wn, float& px, float& py, float& pz, float& vx,
                                         float& vy, float& vz) {
  const float3 nv = sample_velocity(un, vn, wn, d, px, py, pz);
  const float3 ov = sample_velocity(u0, v0, w0, d, px, py, pz);
  const float oc = 1.0f - c;
  vx = c * (vx + (nv.x - ov.x)) + oc * nv.x;
  vy = c * (vy + (nv.y - ov.y)) + oc * nv.y;
  vz = c * (vz + (nv.z - ov.z)) + oc * nv.z;
  const float3 u1 = sample_velocity(un, vn, wn, d, px, py, pz);
  const float3 u2 = sample_velocity(un, vn, wn, d, px + dt * u1.x / 2, py + dt * u1.y / 2, pz + dt * u1.z / 2);
  const float3 u3 = sample_velocity(un, vn, wn, d, px + dt * u2.x * 3 / 4, py + dt * u2.y * 3 / 4,
                                    pz + dt * u2.z * 3 / 4);
  float qx = px + dt * (u1.x * 2 / 9 + u2.x * 3 / 9 + u3.x * 4 / 9);
  float qy = py + dt * (u1.y * 2 / 9 + u2.y * 3 / 9 + u3.y * 4 / 9);
  float qz = pz + dt * (u1.z * 2 / 9 + u2.z * 3 / 9 + u3.z * 4 / 9);
  const float md = d.h / 4;
  const float gx = (float)d.sx * d.h, gy = (float)d.sy * d.h, gz = (float)d.sz * d.h;
  if (qx < md) { qx = md; vx *= -1.f; }
  if (qx > gx - md) { qx = gx - md; vx *= -1.f; }
  if (qy < md) { qy = md; vy *= -1.f; }
  if (qy > gy - md) { qy = gy - md; vy *= -1.f; }
  if (qz < md) { qz = md; vz *= -1.f; }
  if (qz > gz - md) { qz = gz - md; vz *= -1.f; }
  px = qx; py = qy; pz = qz;
}

// Body shared by the single-scene kernel and the batched one.  Particle
// arrays, grids and key/slot are the scene's own (pointers already offset);
// keys are cell indices plus key_base (the scene's first cell in a batch).
template <bool MOVE, bool MULTI>
__device__ __forceinline__ void particles_advance_body(
    const Dims& d, const StepParams& sp, const Particles& cur, const Particles& tmp, const float* __restrict__ u0,
    const float* __restrict__ v0, const float* __restrict__ w0, const float* __restrict__ un,
    const float* __restrict__ vn, const float* __restrict__ wn, const float4* __restrict__ nvf,
    int* __restrict__ key, int* __restrict__ slot, int* __restrict__ count, int n, int key_base, int block) {
  const int i = block * blockDim.x + threadIdx.x;
  const bool valid = i < n;
  int k = -1;
  if (valid) {
    float px = cur.px[i], py = cur.py[i], pz = cur.pz[i];
    float vx = cur.vx[i], vy = cur.vy[i], vz = cur.vz[i];
    float4 fr = make_float4(0.f, 0.f, 0.f, 0.f);
    if (MOVE) {
      if (MULTI) {
        // transferToParticlesImpl: fractions from the cell of the unmoved particle
        int cx = (int)floorf(__fdiv_rn(px, d.h)), cy = (int)floorf(__fdiv_rn(py, d.h)),
            cz = (int)floorf(__fdiv_rn(pz, d.h));
        cx = min(max(cx, 0), d.sx - 1);
        cy = min(max(cy, 0), d.sy - 1);
        cz = min(max(cz, 0), d.sz - 1);
        fr = nvf[cell_index(d, cx, cy, cz)];
        const float s = fr.x * 1.f + fr.y * 1.f + fr.z * 1.f + fr.w * 1.f;
        if (s > 0) {
          fr.x = __fdiv_rn(fr.x, s); fr.y = __fdiv_rn(fr.y, s);
          fr.z = __fdiv_rn(fr.z, s); fr.w = __fdiv_rn(fr.w, s);
        }
      }
      g2p_move(d, sp.flip, sp.dt, u0, v0, w0, un, vn, wn, px, py, pz, vx, vy, vz);
    } else if (MULTI) {
      fr = cur.frac[i];
    }
    tmp.px[i] = px; tmp.py[i] = py; tmp.pz[i] = pz;
    tmp.vx[i] = vx; tmp.vy[i] = vy; tmp.vz[i] = vz;
    if (MULTI) tmp.frac[i] = fr;
    // calcHashImpl: truncation of position / h
    int hx = (int)__fdiv_rn(px, d.h), hy = (int)__fdiv_rn(py, d.h), hz = (int)__fdiv_rn(pz, d.h);
    hx = min(max(hx, 0), d.sx - 1);
    hy = min(max(hy, 0), d.sy - 1);
    hz = min(max(hz, 0), d.sz - 1);
    k = key_base + cell_index(d, hx, hy, hz);
    key[i] = k;
  }
  // Warp-aggregated slot allocation: one atomic per distinct cell per warp.
  const unsigned peers = __match_any_sync(0xffffffffu, k);
  if (valid) {
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(peers) - 1;
    int base = 0;
    if (lane == leader) base = atomicAdd(count + k, __popc(peers));
    base = __shfl_sync(peers, base, leader);
    slot[i] = base + __popc(peers & ((1u << lane) - 1u));
  }
}

template <bool MOVE, bool MULTI>
__global__ void __launch_bounds__(256) k_particles_advance(
    Dims d, StepParams sp, Particles cur, Particles tmp, const float* __restrict__ u0,
    const float* __restrict__ v0, const float* __restrict__ w0, const float* __restrict__ un,
    const float* __restrict__ vn, const float* __restrict__ wn, const float4* __restrict__ nvf,
    int* __restrict__ key, int* __restrict__ slot, int* __restrict__ count, int n) {
  particles_advance_body<MOVE, MULTI>(d, sp, cur, tmp, u0, v0, w0, un, vn, wn, nvf, key, slot, count, n, 0,
                                      blockIdx.x);
}

// Ink particles (Fluid/Fluid_3D_FLIP.cu:711-725): transferToParticlesImpl
// with FLIP coefficient 1 and moveParticlesImpl, in place; ink is never
// sorted or transferred to the grid.
__global__ void __launch_bounds__(256) k_ink_advance(Dims d, float dt, Particles ink, const float* __restrict__ u0,
                                                    const float* __restrict__ v0, const float* __restrict__ w0,
                                                    const float* __restrict__ un, const float* __restrict__ vn,
                                                    const float* __restrict__ wn, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float px = ink.px[i], py = ink.py[i], pz = ink.pz[i];
  float vx = ink.vx[i], vy = ink.vy[i], vz = ink.vz[i];
  g2p_move(d, 1.f, dt, u0, v0, w0, un, vn, wn, px, py, pz, vx, vy, vz);
  ink.px[i] = px; ink.py[i] = py; ink.pz[i] = pz;
  ink.vx[i] = vx; ink.vy[i] = vy; ink.vz[i] = vz;
}

__device__ __forceinline__ Particles offset_particles(const Particles& p, int off) {
  Particles q = p;
  q.px += off; q.py += off; q.pz += off;
  q.vx += off; q.vy += off; q.vz += off;
  if (q.frac) q.frac += off;
  return q;
}

// All scenes of a batch: grid-stride loop over virtual blocks, each block
// belongs to one scene.
template <bool MOVE>
__global__ void __launch_bounds__(256) kb_particles_advance(BatchIndex bi, int total, Particles cur, Particles tmp,
                                                           const float* __restrict__ u0, const float* __restrict__ v0,
                                                           const float* __restrict__ w0, const float* __restrict__ un,
                                                           const float* __restrict__ vn, const float* __restrict__ wn,
                                                           int* __restrict__ key, int* __restrict__ slot,
                                                           int* __restrict__ count) {
  for (int vb = blockIdx.x; vb < total; vb += gridDim.x) {
    const int s = find_scene(bi.particles, bi.n_scenes, vb);
    const SceneDesc S = bi.scenes[s];
    particles_advance_body<MOVE, false>(S.d, S.sp, offset_particles(cur, S.p_off), offset_particles(tmp, S.p_off),
                                        u0 + S.f_off, v0 + S.f_off, w0 + S.f_off, un + S.f_off, vn + S.f_off,
                                        wn + S.f_off, nullptr, key + S.p_off, slot + S.p_off, count, S.n, S.c_off,
                                        vb - bi.particles[s]);
  }
}

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

__device__ __forceinline__ int block_exclusive_scan(int v, int* total) {
  __shared__ int warp_sums[kScanThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int incl = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane == 31) warp_sums[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    int ws = lane < kScanThreads / 32 ? warp_sums[lane] : 0;
    int wi = ws;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, wi, o);
      if (lane >= o) wi += t;
    }
    if (lane < kScanThreads / 32) warp_sums[lane] = wi - ws;
    if (lane == kScanThreads / 32 - 1) *total = wi;
  }
  __syncthreads();
  return warp_sums[warp] + incl - v;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_reduce(const int* __restrict__ count, int n1,
                                                             int* __restrict__ tile_sums) {
  const int base = blockIdx.x * kScanTile;
  int s = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    const int idx = base + k * kScanThreads + threadIdx.x;
    if (idx < n1) s += count[idx];
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  __shared__ int ws[kScanThreads / 32];
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    int t = 0;
    for (int w = 0; w < kScanThreads / 32; ++w) t += ws[w];
    tile_sums[blockIdx.x] = t;
  }
}

// Exclusive scan of the tile sums in place, one CTA.
__global__ void __launch_bounds__(1024) k_scan_top(int* __restrict__ tile_sums, int ntiles) {
  __shared__ int part[1024];
  const int per = (ntiles + 1023) / 1024;
  const int b = threadIdx.x * per;
  int s = 0;
  for (int k = 0; k < per; ++k)
    if (b + k < ntiles) s += tile_sums[b + k];
  part[threadIdx.x] = s;
  __syncthreads();
  // Hillis-Steele inclusive scan over 1024 partial sums.
  for (int o = 1; o < 1024; o <<= 1) {
    const int t = threadIdx.x >= o ? part[threadIdx.x - o] : 0;
    __syncthreads();
    part[threadIdx.x] += t;
    __syncthreads();
  }
  int run = part[threadIdx.x] - s;
  for (int k = 0; k < per; ++k) {
    if (b + k < ntiles) {
      const int c = tile_sums[b + k];
      tile_sums[b + k] = run;
      run += c;
    }
  }
}

__global__ void __launch_bounds__(kScanThreads) k_scan_apply(int* __restrict__ count, int n1,
                                                            const int* __restrict__ tile_sums,
                                                            int* __restrict__ off) {
  const int base = blockIdx.x * kScanTile + threadIdx.x * kScanItems;
  int v[kScanItems];
  int s = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    const int idx = base + k;
    v[k] = idx < n1 ? count[idx] : 0;
    s += v[k];
  }
  int total;
  int run = block_exclusive_scan(s, &total) + tile_sums[blockIdx.x];
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    const int idx = base + k;
    if (idx < n1) {
      off[idx] = run;
      count[idx] = 0;
    }
    run += v[k];
  }
}

__global__ void __launch_bounds__(256) k_scatter(const int* __restrict__ key, const int* __restrict__ slot,
                                                const int* __restrict__ off, int* __restrict__ perm_u, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  perm_u[off[key[i]] + slot[i]] = i;
}

template <bool MULTI>
__global__ void __launch_bounds__(256) k_rank_gather(const int* __restrict__ key, const int* __restrict__ off,
                                                    const int* __restrict__ perm_u, Particles tmp,
                                                    Particles cur, int* __restrict__ sort_index, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int k = key[i];
  const int b = __ldg(off + k), e = __ldg(off + k + 1);
  int r = 0;
  for (int j = b; j < e; ++j) r += __ldg(perm_u + j) < i;
  const int dst = b + r;
  cur.px[dst] = tmp.px[i]; cur.py[dst] = tmp.py[i]; cur.pz[dst] = tmp.pz[i];
  cur.vx[dst] = tmp.vx[i]; cur.vy[dst] = tmp.vy[i]; cur.vz[dst] = tmp.vz[i];
  if (MULTI) cur.frac[dst] = tmp.frac[i];
  sort_index[dst] = i;
}

inline int blocks_for(int n, int t) { return (n + t - 1) / t; }

// Per-block FP64 sums of the particles' volume fractions (4 phases).
__global__ void __launch_bounds__(256) k_frac_sum(const float4* __restrict__ frac, int n, double* __restrict__ part) {
  __shared__ double sm[4][256];
  double a[4] = {0.0, 0.0, 0.0, 0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float4 f = frac[i];
    a[0] += f.x; a[1] += f.y; a[2] += f.z; a[3] += f.w;
  }
  for (int k = 0; k < 4; ++k) sm[k][threadIdx.x] = a[k];
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o)
      for (int k = 0; k < 4; ++k) sm[k][threadIdx.x] += sm[k][threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x < 4) part[blockIdx.x * 4 + threadIdx.x] = sm[threadIdx.x][0];
}

}  // namespace

int frac_sum_parts() { return 512; }

cudaError_t launch_frac_sum(cudaStream_t st, const float4* frac, int n, double* part) {
  k_frac_sum<<<frac_sum_parts(), 256, 0, st>>>(frac, n, part);
  return cudaGetLastError();
}

cudaError_t launch_particles_advance(cudaStream_t st, const Dims& d, const StepParams& sp, bool move,
                                     Particles cur, Particles tmp, const float* u0, const float* v0,
                                     const float* w0, const float* un, const float* vn, const float* wn,
                                     const float4* nvf, int* key, int* slot, int* count, int n) {
  if (n <= 0) return cudaSuccess;
  const int nb = blocks_for(n, 256);
  const bool multi = sp.multiphase != 0;
  if (move && multi)
    k_particles_advance<true, true><<<nb, 256, 0, st>>>(d, sp, cur, tmp, u0, v0, w0, un, vn, wn, nvf, key, slot, count, n);
  else if (move)
    k_particles_advance<true, false><<<nb, 256, 0, st>>>(d, sp, cur, tmp, u0, v0, w0, un, vn, wn, nvf, key, slot, count, n);
  else if (multi)
    k_particles_advance<false, true><<<nb, 256, 0, st>>>(d, sp, cur, tmp, u0, v0, w0, un, vn, wn, nvf, key, slot, count, n);
  else
    k_particles_advance<false, false><<<nb, 256, 0, st>>>(d, sp, cur, tmp, u0, v0, w0, un, vn, wn, nvf, key, slot, count, n);
  return cudaGetLastError();
}

cudaError_t launch_ink_advance(cudaStream_t st, const Dims& d, float dt, Particles ink, const float* u0,
                               const float* v0, const float* w0, const float* un, const float* vn, const float* wn,
                               int n) {
  if (n <= 0) return cudaSuccess;
  k_ink_advance<<<blocks_for(n, 256), 256, 0, st>>>(d, dt, ink, u0, v0, w0, un, vn, wn, n);
  return cudaGetLastError();
}

cudaError_t launch_batch_particles_advance(cudaStream_t st, const BatchIndex& bi, int total_blocks, int grid,
                                           bool move, Particles cur, Particles tmp, const float* u0, const float* v0,
                                           const float* w0, const float* un, const float* vn, const float* wn,
                                           int* key, int* slot, int* count) {
  if (total_blocks <= 0) return cudaSuccess;
  const int g = move ? batch_grid(kb_particles_advance<true>, 256, grid, total_blocks)
                     : batch_grid(kb_particles_advance<false>, 256, grid, total_blocks);
  if (move)
    kb_particles_advance<true><<<g, 256, 0, st>>>(bi, total_blocks, cur, tmp, u0, v0, w0, un, vn, wn, key, slot, count);
  else
    kb_particles_advance<false><<<g, 256, 0, st>>>(bi, total_blocks, cur, tmp, u0, v0, w0, un, vn, wn, key, slot, count);
  return cudaGetLastError();
}

size_t cell_scan_tiles(int C) { return (size_t)((C + 1 + kScanTile - 1) / kScanTile); }

cudaError_t launch_cell_scan(cudaStream_t st, int C, int* count, int* off, int* tile_sums) {
  const int n1 = C + 1;
  const int nt = (int)cell_scan_tiles(C);
  k_scan_reduce<<<nt, kScanThreads, 0, st>>>(count, n1, tile_sums);
  k_scan_top<<<1, 1024, 0, st>>>(tile_sums, nt);
  k_scan_apply<<<nt, kScanThreads, 0, st>>>(count, n1, tile_sums, off);
  return cudaGetLastError();
}

cudaError_t launch_scatter(cudaStream_t st, const int* key, const int* slot, const int* off, int* perm_u, int n) {
  if (n <= 0) return cudaSuccess;
  k_scatter<<<blocks_for(n, 256), 256, 0, st>>>(key, slot, off, perm_u, n);
  return cudaGetLastError();
}

cudaError_t launch_rank_gather(cudaStream_t st, bool multiphase, const int* key, const int* off,
                               const int* perm_u, Particles tmp, Particles cur, int* sort_index, int n) {
  if (n <= 0) return cudaSuccess;
  if (multiphase)
    k_rank_gather<true><<<blocks_for(n, 256), 256, 0, st>>>(key, off, perm_u, tmp, cur, sort_index, n);
  else
    k_rank_gather<false><<<blocks_for(n, 256), 256, 0, st>>>(key, off, perm_u, tmp, cur, sort_index, n);
  return cudaGetLastError();
}

}  // namespace aqb
