// Surface mesher kernels: particle SDF and marching cubes.
//
// Reference: Mesher (Rendering/Renderer3D/Mesher.cuh:20-178,
// Rendering/Renderer3D/Mesher.cu:321-630), built by Fluid::init with
// particle spacing h/2 (Fluid/Fluid_3D_FLIP.cu:495).
//
// The reference re-sorts the particle array by the SDF grid (cell h/2) with
// performSpatialHashing2 and swaps it into the fluid.  Here the fluid's
// particles stay as the step left them (sorted by fluid cell h): an SDF hash
// cell lies inside one fluid cell, so the stable SDF order is each fluid
// cell's particles filtered by sub-cell, which the rank kernel computes
// without moving the fluid's arrays (positions are gathered into a side
// buffer in SDF order).  computeSDF's sums run in the reference's order.
//
// Marching cubes samples the SDF through the texture unit exactly as the
// reference does (cudaArray, linear filter, unnormalised coordinates, border
// in x), so the vertex samples are the reference's.  Records are written in
// cube order through a scan instead of an atomic counter, so the output is
// deterministic; record layout and triangle table are the reference's.
#include "aq_kernels.cuh"
#include "mc_table.h"

namespace aqb {
namespace {

__constant__ uint64_t c_mc_tri[256] = {AQ_MC_TRIANGLE_ROWS};
__constant__ int c_mc_edge[12][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}, {4, 5}, {5, 6},
                                     {6, 7}, {7, 4}, {0, 4}, {1, 5}, {2, 6}, {3, 7}};
__constant__ int c_mc_vertex[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 0, 1}, {0, 0, 1},
                                      {0, 1, 0}, {1, 1, 0}, {1, 1, 1}, {0, 1, 1}};

inline int blocks(long long n, int t) { return (int)((n + t - 1) / t); }

// calcHashImpl on the SDF hash grid (Fluid/Fluid_3D_kernels.cuh:8-27):
// truncation of position / h_sdf, flat index x*(HY*HZ) + y*HZ + z.
// Positions inside the domain never reach the clamps (the hash grid extends
// past it); they keep any other input inside the arrays.
__device__ __forceinline__ int sdf_key(const MeshDims& m, float px, float py, float pz) {
  int x = (int)__fdiv_rn(px, m.hs), y = (int)__fdiv_rn(py, m.hs), z = (int)__fdiv_rn(pz, m.hs);
  x = min(max(x, 0), m.HX - 1);
  y = min(max(y, 0), m.HY - 1);
  z = min(max(z, 0), m.HZ - 1);
  return (x * m.HY + y) * m.HZ + z;
}

__global__ void __launch_bounds__(256) k_sdf_keys(MeshDims m, const float* __restrict__ px,
                                                 const float* __restrict__ py, const float* __restrict__ pz,
                                                 int* __restrict__ skey, int* __restrict__ scount, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int k = sdf_key(m, px[i], py[i], pz[i]);
  skey[i] = k;
  atomicAdd(scount + k, 1);
}

// Stable placement: the rank of particle i among the particles of its fluid
// cell segment [off[c], off[c+1]) that share its SDF key and precede it.
// Particles must be sorted by fluid cell (as every step leaves them); a
// particle outside its cell's segment sets *bad and is not placed.  The
// placed float4 carries the particle's hash z in w.
__global__ void __launch_bounds__(256) k_sdf_scatter(MeshDims m, Dims d, const float* __restrict__ px,
                                                    const float* __restrict__ py, const float* __restrict__ pz,
                                                    const int* __restrict__ off, const int* __restrict__ skey,
                                                    const int* __restrict__ soff, float4* __restrict__ spos,
                                                    int* __restrict__ bad, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float x = px[i], y = py[i], z = pz[i];
  int cx = (int)__fdiv_rn(x, d.h), cy = (int)__fdiv_rn(y, d.h), cz = (int)__fdiv_rn(z, d.h);
  cx = min(max(cx, 0), d.sx - 1);
  cy = min(max(cy, 0), d.sy - 1);
  cz = min(max(cz, 0), d.sz - 1);
  const int c = cell_index(d, cx, cy, cz);
  const int j0 = off[c];
  if (i < j0 || i >= off[c + 1]) {
    atomicOr(bad, 1);
    return;
  }
  const int k = skey[i];
  int rank = 0;
  for (int j = j0; j < i; ++j) rank += skey[j] == k;
  if (rank >= soff[k + 1] - soff[k]) {
    atomicOr(bad, 1);
    return;
  }
  spos[soff[k] + rank] = make_float4(x, y, z, __int_as_float(k % m.HZ));
}

// computeSDF (Mesher.cuh:20-84).  A thread computes ZT consecutive SDF cells
// along z: for each (a, b) hash row it walks the particles of the union of
// their hash-cell windows once (contiguous in SDF order) and adds each
// particle to the cells whose window holds its hash cell, so every cell sums
// its particles in the reference's order (rows a, b, then c, then particle).
// Hash cells outside the hash grid are skipped (the reference reaches them
// only through its flat index, whose far cells carry zero weight).
template <int ZT>
__global__ void __launch_bounds__(256) k_sdf(MeshDims m, const int* __restrict__ soff,
                                            const float4* __restrict__ spos, cudaSurfaceObject_t surf) {
  const int nzq = (m.SZ + ZT - 1) / ZT;
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)m.SX * m.SY * nzq) return;
  const int zq = (int)(idx % nzq);
  const int y = (int)((idx / nzq) % m.SY);
  const int x = (int)(idx / ((long long)m.SY * nzq));
  const int z0 = zq * ZT;
  const float cx = __fmul_rn((float)(x - 1), m.hs), cy = __fmul_rn((float)(y - 1), m.hs);
  float cz[ZT];
#pragma unroll
  for (int k = 0; k < ZT; ++k) cz[k] = __fmul_rn((float)(z0 + k - 1), m.hs);
  const float R = __fmul_rn(m.hs, 2.f);
  const float h2 = __fmul_rn(R, R), h2x3 = __fmul_rn(h2, 3.f);
  float sw[ZT], sx[ZT], sy[ZT], sz[ZT];
#pragma unroll
  for (int k = 0; k < ZT; ++k) sw[k] = sx[k] = sy[k] = sz[k] = 0.f;
  const int a0 = max(x - 3, 0), a1 = min(x, m.HX - 1);
  const int b0 = max(y - 3, 0), b1 = min(y, m.HY - 1);
  const int c0 = max(z0 - 3, 0), c1 = min(z0 + ZT - 1, m.HZ - 1);
  if (c0 <= c1) {
    for (int a = a0; a <= a1; ++a)
      for (int b = b0; b <= b1; ++b) {
        const int row = (a * m.HY + b) * m.HZ;
        const int j0 = __ldg(soff + row + c0), j1 = __ldg(soff + row + c1 + 1);
        for (int j = j0; j < j1; ++j) {
          const float4 p = __ldg(spos + j);
          const int c = __float_as_int(p.w);  // the particle's hash z
          const float rx = __fsub_rn(p.x, cx), ry = __fsub_rn(p.y, cy);
          const float rxy = __fadd_rn(__fmul_rn(rx, rx), __fmul_rn(ry, ry));
#pragma unroll
          for (int k = 0; k < ZT; ++k) {
            if (c < z0 + k - 3 || c > z0 + k) continue;
            // dunfanKernel (Fluid/WeightKernels.cuh:183-189), rounded as
            // written.  Outside the support the weight is 0 and adding it
            // (and 0 * p) leaves every sum unchanged, so those are skipped.
            const float rz = __fsub_rn(p.z, cz[k]);
            const float r2 = __fadd_rn(rxy, __fmul_rn(rz, rz));
            if (r2 > h2) continue;
            const float t = __fsub_rn(1.f, __fdiv_rn(r2, h2x3));
            const float w = fmaxf(0.f, __fmul_rn(__fmul_rn(t, t), t));
            sw[k] = __fadd_rn(sw[k], w);
            sx[k] = __fadd_rn(sx[k], __fmul_rn(w, p.x));
            sy[k] = __fadd_rn(sy[k], __fmul_rn(w, p.y));
            sz[k] = __fadd_rn(sz[k], __fmul_rn(w, p.z));
          }
        }
      }
  }
#pragma unroll
  for (int k = 0; k < ZT; ++k) {
    const int z = z0 + k;
    if (z >= m.SZ) break;
    float v = m.hs;  // "set to some positive value first"
    if (sw[k] != 0.f) {
      const float ex = __fsub_rn(__fdiv_rn(sx[k], sw[k]), cx), ey = __fsub_rn(__fdiv_rn(sy[k], sw[k]), cy),
                  ez = __fsub_rn(__fdiv_rn(sz[k], sw[k]), cz[k]);
      v = __fsub_rn(__fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(ex, ex), __fmul_rn(ey, ey)), __fmul_rn(ez, ez))),
                    m.radius);
    }
    surf3Dwrite(v, surf, x * (int)sizeof(float), y, z);
  }
}

constexpr int kSdfZ = 4;

// getSDF at a world position (Mesher.cu:312-318): texture coordinate
// 1 + position / h_sdf, filtered by the texture unit.
__device__ __forceinline__ float sdf_at(const MeshDims& m, cudaTextureObject_t tex, float px, float py, float pz) {
  return tex3D<float>(tex, __fadd_rn(1.f, __fdiv_rn(px, m.hs)), __fadd_rn(1.f, __fdiv_rn(py, m.hs)),
                      __fadd_rn(1.f, __fdiv_rn(pz, m.hs)));
}

// getSDF on mesh vertex (x, y, z) (Mesher.cu:294-308): 0 on the outer layers.
__global__ void __launch_bounds__(256) k_mc_vertices(MeshDims m, cudaTextureObject_t tex, float* __restrict__ vv) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int VX = m.MX + 1, VY = m.MY + 1, VZ = m.MZ + 1;
  if (idx >= (long long)VX * VY * VZ) return;
  const int z = (int)(idx % VZ);
  const int y = (int)((idx / VZ) % VY);
  const int x = (int)(idx / ((long long)VY * VZ));
  float v = 0.f;
  if (!(x == 0 || y == 0 || z == 0 || x >= m.MX - 1 || y >= m.MY - 1 || z >= m.MZ - 1))
    v = sdf_at(m, tex, __fmul_rn((float)(x - 1), m.hm), __fmul_rn((float)(y - 1), m.hm),
               __fmul_rn((float)(z - 1), m.hm));
  vv[idx] = v;
}

__device__ __forceinline__ int cube_type(const MeshDims& m, const float* __restrict__ vv, int x, int y, int z) {
  const int VY = m.MY + 1, VZ = m.MZ + 1;
  int t = 0;
#pragma unroll
  for (int v = 0; v < 8; ++v) {
    const long long q = ((long long)(x + c_mc_vertex[v][0]) * VY + (y + c_mc_vertex[v][1])) * VZ + (z + c_mc_vertex[v][2]);
    t |= (__ldg(vv + q) < 0.f ? 1 : 0) << v;
  }
  return t;
}

// Occupancy: a cube whose type row holds triangles (every type but 0 and 255).
__global__ void __launch_bounds__(256) k_mc_flags(MeshDims m, const float* __restrict__ vv, uint8_t* __restrict__ ctype,
                                                 int* __restrict__ flag) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)m.MX * m.MY * m.MZ) return;
  const int z = (int)(idx % m.MZ);
  const int y = (int)((idx / m.MZ) % m.MY);
  const int x = (int)(idx / ((long long)m.MY * m.MZ));
  const int t = cube_type(m, vv, x, y, z);
  ctype[idx] = (uint8_t)t;
  flag[idx] = (t != 0 && t != 255) ? 1 : 0;
}

// marchingCubes (Mesher.cu:322-425): the record of an occupied cube, written
// at its rank in cube order; unused slots are zero.
__global__ void __launch_bounds__(128) k_mc_emit(MeshDims m, cudaTextureObject_t tex, const float* __restrict__ vv,
                                                const uint8_t* __restrict__ ctype, const int* __restrict__ moff,
                                                float* __restrict__ out, long long capacity) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)m.MX * m.MY * m.MZ) return;
  const int t = ctype[idx];
  if (t == 0 || t == 255) return;
  const long long r = moff[idx];
  if (r >= capacity) return;
  const int z = (int)(idx % m.MZ);
  const int y = (int)((idx / m.MZ) % m.MY);
  const int x = (int)(idx / ((long long)m.MY * m.MZ));
  const int VY = m.MY + 1, VZ = m.MZ + 1;
  const uint64_t row = c_mc_tri[t];
  const float hm = m.hm;
  const float bx = __fmul_rn((float)(x - 1), hm), by = __fmul_rn((float)(y - 1), hm), bz = __fmul_rn((float)(z - 1), hm);
  const float d = hm / 2;
  float* rec = out + r * 90;
  for (int i = 0; i < 15; ++i) {
    float* o = rec + 6 * i;
    const int e = aq_mc_entry(row, i);
    if (e < 0) {
#pragma unroll
      for (int k = 0; k < 6; ++k) o[k] = 0.f;
      continue;
    }
    const int* ca = c_mc_vertex[c_mc_edge[e][0]];
    const int* cb = c_mc_vertex[c_mc_edge[e][1]];
    const float sa = __ldg(vv + ((long long)(x + ca[0]) * VY + (y + ca[1])) * VZ + (z + ca[2]));
    const float sb = __ldg(vv + ((long long)(x + cb[0]) * VY + (y + cb[1])) * VZ + (z + cb[2]));
    const float f = __fdiv_rn(-sa, __fsub_rn(sb, sa));
    const float g = __fsub_rn(1.f, f);
    const float px = __fadd_rn(bx, __fmul_rn(__fadd_rn(__fmul_rn((float)ca[0], g), __fmul_rn((float)cb[0], f)), hm));
    const float py = __fadd_rn(by, __fmul_rn(__fadd_rn(__fmul_rn((float)ca[1], g), __fmul_rn((float)cb[1], f)), hm));
    const float pz = __fadd_rn(bz, __fmul_rn(__fadd_rn(__fmul_rn((float)ca[2], g), __fmul_rn((float)cb[2], f)), hm));
    const float l = sdf_at(m, tex, __fadd_rn(px, -d), py, pz), rr = sdf_at(m, tex, __fadd_rn(px, d), py, pz);
    const float u = sdf_at(m, tex, px, __fadd_rn(py, d), pz), dn = sdf_at(m, tex, px, __fadd_rn(py, -d), pz);
    const float fr = sdf_at(m, tex, px, py, __fadd_rn(pz, d)), bk = sdf_at(m, tex, px, py, __fadd_rn(pz, -d));
    const float nx = __fsub_rn(rr, l), ny = __fsub_rn(u, dn), nz = __fsub_rn(fr, bk);
    // normalize (helper_math): v * rsqrtf(dot(v, v))
    const float inv = rsqrtf(__fadd_rn(__fadd_rn(__fmul_rn(nx, nx), __fmul_rn(ny, ny)), __fmul_rn(nz, nz)));
    o[0] = px; o[1] = py; o[2] = pz;
    o[3] = __fmul_rn(nx, inv); o[4] = __fmul_rn(ny, inv); o[5] = __fmul_rn(nz, inv);
  }
}

// Zeroes the records the previous call wrote past this call's count, so the
// buffer holds zeros after the last record as the reference's memset leaves
// it; then remembers the count.
__global__ void __launch_bounds__(256) k_mc_tail(const int* __restrict__ total, int* __restrict__ prev,
                                                float* __restrict__ out, long long capacity) {
  const long long cur = min((long long)*total, capacity);
  const long long old = min((long long)*prev, capacity);
  for (long long q = cur * 90 + (long long)blockIdx.x * blockDim.x + threadIdx.x; q < old * 90;
       q += (long long)gridDim.x * blockDim.x)
    out[q] = 0.f;
}

__global__ void k_mc_remember(const int* __restrict__ total, int* __restrict__ prev) { *prev = *total; }

}  // namespace

cudaError_t launch_sdf_keys(cudaStream_t st, const MeshDims& m, const float* px, const float* py, const float* pz,
                            int* skey, int* scount, int n) {
  if (n <= 0) return cudaSuccess;
  k_sdf_keys<<<blocks(n, 256), 256, 0, st>>>(m, px, py, pz, skey, scount, n);
  return cudaGetLastError();
}

cudaError_t launch_sdf_scatter(cudaStream_t st, const MeshDims& m, const Dims& d, const float* px, const float* py,
                               const float* pz, const int* off, const int* skey, const int* soff, float4* spos,
                               int* bad, int n) {
  if (n <= 0) return cudaSuccess;
  k_sdf_scatter<<<blocks(n, 256), 256, 0, st>>>(m, d, px, py, pz, off, skey, soff, spos, bad, n);
  return cudaGetLastError();
}

cudaError_t launch_sdf(cudaStream_t st, const MeshDims& m, const int* soff, const float4* spos,
                       cudaSurfaceObject_t surf) {
  const long long nzq = (m.SZ + kSdfZ - 1) / kSdfZ;
  k_sdf<kSdfZ><<<blocks((long long)m.SX * m.SY * nzq, 256), 256, 0, st>>>(m, soff, spos, surf);
  return cudaGetLastError();
}

cudaError_t launch_mc_vertices(cudaStream_t st, const MeshDims& m, cudaTextureObject_t tex, float* vv) {
  k_mc_vertices<<<blocks((long long)(m.MX + 1) * (m.MY + 1) * (m.MZ + 1), 256), 256, 0, st>>>(m, tex, vv);
  return cudaGetLastError();
}

cudaError_t launch_mc_flags(cudaStream_t st, const MeshDims& m, const float* vv, uint8_t* ctype, int* flag) {
  k_mc_flags<<<blocks((long long)m.MX * m.MY * m.MZ, 256), 256, 0, st>>>(m, vv, ctype, flag);
  return cudaGetLastError();
}

cudaError_t launch_mc_emit(cudaStream_t st, const MeshDims& m, cudaTextureObject_t tex, const float* vv,
                           const uint8_t* ctype, const int* moff, float* out, long long capacity) {
  k_mc_emit<<<blocks((long long)m.MX * m.MY * m.MZ, 128), 128, 0, st>>>(m, tex, vv, ctype, moff, out, capacity);
  return cudaGetLastError();
}

cudaError_t launch_mc_tail(cudaStream_t st, const int* total, int* prev, float* out, long long capacity) {
  k_mc_tail<<<296, 256, 0, st>>>(total, prev, out, capacity);
  k_mc_remember<<<1, 1, 0, st>>>(total, prev);
  return cudaGetLastError();
}

}  // namespace aqb
