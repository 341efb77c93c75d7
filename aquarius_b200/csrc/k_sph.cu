// Kernels of the particle-only solvers: position-based fluids and PCISPH.
//
// Reference: Fluid_3D_PBF (Fluid/Fluid_3D_PBF.cu:6-267) and Fluid_3D_PCISPH
// (Fluid/Fluid_3D_PCISPH.cu:13-202), with poly6 / spikey_grad /
// cubic_spline_kernel (Fluid/WeightKernels.cuh:13-58, 196-206) and the
// spatial hash of performSpatialHashing2 (Fluid/Fluid_3D_common.cuh:27-56).
//
// Particles live as float4 arrays (16-byte loads in the neighbour loops):
//   PBF:    P = (position, restDensity), L = (lastPosition, -),
//           V = (velocity, density), Q = (position, lambda) written by the
//           lambda pass and read by the delta pass, which writes P.
//   PCISPH: P = (position, restDensity), V = (velocity, density),
//           Q = (predictedPosition, -), W = (predictedVelocity, pressure),
//           F = (pressureForces, -), R = (predictedPosition, p / rho^2)
//           written by the density pass and read by the force pass.
// No pass reads a float4 another thread of the same pass writes.
//
// Every float operation is an explicitly rounded intrinsic in the order the
// reference writes it (no contraction), and neighbours are walked in the
// reference's order (27 cells x-major, particles in stable sorted order), so
// results equal the CPU oracle's bit for bit.
#include "aq_kernels.cuh"

namespace aqb {
namespace {

constexpr float kPi = 3.14159265358979323846f;  // PI (Fluid/WeightKernels.cuh:8)
constexpr float k64Pi = 64.f * kPi;

inline int blocks(int n, int t) { return (n + t - 1) / t; }

__device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float dvd(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ float clampw(float v, float lo, float hi) { return fminf(hi, fmaxf(lo, v)); }

__device__ __forceinline__ float dot3(float x, float y, float z) { return add(add(mul(x, x), mul(y, y)), mul(z, z)); }

// Neighbour pairs with r2 > p.skip_r2 lie outside both kernels' support:
// poly6 is 0 (r2 > h2) and spikey_grad is the zero vector (sqrt(r2) > h).
// Adding their zero terms changes no sum (at most the sign of a zero that is
// then squared or added to a nonzero value), so the passes skip them; about
// 85% of the 27-cell candidates are such pairs.
__device__ __forceinline__ bool outside(float r2, const SphParams& p) { return r2 > p.skip_r2; }

// poly6 (Fluid/WeightKernels.cuh:13-26)
__device__ __forceinline__ float poly6(float vx, float vy, float vz, const SphParams& p) {
  const float r2 = dot3(vx, vy, vz);
  if (r2 <= p.kr2) {
    const float t = sub(p.kr2, r2);
    return dvd(mul(mul(mul(t, t), t), 315.f), mul(k64Pi, p.kr9));
  }
  return 0.f;
}

// spikey_grad (Fluid/WeightKernels.cuh:43-58)
__device__ __forceinline__ float3 spikey(float vx, float vy, float vz, const SphParams& p) {
  const float r = __fsqrt_rn(dot3(vx, vy, vz));
  float ux = vx, uy = vy, uz = vz;
  if (r != 0.f) { ux = dvd(ux, r); uy = dvd(uy, r); uz = dvd(uz, r); }
  if (0.f <= r && r <= p.kr) {
    const float hr = sub(p.kr, r), d = mul(kPi, p.kr6);
    return make_float3(dvd(mul(mul(mul(-ux, hr), hr), 45.f), d), dvd(mul(mul(mul(-uy, hr), hr), 45.f), d),
                       dvd(mul(mul(mul(-uz, hr), hr), 45.f), d));
  }
  return make_float3(0.f, 0.f, 0.f);
}

__device__ __forceinline__ int3 cell_of(const SphParams& p, float x, float y, float z) {
  return make_int3((int)dvd(x, p.kr), (int)dvd(y, p.kr), (int)dvd(z, p.kr));
}

// The 27 cells around c, dx, dy, dz from -1 to 1, outside ones skipped
// (Fluid/Fluid_3D_PBF.cu:37-58); body(j) for every particle j in them.
template <typename Body>
__device__ __forceinline__ void for_neighbours(const SphParams& p, int3 c, const int* __restrict__ off, Body&& body) {
  for (int dx = -1; dx <= 1; ++dx) {
    const int x = c.x + dx;
    if (x < 0 || x >= p.gx) continue;
    for (int dy = -1; dy <= 1; ++dy) {
      const int y = c.y + dy;
      if (y < 0 || y >= p.gy) continue;
      const int row = (x * p.gy + y) * p.gz;
      for (int dz = -1; dz <= 1; ++dz) {
        const int z = c.z + dz;
        if (z < 0 || z >= p.gz) continue;
        const int j1 = __ldg(off + row + z + 1);
        for (int j = __ldg(off + row + z); j < j1; ++j) body(j);
      }
    }
  }
}

// The neighbour walk in two phases, still in the reference's order: a cheap
// scan keeps the candidates inside the support (their indices, in shared
// memory, kBuf per thread), then the costly terms are evaluated from that
// list.  Inside candidates are about 15% of the scan and fall on different
// lanes; evaluated in the scan the warp would run the costly arithmetic with
// a few lanes at a time, from the lists all lanes run it together.  Used by
// the two PBF passes, whose terms cost most (measured: 1.5x); PCISPH's were
// faster evaluated in the scan.
constexpr int kBuf = 48;  // 48 x 256 threads x 4 B = the 48 KB of static shared memory

template <typename Inside, typename Eval>
__device__ __forceinline__ void walk_inside(const SphParams& p, int3 c, const int* __restrict__ off, int* buf,
                                            Inside&& inside, Eval&& eval) {
  const int stride = blockDim.x, tid = threadIdx.x;
  int cnt = 0;
  for_neighbours(p, c, off, [&](int j) {
    if (!inside(j)) return;
    buf[cnt * stride + tid] = j;
    if (++cnt == kBuf) {
      for (int q = 0; q < kBuf; ++q) eval(buf[q * stride + tid]);
      cnt = 0;
    }
  });
  for (int q = 0; q < cnt; ++q) eval(buf[q * stride + tid]);
}

// --------------------------------------------------------------- sorting

// calcHashImpl (Fluid/Fluid_3D_kernels.cuh:8-27) on the kernel-radius grid,
// and a warp-aggregated slot in the cell's count.  Positions are kept inside
// the container, so the clamps only guard against other input.
__global__ void __launch_bounds__(256) k_sph_keys(SphParams p, const float4* __restrict__ pos, int* __restrict__ key,
                                                 int* __restrict__ slot, int* __restrict__ count, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const bool valid = i < n;
  int k = -1;
  if (valid) {
    const float4 q = pos[i];
    int3 c = cell_of(p, q.x, q.y, q.z);
    c.x = min(max(c.x, 0), p.gx - 1);
    c.y = min(max(c.y, 0), p.gy - 1);
    c.z = min(max(c.z, 0), p.gz - 1);
    k = (c.x * p.gy + c.y) * p.gz + c.z;
    key[i] = k;
  }
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

// Stable placement (rank among the cell's particles by previous index, as
// thrust's stable sort orders them) and the gather of every particle array.
__global__ void __launch_bounds__(256) k_sph_gather(const int* __restrict__ key, const int* __restrict__ off,
                                                   const int* __restrict__ perm_u, SphArrays src, SphArrays dst, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int k = key[i];
  const int b = __ldg(off + k), e = __ldg(off + k + 1);
  int r = 0;
  for (int j = b; j < e; ++j) r += __ldg(perm_u + j) < i;
  const int d = b + r;
#pragma unroll
  for (int a = 0; a < kSphArrays; ++a)
    if (src.a[a]) dst.a[a][d] = src.a[a][i];
}

// ------------------------------------------------------------------- PBF

// applyForcesImpl + predictPositionImpl (Fluid_3D_PBF.cu:6-26)
__global__ void __launch_bounds__(256) k_pbf_predict(SphParams p, float4* __restrict__ P, const float4* __restrict__ L,
                                                    float4* __restrict__ V, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float4 v = V[i], q = P[i];
  const float4 l = L[i];
  v.x = add(v.x, mul(p.dt, p.g.x));
  v.y = add(v.y, mul(p.dt, p.g.y));
  v.z = add(v.z, mul(p.dt, p.g.z));
  q.x = clampw(add(l.x, mul(p.dt, v.x)), p.md, sub(p.size, p.md));
  q.y = clampw(add(l.y, mul(p.dt, v.y)), p.md, sub(p.size, p.md));
  q.z = clampw(add(l.z, mul(p.dt, v.z)), p.md, sub(p.size, p.md));
  V[i] = v;
  P[i] = q;
}

// computeDensityAndLambdaImpl (Fluid_3D_PBF.cu:28-110): reads P, writes
// Q = (position, lambda), the density into V.w and, on the rest-density
// pass, P.w.
__global__ void __launch_bounds__(256) k_pbf_lambda(SphParams p, const int* __restrict__ off, float4* __restrict__ P,
                                                   float4* __restrict__ V, float4* __restrict__ Q, int set_rest, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  __shared__ int buf[kBuf * 256];
  const float4 me = P[i];
  float gx = 0.f, gy = 0.f, gz = 0.f, sdot = 0.f, density = 0.f;
  walk_inside(
      p, cell_of(p, me.x, me.y, me.z), off, buf,
      [&](int j) {
        const float4 o = __ldg(P + j);
        return !outside(dot3(sub(me.x, o.x), sub(me.y, o.y), sub(me.z, o.z)), p);
      },
      [&](int j) {
        const float4 o = __ldg(P + j);
        const float dx = sub(me.x, o.x), dy = sub(me.y, o.y), dz = sub(me.z, o.z);
        density = add(density, poly6(dx, dy, dz, p));
        const float3 w = spikey(dx, dy, dz, p);
        gx = add(gx, w.x);
        gy = add(gy, w.y);
        gz = add(gz, w.z);
        sdot = add(sdot, dot3(w.x, w.y, w.z));
      });
  const float rho0 = set_rest ? density : me.w;
  const float ci = sub(dvd(density, rho0), 1.f);
  const float q = dvd(add(sdot, dot3(gx, gy, gz)), mul(rho0, rho0));
  const float den = __double2float_rn(__dadd_rn(1e-3, (double)q));
  float lambda = dvd(-ci, den);
  if (ci < 0.f) lambda = __double2float_rn(__dmul_rn((double)lambda, 1e-2));
  V[i].w = density;
  if (set_rest) P[i].w = density;
  Q[i] = make_float4(me.x, me.y, me.z, lambda);
}

// computeDeltaPositionImpl + applyDeltaPositionImpl (Fluid_3D_PBF.cu:114-206):
// reads Q, writes the moved position into P (its w, the rest density, kept).
__global__ void __launch_bounds__(256) k_pbf_delta(SphParams p, const int* __restrict__ off,
                                                  const float4* __restrict__ Q, float4* __restrict__ P, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  __shared__ int buf[kBuf * 256];
  const float4 me = Q[i];
  const float rho0 = P[i].w;
  float ax = 0.f, ay = 0.f, az = 0.f;
  walk_inside(
      p, cell_of(p, me.x, me.y, me.z), off, buf,
      [&](int j) {
        const float4 o = __ldg(Q + j);
        return !outside(dot3(sub(me.x, o.x), sub(me.y, o.y), sub(me.z, o.z)), p);
      },
      [&](int j) {
        const float4 o = __ldg(Q + j);
        const float dx = sub(me.x, o.x), dy = sub(me.y, o.y), dz = sub(me.z, o.z);
        const float3 w = spikey(dx, dy, dz, p);
        const float t = dvd(poly6(dx, dy, dz, p), p.s_corr_den);
        const float t2 = mul(t, t);
        const float sc = mul(mul(t2, t2), -p.s_corr_k);
        const float f = add(add(me.w, o.w), sc);
        ax = add(ax, dvd(mul(w.x, f), rho0));
        ay = add(ay, dvd(mul(w.y, f), rho0));
        az = add(az, dvd(mul(w.z, f), rho0));
      });
  const float hi = sub(p.size, p.md);
  P[i] = make_float4(clampw(add(me.x, ax), p.md, hi), clampw(add(me.y, ay), p.md, hi), clampw(add(me.z, az), p.md, hi),
                     rho0);
}

// updatePositionAndVelocityImpl (Fluid_3D_PBF.cu:209-267)
__device__ __forceinline__ float pbf_wall(float v, bool low, bool high, float leave) {
  if (low) v = v == 0.f ? leave : mul(v, -0.5f);
  if (high) v = v == 0.f ? -leave : mul(v, -0.5f);
  return v;
}

__global__ void __launch_bounds__(256) k_pbf_update(SphParams p, const float4* __restrict__ P, float4* __restrict__ L,
                                                   float4* __restrict__ V, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float4 q = P[i];
  const float4 l = L[i];
  float4 v = V[i];
  const float hi = sub(p.size, p.md);
  v.x = pbf_wall(dvd(sub(q.x, l.x), p.dt), q.x == p.md, q.x >= hi, p.leave);
  v.y = pbf_wall(dvd(sub(q.y, l.y), p.dt), q.y <= p.md, q.y >= hi, p.leave);
  v.z = pbf_wall(dvd(sub(q.z, l.z), p.dt), q.z <= p.md, q.z >= hi, p.leave);
  V[i] = v;
  L[i] = make_float4(q.x, q.y, q.z, l.w);
}

// ---------------------------------------------------------------- PCISPH

// predictVelocityAndPositionImpl (Fluid_3D_PCISPH.cu:32-86): the predicted
// position / velocity (into Q, W) or, at the end of a substep, the actual
// ones (into P, V); the acceleration is the gravity.
__device__ __forceinline__ void pci_wall(float& q, float& v, float md, float hi) {
  if (q < md) { q = md; v = mul(v, -0.0f); }
  if (q > hi) { q = hi; v = mul(v, -0.0f); }
}

__global__ void __launch_bounds__(256) k_pci_predict(SphParams p, float4* __restrict__ P, float4* __restrict__ V,
                                                    float4* __restrict__ Q, float4* __restrict__ W,
                                                    const float4* __restrict__ F, int actual, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float4 q = P[i], v = V[i], f = F[i];
  float vx = add(v.x, mul(add(p.g.x, f.x), p.dt)), vy = add(v.y, mul(add(p.g.y, f.y), p.dt)),
        vz = add(v.z, mul(add(p.g.z, f.z), p.dt));
  float px = add(q.x, mul(vx, p.dt)), py = add(q.y, mul(vy, p.dt)), pz = add(q.z, mul(vz, p.dt));
  const float hi = sub(p.size, p.md);
  pci_wall(px, vx, p.md, hi);
  pci_wall(py, vy, p.md, hi);
  pci_wall(pz, vz, p.md, hi);
  if (actual) {
    P[i] = make_float4(px, py, pz, q.w);
    V[i] = make_float4(vx, vy, vz, v.w);
  } else {
    Q[i] = make_float4(px, py, pz, 0.f);
    W[i] = make_float4(vx, vy, vz, W[i].w);
  }
}

// predictDensityAndPressureImpl (Fluid_3D_PCISPH.cu:88-159): cells from the
// position, distances from the predicted positions; pressure += 50 * (density
// - rest density), the coefficient the kernel ends with.  Writes the density
// into V.w, the pressure into W.w, R = (predicted position, p / rho^2) and, on
// the rest-density pass, P.w.
__global__ void __launch_bounds__(256) k_pci_density(SphParams p, const int* __restrict__ off, float4* __restrict__ P,
                                                    float4* __restrict__ V, const float4* __restrict__ Q,
                                                    float4* __restrict__ W, float4* __restrict__ R, int set_rest,
                                                    int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float4 me = P[i];
  const float4 pq = Q[i];
  float density = 0.f;
  for_neighbours(p, cell_of(p, me.x, me.y, me.z), off, [&](int j) {
    const float4 o = __ldg(Q + j);
    const float dx = sub(pq.x, o.x), dy = sub(pq.y, o.y), dz = sub(pq.z, o.z);
    if (outside(dot3(dx, dy, dz), p)) return;
    density = add(density, poly6(dx, dy, dz, p));
  });
  const float err = sub(density, me.w);
  const float pressure = add(W[i].w, mul(50.0f, err));
  V[i].w = density;
  W[i].w = pressure;
  if (set_rest) P[i].w = density;
  R[i] = make_float4(pq.x, pq.y, pq.z, dvd(pressure, mul(density, density)));
}

// computePressureForceImpl (Fluid_3D_PCISPH.cu:161-202)
__global__ void __launch_bounds__(256) k_pci_force(SphParams p, const int* __restrict__ off,
                                                  const float4* __restrict__ P, const float4* __restrict__ R,
                                                  float4* __restrict__ F, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float4 me = P[i];
  const float4 r = R[i];
  float fx = 0.f, fy = 0.f, fz = 0.f;
  for_neighbours(p, cell_of(p, me.x, me.y, me.z), off, [&](int j) {
    const float4 o = __ldg(R + j);
    const float dx = sub(r.x, o.x), dy = sub(r.y, o.y), dz = sub(r.z, o.z);
    if (outside(dot3(dx, dy, dz), p)) return;
    const float3 w = spikey(dx, dy, dz, p);
    const float s = add(o.w, r.w);
    fx = sub(fx, mul(w.x, s));
    fy = sub(fy, mul(w.y, s));
    fz = sub(fz, mul(w.z, s));
  });
  F[i] = make_float4(fx, fy, fz, 0.f);
}

// initPressureImpl (Fluid_3D_PCISPH.cu:22-30): pressure and pressure force 0.
__global__ void __launch_bounds__(256) k_pci_init(float4* __restrict__ W, float4* __restrict__ F, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  W[i].w = 0.f;
  F[i] = make_float4(0.f, 0.f, 0.f, 0.f);
}

}  // namespace

cudaError_t launch_sph_keys(cudaStream_t st, const SphParams& p, const float4* pos, int* key, int* slot, int* count,
                            int n) {
  if (n <= 0) return cudaSuccess;
  k_sph_keys<<<blocks(n, 256), 256, 0, st>>>(p, pos, key, slot, count, n);
  return cudaGetLastError();
}

cudaError_t launch_sph_gather(cudaStream_t st, const int* key, const int* off, const int* perm_u, const SphArrays& src,
                              const SphArrays& dst, int n) {
  if (n <= 0) return cudaSuccess;
  k_sph_gather<<<blocks(n, 256), 256, 0, st>>>(key, off, perm_u, src, dst, n);
  return cudaGetLastError();
}

cudaError_t launch_pbf_predict(cudaStream_t st, const SphParams& p, float4* P, const float4* L, float4* V, int n) {
  if (n <= 0) return cudaSuccess;
  k_pbf_predict<<<blocks(n, 256), 256, 0, st>>>(p, P, L, V, n);
  return cudaGetLastError();
}

cudaError_t launch_pbf_lambda(cudaStream_t st, const SphParams& p, const int* off, float4* P, float4* V, float4* Q,
                              bool set_rest, int n) {
  if (n <= 0) return cudaSuccess;
  k_pbf_lambda<<<blocks(n, 256), 256, 0, st>>>(p, off, P, V, Q, set_rest ? 1 : 0, n);
  return cudaGetLastError();
}

cudaError_t launch_pbf_delta(cudaStream_t st, const SphParams& p, const int* off, const float4* Q, float4* P, int n) {
  if (n <= 0) return cudaSuccess;
  k_pbf_delta<<<blocks(n, 256), 256, 0, st>>>(p, off, Q, P, n);
  return cudaGetLastError();
}

cudaError_t launch_pbf_update(cudaStream_t st, const SphParams& p, const float4* P, float4* L, float4* V, int n) {
  if (n <= 0) return cudaSuccess;
  k_pbf_update<<<blocks(n, 256), 256, 0, st>>>(p, P, L, V, n);
  return cudaGetLastError();
}

cudaError_t launch_pci_init(cudaStream_t st, float4* W, float4* F, int n) {
  if (n <= 0) return cudaSuccess;
  k_pci_init<<<blocks(n, 256), 256, 0, st>>>(W, F, n);
  return cudaGetLastError();
}

cudaError_t launch_pci_predict(cudaStream_t st, const SphParams& p, float4* P, float4* V, float4* Q, float4* W,
                               const float4* F, bool actual, int n) {
  if (n <= 0) return cudaSuccess;
  k_pci_predict<<<blocks(n, 256), 256, 0, st>>>(p, P, V, Q, W, F, actual ? 1 : 0, n);
  return cudaGetLastError();
}

cudaError_t launch_pci_density(cudaStream_t st, const SphParams& p, const int* off, float4* P, float4* V,
                               const float4* Q, float4* W, float4* R, bool set_rest, int n) {
  if (n <= 0) return cudaSuccess;
  k_pci_density<<<blocks(n, 256), 256, 0, st>>>(p, off, P, V, Q, W, R, set_rest ? 1 : 0, n);
  return cudaGetLastError();
}

cudaError_t launch_pci_force(cudaStream_t st, const SphParams& p, const int* off, const float4* P, const float4* R,
                             float4* F, int n) {
  if (n <= 0) return cudaSuccess;
  k_pci_force<<<blocks(n, 256), 256, 0, st>>>(p, off, P, R, F, n);
  return cudaGetLastError();
}

}  // namespace aqb
