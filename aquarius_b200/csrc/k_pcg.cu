// FP64 preconditioned conjugate gradient on the pressure system — the
// pressure-error reference (no counterpart in the reference; it is the
// system jacobiImpl relaxes, Fluid/Fluid_3D_kernels.cu:460-505):
//   for fluid cell i:  (6 - n_out) p_i - sum_{in-domain fluid nbrs} p_j = b_i,
//   b = -div*rho, air neighbours 0 (Dirichlet), out-of-domain neighbours
//   dropped (Neumann).  Unknowns live on fluid cells; air entries stay 0.
// Preconditioner: the diagonal (6 - n_out).  Dot products are per-block
// partial sums in fixed order, finished on the host.
#include "aq_kernels.cuh"

namespace aqb {
namespace {

__device__ __forceinline__ void cell_coords(const Dims& d, int c, int& x, int& y, int& z) {
  z = c % d.sz;
  const int t = c / d.sz;
  y = t % d.sy;
  x = t / d.sy;
}

__global__ void k_pcg_init(Dims d, const int8_t* __restrict__ type, const float* __restrict__ rhs,
                           double* __restrict__ b, double* __restrict__ x) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= d.C) return;
  b[c] = type[c] == kFluid ? (double)rhs[c] : 0.0;
  x[c] = 0.0;
}

__global__ void k_pcg_apply(Dims d, const int8_t* __restrict__ type, const double* __restrict__ in,
                            double* __restrict__ out) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= d.C) return;
  if (type[c] != kFluid) { out[c] = 0.0; return; }
  int x, y, z;
  cell_coords(d, c, x, y, z);
  const int sxy = d.sy * d.sz;
  int nin = 0;
  double s = 0.0;
  if (x + 1 < d.sx) { ++nin; s += in[c + sxy]; }
  if (x - 1 >= 0) { ++nin; s += in[c - sxy]; }
  if (y + 1 < d.sy) { ++nin; s += in[c + d.sz]; }
  if (y - 1 >= 0) { ++nin; s += in[c - d.sz]; }
  if (z + 1 < d.sz) { ++nin; s += in[c + 1]; }
  if (z - 1 >= 0) { ++nin; s += in[c - 1]; }
  out[c] = (double)nin * in[c] - s;
}

__global__ void k_pcg_precond(Dims d, const int8_t* __restrict__ type, const double* __restrict__ r,
                              double* __restrict__ z) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= d.C) return;
  if (type[c] != kFluid) { z[c] = 0.0; return; }
  int x, y, zz;
  cell_coords(d, c, x, y, zz);
  const int nin = (x + 1 < d.sx) + (x - 1 >= 0) + (y + 1 < d.sy) + (y - 1 >= 0) + (zz + 1 < d.sz) + (zz - 1 >= 0);
  z[c] = r[c] / (double)nin;
}

__global__ void __launch_bounds__(256) k_pcg_dot(int n, const double* __restrict__ a, const double* __restrict__ b,
                                                double* __restrict__ part) {
  double s = 0.0;
  for (int i = blockIdx.x * 256 + threadIdx.x; i < n; i += gridDim.x * 256) s += a[i] * b[i];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  __shared__ double ws[8];
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int k = 0; k < 8; ++k) t += ws[k];
    part[blockIdx.x] = t;
  }
}

__global__ void k_pcg_axpy(int n, double alpha, const double* __restrict__ xv, double* __restrict__ yv) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) yv[i] += alpha * xv[i];
}

__global__ void k_pcg_xpby(int n, const double* __restrict__ xv, double beta, double* __restrict__ yv) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) yv[i] = xv[i] + beta * yv[i];
}

inline int nb(int n) { return (n + 255) / 256; }

}  // namespace

cudaError_t launch_pcg_init(cudaStream_t st, const Dims& d, const int8_t* type, const float* rhs, double* b,
                            double* x) {
  k_pcg_init<<<nb(d.C), 256, 0, st>>>(d, type, rhs, b, x);
  return cudaGetLastError();
}
cudaError_t launch_pcg_apply(cudaStream_t st, const Dims& d, const int8_t* type, const double* in, double* out) {
  k_pcg_apply<<<nb(d.C), 256, 0, st>>>(d, type, in, out);
  return cudaGetLastError();
}
cudaError_t launch_pcg_dot(cudaStream_t st, int C, const double* a, const double* b, double* part, int nparts) {
  k_pcg_dot<<<nparts, 256, 0, st>>>(C, a, b, part);
  return cudaGetLastError();
}
cudaError_t launch_pcg_axpy(cudaStream_t st, int C, double alpha, const double* xv, double* yv) {
  k_pcg_axpy<<<nb(C), 256, 0, st>>>(C, alpha, xv, yv);
  return cudaGetLastError();
}
cudaError_t launch_pcg_precond(cudaStream_t st, const Dims& d, const int8_t* type, const double* r, double* z) {
  k_pcg_precond<<<nb(d.C), 256, 0, st>>>(d, type, r, z);
  return cudaGetLastError();
}
cudaError_t launch_pcg_xpby(cudaStream_t st, int C, const double* xv, double beta, double* yv) {
  k_pcg_xpby<<<nb(C), 256, 0, st>>>(C, xv, beta, yv);
  return cudaGetLastError();
}

}  // namespace aqb
