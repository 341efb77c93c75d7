// Kernels of the learned pressure warm start: a small 3D U-Net in BF16 with
// FP32 accumulation.  No counterpart in the reference.
//
// Activations are channels-last over the cell layout: element (x,y,z,c) of a
// grid s = (sx,sy,sz) with C channels is at ((x*sy + y)*sz + z)*C + c.
// Convolutions are 3x3x3, stride 1, zero padding 1, as implicit GEMMs on the
// tensor cores (mma.sync m16n8k16, bf16 x bf16 -> f32):
//   forward   out[v][co] = act(b[co] + sum_t sum_ci in[v + o_t][ci] w[t][co][ci])
//             M = voxels, N = Cout, K = 27 taps x Cin; operands staged in shared
//             memory by cp.async (zero fill outside the grid), fragments by ldmatrix.
//   data grad the forward kernel on dY with the flipped, transposed weights
//             w'[t][ci][co] = w[26-t][co][ci].
//   weight grad dw[t][co][ci] = sum_v dY[v][co] x[v + o_t][ci]: M = Cout, N = Cin,
//             K = voxels, per (tap, voxel chunk) partial sums reduced in a fixed
//             order (deterministic).
// Tap t = (dx+1)*9 + (dy+1)*3 + (dz+1).
#include <cuda_bf16.h>

#include <algorithm>

#include "aq_kernels.cuh"

namespace aqb {
namespace {

using bf16 = __nv_bfloat16;

constexpr int kTileM = 128;  // voxels per forward CTA (4 warps x 32)
constexpr int kRowK = 24;    // smem row of one 16-wide k chunk: 16 + 8 pad bf16 (48 B, conflict-free ldmatrix)

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, bool pred) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  const int n = pred ? 16 : 0;  // n = 0: no bytes read, 16 zero bytes written
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(n));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

__device__ __forceinline__ void ldsm_x4(unsigned (&r)[4], const void* p) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(p);
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(s));
}
__device__ __forceinline__ void ldsm_x2(unsigned (&r)[2], const void* p) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(p);
  asm volatile("ldmatrix.sync.aligned.m8n8.x2.shared.b16 {%0,%1}, [%2];\n" : "=r"(r[0]), "=r"(r[1]) : "r"(s));
}
__device__ __forceinline__ void ldsm_x4_t(unsigned (&r)[4], const void* p) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(p);
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(s));
}
__device__ __forceinline__ void ldsm_x2_t(unsigned (&r)[2], const void* p) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(p);
  asm volatile("ldmatrix.sync.aligned.m8n8.x2.trans.shared.b16 {%0,%1}, [%2];\n" : "=r"(r[0]), "=r"(r[1]) : "r"(s));
}

// d += a * b, m16n8k16, bf16 inputs, f32 accumulators
__device__ __forceinline__ void mma_bf16(float (&d)[4], const unsigned (&a)[4], const unsigned (&b)[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

__device__ __forceinline__ void tap_offset(int tap, int& dx, int& dy, int& dz) {
  dx = tap / 9 - 1;
  dy = (tap / 3) % 3 - 1;
  dz = tap % 3 - 1;
}

// ------------------------------------------------------------------ forward
// 128 threads; CTA = 128 consecutive voxels x all COUT channels; warp w owns
// voxels [32w, 32w+32) as two m16 tiles.  K steps: 27 taps x CIN/16 chunks,
// double-buffered in shared memory.
template <int CIN, int COUT, bool RELU, bool BIAS>
__global__ void __launch_bounds__(128) k_conv3_fwd(const bf16* __restrict__ in, const bf16* __restrict__ w,
                                                  const float* __restrict__ bias, bf16* __restrict__ out, int sx,
                                                  int sy, int sz) {
  static_assert(CIN % 16 == 0 && COUT % 8 == 0, "channel counts");
  constexpr int KC = CIN / 16;
  constexpr int STEPS = 27 * KC;
  constexpr int NT = COUT / 8;
  __shared__ __align__(16) bf16 sA[2][kTileM * kRowK];
  __shared__ __align__(16) bf16 sB[2][COUT * kRowK];
  const int V = sx * sy * sz;
  const int m0 = blockIdx.x * kTileM;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int v = m0 + tid;  // the A row this thread stages
  const bool vin = v < V;
  int vx = 0, vy = 0, vz = 0;
  if (vin) {
    vz = v % sz;
    const int t = v / sz;
    vy = t % sy;
    vx = t / sy;
  }
  auto stage = [&](int step, int buf) {
    const int tap = step / KC, kc = step % KC;
    int dx, dy, dz;
    tap_offset(tap, dx, dy, dz);
    const int nx = vx + dx, ny = vy + dy, nz = vz + dz;
    const bool ok = vin && nx >= 0 && nx < sx && ny >= 0 && ny < sy && nz >= 0 && nz < sz;
    const bf16* src = ok ? in + ((size_t)((nx * sy + ny) * sz + nz) * CIN + kc * 16) : in;
    bf16* dst = &sA[buf][tid * kRowK];
    cp_async16(dst, src, ok);
    cp_async16(dst + 8, ok ? src + 8 : in, ok);
    for (int i = tid; i < COUT * 2; i += 128) {
      const int n = i >> 1, h = i & 1;
      cp_async16(&sB[buf][n * kRowK + h * 8], w + ((size_t)(tap * COUT + n) * CIN + kc * 16 + h * 8), true);
    }
  };
  float acc[2][NT][4];
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int b = 0; b < NT; ++b)
#pragma unroll
      for (int c = 0; c < 4; ++c) acc[a][b][c] = 0.f;
  stage(0, 0);
  cp_async_commit();
  for (int step = 0; step < STEPS; ++step) {
    const int buf = step & 1;
    if (step + 1 < STEPS) stage(step + 1, buf ^ 1);
    cp_async_commit();
    cp_async_wait<1>();
    __syncthreads();
    unsigned bfr[NT][2];
#pragma unroll
    for (int nt = 0; nt < NT; ++nt) ldsm_x2(bfr[nt], &sB[buf][(nt * 8 + (lane & 7)) * kRowK + ((lane >> 3) & 1) * 8]);
#pragma unroll
    for (int mt = 0; mt < 2; ++mt) {
      unsigned afr[4];
      ldsm_x4(afr, &sA[buf][(warp * 32 + mt * 16 + (lane & 15)) * kRowK + (lane >> 4) * 8]);
#pragma unroll
      for (int nt = 0; nt < NT; ++nt) mma_bf16(acc[mt][nt], afr, bfr[nt]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int mt = 0; mt < 2; ++mt)
#pragma unroll
    for (int nt = 0; nt < NT; ++nt) {
      const int co = nt * 8 + (lane & 3) * 2;
      const float b0 = BIAS ? bias[co] : 0.f, b1 = BIAS ? bias[co + 1] : 0.f;
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int r = m0 + warp * 32 + mt * 16 + (lane >> 2) + h * 8;
        if (r < V) {
          float a = acc[mt][nt][2 * h] + b0, c = acc[mt][nt][2 * h + 1] + b1;
          if (RELU) {
            a = fmaxf(a, 0.f);
            c = fmaxf(c, 0.f);
          }
          *reinterpret_cast<__nv_bfloat162*>(out + (size_t)r * COUT + co) = __floats2bfloat162_rn(a, c);
        }
      }
    }
}

// ------------------------------------------------------------- weight grad
// grid (chunks, 27): one tap, `cv` voxels per CTA in tiles of 128.  A = dY^T
// (COUT x voxels), B = x shifted by the tap (voxels x CIN); both staged with
// voxels as rows and read transposed by ldmatrix.trans.  Warp w owns the
// n tiles nt = w, w+4, ...
template <int CIN, int COUT>
__global__ void __launch_bounds__(128) k_conv3_wgrad(const bf16* __restrict__ x, const bf16* __restrict__ dy,
                                                    float* __restrict__ part, int sx, int sy, int sz, int cv) {
  static_assert(CIN % 16 == 0 && COUT % 16 == 0, "channel counts");
  constexpr int RX = CIN + 8, RD = COUT + 8;  // padded smem rows (odd count of 16 B chunks)
  constexpr int MT = COUT / 16, NTT = CIN / 8, NTW = (NTT + 3) / 4;
  extern __shared__ __align__(16) unsigned char wg_smem[];
  bf16(*sX)[kTileM * RX] = reinterpret_cast<bf16(*)[kTileM * RX]>(wg_smem);
  bf16(*sD)[kTileM * RD] = reinterpret_cast<bf16(*)[kTileM * RD]>(wg_smem + 2 * kTileM * RX * sizeof(bf16));
  const int V = sx * sy * sz;
  const int tap = blockIdx.y;
  int dx, dy_, dz;
  tap_offset(tap, dx, dy_, dz);
  const int v0 = blockIdx.x * cv, v1 = min(V, v0 + cv);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int tiles = (v1 - v0 + kTileM - 1) / kTileM;
  auto stage = [&](int tile, int buf) {
    const int base = v0 + tile * kTileM;
    // x rows: CIN/8 chunks each
    for (int i = tid; i < kTileM * (CIN / 8); i += 128) {
      const int r = i / (CIN / 8), c = i % (CIN / 8);
      const int v = base + r;
      bool ok = v < v1;
      const bf16* src = x;
      if (ok) {
        const int vz = v % sz, t = v / sz, vy = t % sy, vx = t / sy;
        const int nx = vx + dx, ny = vy + dy_, nz = vz + dz;
        ok = nx >= 0 && nx < sx && ny >= 0 && ny < sy && nz >= 0 && nz < sz;
        if (ok) src = x + ((size_t)((nx * sy + ny) * sz + nz) * CIN + c * 8);
      }
      cp_async16(&sX[buf][r * RX + c * 8], src, ok);
    }
    for (int i = tid; i < kTileM * (COUT / 8); i += 128) {
      const int r = i / (COUT / 8), c = i % (COUT / 8);
      const int v = base + r;
      const bool ok = v < v1;
      cp_async16(&sD[buf][r * RD + c * 8], ok ? dy + ((size_t)v * COUT + c * 8) : dy, ok);
    }
  };
  float acc[MT][NTW][4];
#pragma unroll
  for (int a = 0; a < MT; ++a)
#pragma unroll
    for (int b = 0; b < NTW; ++b)
#pragma unroll
      for (int c = 0; c < 4; ++c) acc[a][b][c] = 0.f;
  if (tiles > 0) stage(0, 0);
  cp_async_commit();
  for (int tile = 0; tile < tiles; ++tile) {
    const int buf = tile & 1;
    if (tile + 1 < tiles) stage(tile + 1, buf ^ 1);
    cp_async_commit();
    cp_async_wait<1>();
    __syncthreads();
#pragma unroll
    for (int k0 = 0; k0 < kTileM; k0 += 16) {
      unsigned afr[MT][4];
#pragma unroll
      for (int mt = 0; mt < MT; ++mt)
        ldsm_x4_t(afr[mt], &sD[buf][(k0 + (lane & 7) + (lane >> 4) * 8) * RD + mt * 16 + ((lane >> 3) & 1) * 8]);
#pragma unroll
      for (int j = 0; j < NTW; ++j) {
        const int nt = warp + 4 * j;
        if (nt < NTT) {
          unsigned bfr[2];
          ldsm_x2_t(bfr, &sX[buf][(k0 + (lane & 15)) * RX + nt * 8]);
#pragma unroll
          for (int mt = 0; mt < MT; ++mt) mma_bf16(acc[mt][j], afr[mt], bfr);
        }
      }
    }
    __syncthreads();
  }
  float* dst = part + ((size_t)blockIdx.x * 27 + tap) * COUT * CIN;
#pragma unroll
  for (int mt = 0; mt < MT; ++mt)
#pragma unroll
    for (int j = 0; j < NTW; ++j) {
      const int nt = warp + 4 * j;
      if (nt < NTT) {
        const int ci = nt * 8 + (lane & 3) * 2;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int co = mt * 16 + (lane >> 2) + h * 8;
          dst[co * CIN + ci] = acc[mt][j][2 * h];
          dst[co * CIN + ci + 1] = acc[mt][j][2 * h + 1];
        }
      }
    }
}

// dst[i] = sum over k of part[k*n + i], k ascending
__global__ void k_sum_parts(const float* __restrict__ part, int nparts, int n, float* __restrict__ dst) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float s = 0.f;
    for (int k = 0; k < nparts; ++k) s += part[(size_t)k * n + i];
    dst[i] = s;
  }
}

// w'[t][ci][co] = w[26-t][co][ci]
__global__ void k_flip_transpose(const bf16* __restrict__ w, bf16* __restrict__ wt, int cin, int cout) {
  const int n = 27 * cin * cout;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int co = i % cout, t = i / cout, ci = t % cin, tap = t / cin;
    wt[i] = w[((size_t)(26 - tap) * cout + co) * cin + ci];
  }
}

template <int CIN, int COUT, bool RELU, bool BIAS>
cudaError_t fwd_launch(cudaStream_t st, const bf16* in, const bf16* w, const float* b, bf16* out, int sx, int sy,
                       int sz) {
  const int V = sx * sy * sz;
  k_conv3_fwd<CIN, COUT, RELU, BIAS><<<(V + kTileM - 1) / kTileM, 128, 0, st>>>(in, w, b, out, sx, sy, sz);
  return cudaGetLastError();
}

template <int CIN, int COUT, bool RELU>
cudaError_t fwd_bias(cudaStream_t st, bool has_bias, const bf16* in, const bf16* w, const float* b, bf16* out, int sx,
                     int sy, int sz) {
  return has_bias ? fwd_launch<CIN, COUT, RELU, true>(st, in, w, b, out, sx, sy, sz)
                  : fwd_launch<CIN, COUT, RELU, false>(st, in, w, b, out, sx, sy, sz);
}

template <int CIN, int COUT>
cudaError_t fwd_relu(cudaStream_t st, bool relu, bool has_bias, const bf16* in, const bf16* w, const float* b,
                     bf16* out, int sx, int sy, int sz) {
  return relu ? fwd_bias<CIN, COUT, true>(st, has_bias, in, w, b, out, sx, sy, sz)
              : fwd_bias<CIN, COUT, false>(st, has_bias, in, w, b, out, sx, sy, sz);
}

}  // namespace

int unet_wgrad_chunk(int voxels) {
  // about 2 CTAs per SM per tap at 128^3, at least one 128-voxel tile
  const int target = std::max(1, voxels / 512);
  return std::max(kTileM, (target + kTileM - 1) / kTileM * kTileM);
}

// Channel pairs the kernels are instantiated for (the U-Net's layers and
// their data-gradient transposes).
#define AQ_CONV_LAYERS(X) X(16, 16) X(16, 32) X(32, 32) X(32, 64) X(64, 64) X(96, 32) X(48, 16)
#define AQ_CONV_PAIRS(X) AQ_CONV_LAYERS(X) X(32, 16) X(64, 32) X(32, 96) X(16, 48)

template <int CIN, int COUT>
constexpr size_t wgrad_smem() {
  return (size_t)2 * kTileM * ((CIN + 8) + (COUT + 8)) * sizeof(bf16);
}

cudaError_t launch_conv3_fwd(cudaStream_t st, int cin, int cout, bool relu, const void* in, const void* w,
                             const float* bias, void* out, int sx, int sy, int sz) {
  const bf16* i = (const bf16*)in;
  const bf16* ww = (const bf16*)w;
  bf16* o = (bf16*)out;
#define X(A, B) \
  if (cin == A && cout == B) return fwd_relu<A, B>(st, relu, bias != nullptr, i, ww, bias, o, sx, sy, sz);
  AQ_CONV_PAIRS(X)
#undef X
  return cudaErrorInvalidValue;
}

cudaError_t launch_conv3_wgrad(cudaStream_t st, int cin, int cout, const void* x, const void* dy, float* part,
                               float* dw, int sx, int sy, int sz) {
  const int V = sx * sy * sz;
  const int cv = unet_wgrad_chunk(V);
  const int chunks = (V + cv - 1) / cv;
  const dim3 grid(chunks, 27);
  bool done = false;
#define X(A, B)                                                                                   \
  if (!done && cin == A && cout == B) {                                                           \
    static const cudaError_t attr = cudaFuncSetAttribute(                                         \
        k_conv3_wgrad<A, B>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)wgrad_smem<A, B>()); \
    if (attr != cudaSuccess) return attr;                                                         \
    k_conv3_wgrad<A, B><<<grid, 128, wgrad_smem<A, B>(), st>>>((const bf16*)x, (const bf16*)dy, part, sx, sy, \
                                                             sz, cv);                             \
    done = true;                                                                                  \
  }
  AQ_CONV_LAYERS(X)
#undef X
  if (!done) return cudaErrorInvalidValue;
  const int n = 27 * cin * cout;
  k_sum_parts<<<(n + 255) / 256, 256, 0, st>>>(part, chunks, n, dw);
  return cudaGetLastError();
}

size_t conv3_wgrad_part_floats(int cin, int cout, int voxels) {
  const int cv = unet_wgrad_chunk(voxels);
  return (size_t)((voxels + cv - 1) / cv) * 27 * cin * cout;
}

cudaError_t launch_flip_transpose(cudaStream_t st, const void* w, void* wt, int cin, int cout) {
  const int n = 27 * cin * cout;
  k_flip_transpose<<<(n + 255) / 256, 256, 0, st>>>((const bf16*)w, (bf16*)wt, cin, cout);
  return cudaGetLastError();
}

}  // namespace aqb
