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

// Forward convolution variant: 2 = tcgen05 UMMA where its operands fit in
// shared memory, else halo-tiled mma.sync (default); 1 = halo-tiled
// mma.sync; 0 = im2col streaming mma.sync.
int g_conv_impl = 2;

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

// Halo-tiled forward: a CTA computes a 4 (x) x 4 (y) x 16 (z) block of
// output voxels.  The input block with its one-voxel halo (6 x 6 x 18
// voxels x CIN channels) is staged in shared memory once (cp.async, zero
// fill outside the grid); every tap then gathers its A fragments straight
// from that block with ldmatrix (each lane addresses its own voxel row), so
// the input is read ~2.5x instead of 27x.  Weights stream per tap, double
// buffered.  8 warps; m tile j = 16 z voxels at (x, y) = (j / 4, j % 4),
// warp w owns tiles 2w and 2w+1.  Rows are padded by 16 B (odd count of 16 B
// chunks: ldmatrix without bank conflicts).
constexpr int kTX = 4, kTY = 4, kTZ = 16;
constexpr int kHX = kTX + 2, kHY = kTY + 2, kHZ = kTZ + 2, kHalo = kHX * kHY * kHZ;

template <int CIN, int COUT>
constexpr size_t fwd_tile_smem() {
  return (size_t)kHalo * (CIN + 8) * sizeof(bf16) + (size_t)2 * COUT * (CIN + 8) * sizeof(bf16);
}

template <int CIN, int COUT, bool RELU, bool BIAS>
__global__ void __launch_bounds__(256) k_conv3_fwd_tile(const bf16* __restrict__ in, const bf16* __restrict__ w,
                                                       const float* __restrict__ bias, bf16* __restrict__ out,
                                                       int sx, int sy, int sz) {
  static_assert(CIN % 16 == 0 && COUT % 8 == 0, "channel counts");
  constexpr int RS = CIN + 8;  // row stride (bf16)
  constexpr int KS = CIN / 16, NT = COUT / 8, CH = CIN / 8;
  extern __shared__ __align__(16) unsigned char ft_smem[];
  bf16* sH = reinterpret_cast<bf16*>(ft_smem);
  bf16* sW = sH + kHalo * RS;  // [2][COUT][RS]
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int z0 = blockIdx.x * kTZ, y0 = blockIdx.y * kTY, x0 = blockIdx.z * kTX;
  // stage the halo block
  for (int i = tid; i < kHalo * CH; i += 256) {
    const int c = i % CH, h = i / CH;
    const int hz = h % kHZ, t = h / kHZ, hy = t % kHY, hx = t / kHY;
    const int gx = x0 + hx - 1, gy = y0 + hy - 1, gz = z0 + hz - 1;
    const bool ok = gx >= 0 && gx < sx && gy >= 0 && gy < sy && gz >= 0 && gz < sz;
    cp_async16(sH + h * RS + c * 8, ok ? in + ((size_t)((gx * sy + gy) * sz + gz) * CIN + c * 8) : in, ok);
  }
  auto stage_w = [&](int tap, int buf) {
    bf16* dst = sW + buf * COUT * RS;
    for (int i = tid; i < COUT * CH; i += 256) {
      const int c = i % CH, n = i / CH;
      cp_async16(dst + n * RS + c * 8, w + ((size_t)(tap * COUT + n) * CIN + c * 8), true);
    }
  };
  stage_w(0, 0);
  cp_async_commit();
  float acc[2][NT][4];
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int b = 0; b < NT; ++b)
#pragma unroll
      for (int c = 0; c < 4; ++c) acc[a][b][c] = 0.f;
  for (int tap = 0; tap < 27; ++tap) {
    const int buf = tap & 1;
    if (tap + 1 < 27) stage_w(tap + 1, buf ^ 1);
    cp_async_commit();
    cp_async_wait<1>();
    __syncthreads();
    int dx, dy, dz;
    tap_offset(tap, dx, dy, dz);
    const bf16* wb = sW + buf * COUT * RS;
#pragma unroll
    for (int ks = 0; ks < KS; ++ks) {
      unsigned bfr[NT][2];
#pragma unroll
      for (int nt = 0; nt < NT; ++nt) ldsm_x2(bfr[nt], wb + (nt * 8 + (lane & 7)) * RS + ks * 16 + ((lane >> 3) & 1) * 8);
#pragma unroll
      for (int mt = 0; mt < 2; ++mt) {
        const int j = warp * 2 + mt;
        const int ox = j >> 2, oy = j & 3;
        const int h = ((ox + dx + 1) * kHY + (oy + dy + 1)) * kHZ + (lane & 15) + dz + 1;
        unsigned afr[4];
        ldsm_x4(afr, sH + h * RS + ks * 16 + (lane >> 4) * 8);
#pragma unroll
        for (int nt = 0; nt < NT; ++nt) mma_bf16(acc[mt][nt], afr, bfr[nt]);
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int mt = 0; mt < 2; ++mt) {
    const int j = warp * 2 + mt;
    const int gx = x0 + (j >> 2), gy = y0 + (j & 3);
    if (gx >= sx || gy >= sy) continue;
#pragma unroll
    for (int nt = 0; nt < NT; ++nt) {
      const int co = nt * 8 + (lane & 3) * 2;
      const float b0 = BIAS ? bias[co] : 0.f, b1 = BIAS ? bias[co + 1] : 0.f;
#pragma unroll
      for (int hh = 0; hh < 2; ++hh) {
        const int gz = z0 + (lane >> 2) + hh * 8;
        if (gz < sz) {
          float a = acc[mt][nt][2 * hh] + b0, c = acc[mt][nt][2 * hh + 1] + b1;
          if (RELU) {
            a = fmaxf(a, 0.f);
            c = fmaxf(c, 0.f);
          }
          *reinterpret_cast<__nv_bfloat162*>(out + (size_t)((gx * sy + gy) * sz + gz) * COUT + co) =
              __floats2bfloat162_rn(a, c);
        }
      }
    }
  }
}

// ------------------------------------------------- forward on tcgen05 (TMEM)
// UMMA implicit GEMM: D[voxels x COUT] (f32, TMEM) += A[voxels x 16 channels]
// x B[16 channels x COUT] per tap and k step, bf16 operands in shared memory
// read through matrix descriptors (canonical K-major layout, no swizzle:
// 8-row x 16-byte core matrices), tcgen05.mma.cta_group::1.kind::f16 issued by
// one thread, completion through tcgen05.commit on an mbarrier whose wait is
// bounded (a timeout is recorded in g_umma_timeout; the kernel then frees its
// TMEM without storing), results read back with tcgen05.ld.
__device__ int g_umma_timeout;
// Test hook of the bounded wait: when set, the issuing thread neither issues
// the MMAs nor commits (nothing is left in flight), so every thread's wait
// runs out; g_umma_wait_ns bounds the wait (default one second).
__device__ int g_umma_test_skip;
__device__ unsigned long long g_umma_wait_ns = 1000000000ull;

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor: start, leading (K) and stride (M/N) byte
// offsets of the core matrices, the fixed version bits 46-47 = 1, no swizzle.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr & 0x3FFFFu) >> 4) | ((uint64_t)(lbo >> 4) << 16) | ((uint64_t)(sbo >> 4) << 32) |
         (1ull << 46);
}

// Instruction descriptor, kind::f16: D f32, A and B bf16, both K-major, N, M.
__host__ __device__ constexpr uint32_t umma_idesc(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void umma_f16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void umma_commit(uint64_t* mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(smem_u32(mbar))
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* mbar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n.reg .pred P1;\nmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\nselp.b32 %0, 1, 0, P1;\n}\n"
      : "=r"(done)
      : "r"(smem_u32(mbar)), "r"(parity)
      : "memory");
  return done != 0;
}

__device__ __forceinline__ unsigned long long umma_now_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Bounded wait on an mbarrier phase; false (and the timeout recorded) if it
// does not complete within g_umma_wait_ns or 2^22 polls, whichever is first.
__device__ __forceinline__ bool mbar_wait(uint64_t* mbar, uint32_t parity) {
  const unsigned long long t0 = umma_now_ns(), limit = g_umma_wait_ns;
  for (int i = 0; i < (1 << 22); ++i) {
    if (mbar_try_wait(mbar, parity)) return true;
    if ((i & 255) == 255 && umma_now_ns() - t0 > limit) break;
  }
  atomicExch(&g_umma_timeout, 1);
  return false;
}

// 16 consecutive f32 columns of this thread's TMEM lane (32x32b shape).
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__host__ __device__ constexpr int tmem_cols(int n) { return n <= 32 ? 32 : n <= 64 ? 64 : n <= 128 ? 128 : 256; }

// Output block of the tcgen05 kernel: 2 (x) x 16 (y) x 8 (z) voxels, two
// M = 128 tiles (one per x plane, row m = 8 y + z).  Its input halo
// (4 x 18 x 10 voxels) is stored per 8-channel chunk as z columns of 10 rows
// of 16 B: the A operand of any tap is then a descriptor into the halo
// itself — rows of a core matrix are 8 consecutive z (16 B apart), the 16
// core matrices along M are the y columns (SBO = 160 B), the two along K the
// chunk planes (LBO) — so no per-tap copy and no per-tap barrier: the CTA
// loads the halo and all 27 taps' weights, one thread issues every MMA and
// commits once.  On B200 the 128^3 network's inference takes 1.55 ms this
// way against 1.64 ms with k_conv3_fwd_tile; per layer it is ahead where
// COUT is 32 and behind at 128^3 with COUT = 16, whose N = 16 MMAs are too
// narrow to keep the tensor pipe busy.
constexpr int kUX = 2, kUY = 16, kUZ = 8;
constexpr int kUHX = kUX + 2, kUHY = kUY + 2, kUHZ = kUZ + 2;
constexpr int kUPlane = kUHX * kUHY * kUHZ * 16;  // bytes of one 8-channel chunk of the halo

template <int CIN, int COUT>
__host__ __device__ constexpr size_t fwd_umma_smem() {
  return (size_t)(CIN / 8) * kUPlane + (size_t)27 * COUT * CIN * 2 + 1024;
}

// The pairs the tcgen05 kernel takes: cout a multiple of 16 (UMMA N), the
// halo and all weights resident.
template <int CIN, int COUT>
__host__ __device__ constexpr bool umma_fits() {
  return COUT % 16 == 0 && COUT <= 128 && fwd_umma_smem<CIN, COUT>() <= 200 * 1024;
}

template <int CIN, int COUT, bool RELU, bool BIAS>
__global__ void __launch_bounds__(256) k_conv3_fwd_umma(const bf16* __restrict__ in, const bf16* __restrict__ w,
                                                       const float* __restrict__ bias, bf16* __restrict__ out,
                                                       int sx, int sy, int sz) {
  static_assert(umma_fits<CIN, COUT>(), "UMMA shapes: M = 128, N = COUT, operands resident");
  constexpr int CH = CIN / 8, KS = CIN / 16;
  constexpr int TAPB = COUT * CIN * 2;  // one tap's weights
  constexpr int COLS = tmem_cols(2 * COUT);
  constexpr uint32_t IDESC = umma_idesc(128, COUT);
  extern __shared__ __align__(1024) unsigned char um_smem[];
  unsigned char* sH = um_smem;                // [CH][kUHX][kUHY][kUHZ][16 B]
  unsigned char* sB = um_smem + CH * kUPlane;  // [27][canonical COUT x CIN]
  __shared__ __align__(8) uint64_t s_mbar;
  __shared__ uint32_t s_tmem;
  const int tid = threadIdx.x, warp = tid >> 5;
  const int z0 = blockIdx.x * kUZ, y0 = blockIdx.y * kUY, x0 = blockIdx.z * kUX;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(&s_tmem)),
                 "r"(COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(&s_mbar)), "r"(1));
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  // the halo: chunk c of voxel (hx, hy, hz), zero outside the grid
  for (int i = tid; i < kUHX * kUHY * kUHZ * CH; i += 256) {
    const int c = i % CH, h = i / CH;
    const int hz = h % kUHZ, t = h / kUHZ, hy = t % kUHY, hx = t / kUHY;
    const int gx = x0 + hx - 1, gy = y0 + hy - 1, gz = z0 + hz - 1;
    const bool ok = gx >= 0 && gx < sx && gy >= 0 && gy < sy && gz >= 0 && gz < sz;
    cp_async16(sH + c * kUPlane + h * 16, ok ? in + ((size_t)((gx * sy + gy) * sz + gz) * CIN + c * 8) : in, ok);
  }
  // all weights: tap t, row n, chunk c in the canonical K-major layout
  for (int i = tid; i < 27 * COUT * CH; i += 256) {
    const int c = i % CH, n = (i / CH) % COUT, t = i / (CH * COUT);
    cp_async16(sB + t * TAPB + (c >> 1) * (COUT * 32) + (n >> 3) * 256 + (c & 1) * 128 + (n & 7) * 16,
               w + ((size_t)(t * COUT + n) * CIN + c * 8), true);
  }
  cp_async_commit();
  cp_async_wait<0>();
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  const uint32_t tmem = s_tmem;
  if (tid == 0 && !g_umma_test_skip) {
    const uint32_t h0 = smem_u32(sH), b0 = smem_u32(sB);
    for (int tap = 0; tap < 27; ++tap) {
      int dx, dy, dz;
      tap_offset(tap, dx, dy, dz);
#pragma unroll
      for (int j = 0; j < kUX; ++j) {
        // tile j: output x plane j reads halo plane j + dx + 1, columns from dy + 1, rows from dz + 1
        const uint32_t a0 = h0 + (uint32_t)((((j + dx + 1) * kUHY + (dy + 1)) * kUHZ + (dz + 1)) * 16);
#pragma unroll
        for (int ks = 0; ks < KS; ++ks) {
          const uint64_t ad = umma_desc(a0 + (uint32_t)(2 * ks * kUPlane), kUPlane, kUHZ * 16);
          const uint64_t bd = umma_desc(b0 + (uint32_t)(tap * TAPB + ks * (COUT * 32)), 128, 256);
          umma_f16(tmem + (uint32_t)(j * COUT), ad, bd, IDESC, (tap > 0 || ks > 0) ? 1u : 0u);
        }
      }
    }
    umma_commit(&s_mbar);
  }
  const bool ok_wait = mbar_wait(&s_mbar, 0u);
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  // warp w reads TMEM lanes 32 (w % 4) .. of tile w / 4: its row m -> (y, z)
  const int j = warp >> 2, m = (warp & 3) * 32 + (tid & 31);
  const int gx = x0 + j, gy = y0 + (m >> 3), gz = z0 + (m & 7);
  const bool store = ok_wait && gx < sx && gy < sy && gz < sz;
  const uint32_t trow = tmem + ((uint32_t)((warp & 3) * 32) << 16) + (uint32_t)(j * COUT);
  bf16* dst = out + (size_t)((gx * sy + gy) * sz + gz) * COUT;
#pragma unroll
  for (int c0 = 0; c0 < COUT; c0 += 16) {
    float v[16];
    tmem_ld16(trow + (uint32_t)c0, v);
    if (store) {
      __align__(16) __nv_bfloat162 pk[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        float a = v[2 * q] + (BIAS ? bias[c0 + 2 * q] : 0.f), b = v[2 * q + 1] + (BIAS ? bias[c0 + 2 * q + 1] : 0.f);
        if (RELU) {
          a = fmaxf(a, 0.f);
          b = fmaxf(b, 0.f);
        }
        pk[q] = __floats2bfloat162_rn(a, b);
      }
      uint4* d4 = reinterpret_cast<uint4*>(dst + c0);
      d4[0] = reinterpret_cast<const uint4*>(pk)[0];
      d4[1] = reinterpret_cast<const uint4*>(pk)[1];
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(COLS));
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
  if constexpr (umma_fits<CIN, COUT>()) {
    if (g_conv_impl == 2) {
      constexpr size_t smem = fwd_umma_smem<CIN, COUT>();
      static const cudaError_t attr = cudaFuncSetAttribute(
          k_conv3_fwd_umma<CIN, COUT, RELU, BIAS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if (attr != cudaSuccess) return attr;
      const dim3 grid((sz + kUZ - 1) / kUZ, (sy + kUY - 1) / kUY, (sx + kUX - 1) / kUX);
      k_conv3_fwd_umma<CIN, COUT, RELU, BIAS><<<grid, 256, smem, st>>>(in, w, b, out, sx, sy, sz);
      return cudaGetLastError();
    }
  }
  if (g_conv_impl >= 1) {
    constexpr size_t smem = fwd_tile_smem<CIN, COUT>();
    static const cudaError_t attr =
        cudaFuncSetAttribute(k_conv3_fwd_tile<CIN, COUT, RELU, BIAS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem);
    if (attr != cudaSuccess) return attr;
    const dim3 grid((sz + kTZ - 1) / kTZ, (sy + kTY - 1) / kTY, (sx + kTX - 1) / kTX);
    k_conv3_fwd_tile<CIN, COUT, RELU, BIAS><<<grid, 256, smem, st>>>(in, w, b, out, sx, sy, sz);
    return cudaGetLastError();
  }
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

// ------------------------------------------------------------ U-Net glue
// Grid-stride elementwise kernels over channels-last tensors.  Fine grid
// (sx,sy,sz), coarse grid (sx/2,sy/2,sz/2); every size is even.

__device__ __forceinline__ int coarse_of(int v, int sx, int sy, int sz) {
  const int z = v % sz, t = v / sz, y = t % sy, x = t / sy;
  return (((x >> 1) * (sy >> 1) + (y >> 1)) * (sz >> 1)) + (z >> 1);
}

// max |a[i]| over i < n: per-block maxima, then one block (order-independent)
__global__ void k_absmax_part(const float* __restrict__ a, int n, float* __restrict__ part) {
  __shared__ float sm[256];
  float m = 0.f;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) m = fmaxf(m, fabsf(a[i]));
  sm[threadIdx.x] = m;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) sm[threadIdx.x] = fmaxf(sm[threadIdx.x], sm[threadIdx.x + o]);
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = sm[0];
}
__global__ void k_absmax_final(const float* __restrict__ part, int n, float* __restrict__ out) {
  __shared__ float sm[256];
  float m = 0.f;
  for (int i = threadIdx.x; i < n; i += blockDim.x) m = fmaxf(m, part[i]);
  sm[threadIdx.x] = m;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) sm[threadIdx.x] = fmaxf(sm[threadIdx.x], sm[threadIdx.x + o]);
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = sm[0];
}

// Network input, 16 channels: [rhs / max|rhs|, 1 on fluid cells (0 air), 0 x 14].
__global__ void k_unet_input(const float* __restrict__ rhs, const int8_t* __restrict__ type,
                             const float* __restrict__ scale, bf16* __restrict__ out, int V) {
  const float s = *scale;
  const float inv = s > 0.f ? 1.f / s : 0.f;
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
    __align__(16) bf16 row[16];
    row[0] = __float2bfloat16(rhs[v] * inv);
    row[1] = __float2bfloat16(type[v] == kFluid ? 1.f : 0.f);
#pragma unroll
    for (int c = 2; c < 16; ++c) row[c] = __float2bfloat16(0.f);
    uint4* dst = reinterpret_cast<uint4*>(out + (size_t)v * 16);
    dst[0] = reinterpret_cast<const uint4*>(row)[0];
    dst[1] = reinterpret_cast<const uint4*>(row)[1];
  }
}

// 2x2x2 average pooling: out (coarse) from in (fine), C channels.
__global__ void k_pool2(const bf16* __restrict__ in, bf16* __restrict__ out, int sx, int sy, int sz, int C) {
  const int cx = sx >> 1, cy = sy >> 1, cz = sz >> 1;
  const int n = cx * cy * cz * C;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int c = i % C, V = i / C;
    const int z = V % cz, t = V / cz, y = t % cy, x = t / cy;
    float acc = 0.f;
    for (int a = 0; a < 2; ++a)
      for (int b = 0; b < 2; ++b)
        for (int e = 0; e < 2; ++e)
          acc += __bfloat162float(in[((size_t)(((2 * x + a) * sy + 2 * y + b) * sz + 2 * z + e)) * C + c]);
    out[i] = __float2bfloat16(acc * 0.125f);
  }
}

// din (fine) = [din +] dout(coarse parent) / 8
__global__ void k_pool2_bwd(const bf16* __restrict__ dout, bf16* __restrict__ din, int sx, int sy, int sz, int C,
                            int accumulate) {
  const int n = sx * sy * sz * C;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int c = i % C, v = i / C;
    float g = __bfloat162float(dout[(size_t)coarse_of(v, sx, sy, sz) * C + c]) * 0.125f;
    if (accumulate) g += __bfloat162float(din[i]);
    din[i] = __float2bfloat16(g);
  }
}

// out (fine, Cu + Cs channels) = [coarse(parent) (Cu), skip (Cs)]
__global__ void k_upcat(const bf16* __restrict__ coarse, const bf16* __restrict__ skip, bf16* __restrict__ out,
                        int sx, int sy, int sz, int Cu, int Cs) {
  const int C = Cu + Cs;
  const int n = sx * sy * sz * C;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int c = i % C, v = i / C;
    out[i] = c < Cu ? coarse[(size_t)coarse_of(v, sx, sy, sz) * Cu + c] : skip[(size_t)v * Cs + (c - Cu)];
  }
}

// dskip = dout[:, Cu:]; dcoarse[P] = sum over the 8 children of dout[:, :Cu]
__global__ void k_upcat_bwd_skip(const bf16* __restrict__ dout, bf16* __restrict__ dskip, int V, int Cu, int Cs) {
  const int n = V * Cs;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int c = i % Cs, v = i / Cs;
    dskip[i] = dout[(size_t)v * (Cu + Cs) + Cu + c];
  }
}
__global__ void k_upcat_bwd_coarse(const bf16* __restrict__ dout, bf16* __restrict__ dcoarse, int sx, int sy, int sz,
                                   int Cu, int Cs) {
  const int cx = sx >> 1, cy = sy >> 1, cz = sz >> 1;
  const int n = cx * cy * cz * Cu;
  const int C = Cu + Cs;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int c = i % Cu, V = i / Cu;
    const int z = V % cz, t = V / cz, y = t % cy, x = t / cy;
    float acc = 0.f;
    for (int a = 0; a < 2; ++a)
      for (int b = 0; b < 2; ++b)
        for (int e = 0; e < 2; ++e)
          acc += __bfloat162float(dout[((size_t)(((2 * x + a) * sy + 2 * y + b) * sz + 2 * z + e)) * C + c]);
    dcoarse[i] = __float2bfloat16(acc);
  }
}

// dy = y > 0 ? dy : 0 (ReLU backward, y the layer's output)
__global__ void k_relu_bwd(bf16* __restrict__ dy, const bf16* __restrict__ y, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    if (!(__bfloat162float(y[i]) > 0.f)) dy[i] = __float2bfloat16(0.f);
}

// Per-block channel sums of dy (V x C) over `rows` consecutive voxels.
__global__ void k_chan_sum_part(const bf16* __restrict__ dy, int V, int C, int rows, float* __restrict__ part) {
  const int v0 = blockIdx.x * rows, v1 = min(V, v0 + rows);
  for (int c = threadIdx.x; c < C; c += blockDim.x) {
    float s = 0.f;
    for (int v = v0; v < v1; ++v) s += __bfloat162float(dy[(size_t)v * C + c]);
    part[(size_t)blockIdx.x * C + c] = s;
  }
}

// Output head: out[v] = b + sum_c w[c] h[v][c] (16 channels), f32
__global__ void k_head_fwd(const bf16* __restrict__ h, const float* __restrict__ w, const float* __restrict__ b,
                           float* __restrict__ out, int V) {
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
    float s = *b;
#pragma unroll
    for (int c = 0; c < 16; ++c) s += w[c] * __bfloat162float(h[(size_t)v * 16 + c]);
    out[v] = s;
  }
}

// Adam (bias-corrected) on n parameters; refreshes the bf16 copy if given.
__global__ void k_adam(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, int n, float lr, float b1, float b2, float eps, float c1, float c2,
                       bf16* __restrict__ wb) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    w[i] = wi;
    if (wb) wb[i] = __float2bfloat16(wi);
  }
}

__global__ void k_scale_copy(const float* __restrict__ a, float k, float* __restrict__ b, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) b[i] = a[i] * k;
}

__global__ void k_f32_to_bf16(const float* __restrict__ a, bf16* __restrict__ b, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) b[i] = __float2bfloat16(a[i]);
}

// Warm start: p = out * scale * out_scale on fluid cells, 0 elsewhere.
__global__ void k_unet_to_pressure(const float* __restrict__ out, const float* __restrict__ scale, float out_scale,
                                   const int8_t* __restrict__ type, float* __restrict__ p, int V) {
  const float s = *scale * out_scale;
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x)
    p[v] = type[v] == kFluid ? out[v] * s : 0.f;
}

// Dataset sample: rhs / scale, type, target p / scale.
__global__ void k_unet_sample(const float* __restrict__ rhs, const int8_t* __restrict__ type,
                              const double* __restrict__ p, const float* __restrict__ scale, float* __restrict__ rhs_s,
                              int8_t* __restrict__ type_s, float* __restrict__ target, int V) {
  const float s = *scale;
  const float inv = s > 0.f ? 1.f / s : 0.f;
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
    rhs_s[v] = rhs[v] * inv;
    type_s[v] = type[v];
    target[v] = type[v] == kFluid ? (float)p[v] * inv : 0.f;
  }
}

// ---------------------------------------------------------- training loss
// L = ||e||^2 / ||t||^2 + alpha ||A e||^2 / ||A t||^2 over fluid cells, e = o - t,
// with A the pressure operator the Jacobi sweeps solve ((A x)_i = 6 x_i - sum
// of the six neighbours, a neighbour outside the grid taking x_i, air 0).
// The second term is the prediction's relative residual: it penalises the
// rough error that Jacobi sweeps do not remove.

__device__ __forceinline__ void block_sum2(float a, float b, float* part) {
  __shared__ float sa[256], sb[256];
  sa[threadIdx.x] = a;
  sb[threadIdx.x] = b;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      sa[threadIdx.x] += sa[threadIdx.x + o];
      sb[threadIdx.x] += sb[threadIdx.x + o];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    part[blockIdx.x * 2] = sa[0];
    part[blockIdx.x * 2 + 1] = sb[0];
  }
}

// e = o - t on fluid cells (0 elsewhere); partial sums of e^2 and t^2.
__global__ void __launch_bounds__(256) k_loss_err(const float* __restrict__ o, const float* __restrict__ t,
                                                  const int8_t* __restrict__ type, float* __restrict__ e, int V,
                                                  float* __restrict__ part) {
  float se = 0.f, st = 0.f;
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
    const bool fl = type[v] == kFluid;
    const float ev = fl ? o[v] - t[v] : 0.f;
    e[v] = ev;
    se += ev * ev;
    st += fl ? t[v] * t[v] : 0.f;
  }
  block_sum2(se, st, part);
}

// y = A x on fluid cells (0 elsewhere); partial sums of y^2 (and 0).
__global__ void __launch_bounds__(256) k_apply_A(const float* __restrict__ x, const int8_t* __restrict__ type,
                                                 float* __restrict__ y, int sx, int sy, int sz,
                                                 float* __restrict__ part) {
  float sq = 0.f;
  const int V = sx * sy * sz;
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
    float r = 0.f;
    if (type[v] == kFluid) {
      const int z = v % sz, tt = v / sz, yy = tt % sy, xx = tt / sy;
      const float c = x[v];
      float s = xx + 1 < sx ? x[v + sy * sz] : c;
      s += xx > 0 ? x[v - sy * sz] : c;
      s += yy + 1 < sy ? x[v + sz] : c;
      s += yy > 0 ? x[v - sz] : c;
      s += z + 1 < sz ? x[v + 1] : c;
      s += z > 0 ? x[v - 1] : c;
      r = 6.f * c - s;
    }
    y[v] = r;
    sq += r * r;
  }
  block_sum2(sq, 0.f, part);
}

// y = J x on fluid cells (0 elsewhere): one homogeneous Jacobi sweep, the
// mean of the six neighbours (a neighbour outside the grid taking x_i).
// J is symmetric, so it is its own adjoint in the gradient.
__global__ void __launch_bounds__(256) k_apply_J(const float* __restrict__ x, const int8_t* __restrict__ type,
                                                 float* __restrict__ y, int sx, int sy, int sz) {
  const int V = sx * sy * sz;
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
    float r = 0.f;
    if (type[v] == kFluid) {
      const int z = v % sz, tt = v / sz, yy = tt % sy, xx = tt / sy;
      const float c = x[v];
      float s = xx + 1 < sx ? x[v + sy * sz] : c;
      s += xx > 0 ? x[v - sy * sz] : c;
      s += yy + 1 < sy ? x[v + sz] : c;
      s += yy > 0 ? x[v - sz] : c;
      s += z + 1 < sz ? x[v + 1] : c;
      s += z > 0 ? x[v - 1] : c;
      r = s * (1.f / 6.f);
    }
    y[v] = r;
  }
}

// g = 2 e / ||t||^2 + 2 alpha q / ||A t||^2 on fluid cells (q = A A e);
// sums = [||e||^2, ||t||^2, ||Ae||^2, ||At||^2]; loss written to *loss.
__global__ void k_loss_grad(const float* __restrict__ e, const float* __restrict__ q, const int8_t* __restrict__ type,
                            const float* __restrict__ sums, float alpha, float* __restrict__ g, int V,
                            float* __restrict__ loss) {
  const float st = fmaxf(sums[1], 1e-30f), sat = fmaxf(sums[3], 1e-30f);
  const float a = 2.f / st, c = 2.f * alpha / sat;
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x)
    g[v] = type[v] == kFluid ? a * e[v] + c * q[v] : 0.f;
  if (blockIdx.x == 0 && threadIdx.x == 0) *loss = sums[0] / st + alpha * sums[2] / sat;
}

// Head backward from the output gradient g: dh[v][c] = g_v w[c]; per-block
// partial sums of g_v h[v][c] (16) and g_v.
__global__ void __launch_bounds__(256) k_head_bwd(const float* __restrict__ g, const bf16* __restrict__ h,
                                                  const float* __restrict__ w, bf16* __restrict__ dh, int V,
                                                  float* __restrict__ part) {
  __shared__ float sm[17][256];
  float acc[17];
#pragma unroll
  for (int k = 0; k < 17; ++k) acc[k] = 0.f;
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
    const float gv = g[v];
#pragma unroll
    for (int c = 0; c < 16; ++c) {
      acc[c] += gv * __bfloat162float(h[(size_t)v * 16 + c]);
      dh[(size_t)v * 16 + c] = __float2bfloat16(gv * w[c]);
    }
    acc[16] += gv;
  }
#pragma unroll
  for (int k = 0; k < 17; ++k) sm[k][threadIdx.x] = acc[k];
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o)
#pragma unroll
      for (int k = 0; k < 17; ++k) sm[k][threadIdx.x] += sm[k][threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x < 17) part[(size_t)blockIdx.x * 17 + threadIdx.x] = sm[threadIdx.x][0];
}

inline int ew_grid(long long n) {
  const long long b = (n + 255) / 256;
  return (int)std::min<long long>(std::max<long long>(b, 1), 148 * 16);
}

}  // namespace

void set_conv_impl(int impl) { g_conv_impl = impl; }

int conv_umma_timeouts() {
  int v = 0;
  cudaMemcpyFromSymbol(&v, g_umma_timeout, sizeof(int));
  return v;
}

cudaError_t conv_umma_test_hook(int skip, unsigned long long wait_ns) {
  const int zero = 0;
  const unsigned long long ns = wait_ns ? wait_ns : 1000000000ull;
  cudaError_t e = cudaMemcpyToSymbol(g_umma_test_skip, &skip, sizeof(int));
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(g_umma_wait_ns, &ns, sizeof(ns));
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(g_umma_timeout, &zero, sizeof(int));
  return e;
}

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

namespace aqb {

cudaError_t launch_absmax(cudaStream_t st, const float* a, int n, float* part /*>= 1024*/, float* out) {
  const int g = std::min(1024, std::max(1, (n + 255) / 256));
  k_absmax_part<<<g, 256, 0, st>>>(a, n, part);
  k_absmax_final<<<1, 256, 0, st>>>(part, g, out);
  return cudaGetLastError();
}
cudaError_t launch_unet_input(cudaStream_t st, const float* rhs, const int8_t* type, const float* scale, void* out,
                              int V) {
  k_unet_input<<<ew_grid(V), 256, 0, st>>>(rhs, type, scale, (bf16*)out, V);
  return cudaGetLastError();
}
cudaError_t launch_pool2(cudaStream_t st, const void* in, void* out, int sx, int sy, int sz, int C) {
  k_pool2<<<ew_grid((long long)sx * sy * sz * C / 8), 256, 0, st>>>((const bf16*)in, (bf16*)out, sx, sy, sz, C);
  return cudaGetLastError();
}
cudaError_t launch_pool2_bwd(cudaStream_t st, const void* dout, void* din, int sx, int sy, int sz, int C,
                             bool accumulate) {
  k_pool2_bwd<<<ew_grid((long long)sx * sy * sz * C), 256, 0, st>>>((const bf16*)dout, (bf16*)din, sx, sy, sz, C,
                                                                    accumulate ? 1 : 0);
  return cudaGetLastError();
}
cudaError_t launch_upcat(cudaStream_t st, const void* coarse, const void* skip, void* out, int sx, int sy, int sz,
                         int Cu, int Cs) {
  k_upcat<<<ew_grid((long long)sx * sy * sz * (Cu + Cs)), 256, 0, st>>>((const bf16*)coarse, (const bf16*)skip,
                                                                        (bf16*)out, sx, sy, sz, Cu, Cs);
  return cudaGetLastError();
}
cudaError_t launch_upcat_bwd(cudaStream_t st, const void* dout, void* dcoarse, void* dskip, int sx, int sy, int sz,
                             int Cu, int Cs) {
  const int V = sx * sy * sz;
  k_upcat_bwd_skip<<<ew_grid((long long)V * Cs), 256, 0, st>>>((const bf16*)dout, (bf16*)dskip, V, Cu, Cs);
  k_upcat_bwd_coarse<<<ew_grid((long long)V / 8 * Cu), 256, 0, st>>>((const bf16*)dout, (bf16*)dcoarse, sx, sy, sz,
                                                                     Cu, Cs);
  return cudaGetLastError();
}
cudaError_t launch_relu_bwd(cudaStream_t st, void* dy, const void* y, int n) {
  k_relu_bwd<<<ew_grid(n), 256, 0, st>>>((bf16*)dy, (const bf16*)y, n);
  return cudaGetLastError();
}
int chan_sum_parts(int V) { return std::min(1024, std::max(1, (V + 255) / 256)); }
cudaError_t launch_chan_sum(cudaStream_t st, const void* dy, int V, int C, float* part, float* out) {
  const int np = chan_sum_parts(V);
  const int rows = (V + np - 1) / np;
  k_chan_sum_part<<<np, 64, 0, st>>>((const bf16*)dy, V, C, rows, part);
  k_sum_parts<<<(C + 255) / 256, 256, 0, st>>>(part, np, C, out);
  return cudaGetLastError();
}
cudaError_t launch_head_fwd(cudaStream_t st, const void* h, const float* w, const float* b, float* out, int V) {
  k_head_fwd<<<ew_grid(V), 256, 0, st>>>((const bf16*)h, w, b, out, V);
  return cudaGetLastError();
}
cudaError_t launch_adam(cudaStream_t st, float* w, const float* g, float* m, float* v, int n, float lr, float b1,
                        float b2, float eps, int t, void* wb) {
  const float c1 = 1.f - powf(b1, (float)t), c2 = 1.f - powf(b2, (float)t);
  k_adam<<<ew_grid(n), 256, 0, st>>>(w, g, m, v, n, lr, b1, b2, eps, c1, c2, (bf16*)wb);
  return cudaGetLastError();
}
cudaError_t launch_f32_to_bf16(cudaStream_t st, const float* a, void* b, int n) {
  k_f32_to_bf16<<<ew_grid(n), 256, 0, st>>>(a, (bf16*)b, n);
  return cudaGetLastError();
}
cudaError_t launch_unet_to_pressure(cudaStream_t st, const float* out, const float* scale, float out_scale,
                                    const int8_t* type, float* p, int V) {
  k_unet_to_pressure<<<ew_grid(V), 256, 0, st>>>(out, scale, out_scale, type, p, V);
  return cudaGetLastError();
}
cudaError_t launch_unet_scale_copy(cudaStream_t st, const float* a, float k, float* b, int n) {
  k_scale_copy<<<ew_grid(n), 256, 0, st>>>(a, k, b, n);
  return cudaGetLastError();
}
cudaError_t launch_unet_sample(cudaStream_t st, const float* rhs, const int8_t* type, const double* p,
                               const float* scale, float* rhs_s, int8_t* type_s, float* target, int V) {
  k_unet_sample<<<ew_grid(V), 256, 0, st>>>(rhs, type, p, scale, rhs_s, type_s, target, V);
  return cudaGetLastError();
}

}  // namespace aqb

namespace aqb {

int loss_parts() { return 296; }

// L = ||e||^2/||t||^2 + alpha ||A J^k e||^2 / ||A J^k t||^2: the second term is
// (residual after k Jacobi sweeps from the prediction / the same from zero)^2.
// Scratch: e, p0..p3, g (V floats each), part (loss_parts() * 8), sums (6).
cudaError_t launch_unet_loss_bwd(cudaStream_t st, const float* out, const float* target, const int8_t* type,
                                 const void* h, const float* w, float alpha, int k, void* dh, int sx, int sy, int sz,
                                 float* e, float* p0, float* p1, float* p2, float* p3, float* g, float* part,
                                 float* sums, float* head_part, float* head_sums /* 18: dw 16, db, loss */) {
  const int V = sx * sy * sz;
  const int P = loss_parts();
  // J^k x into p0/p1; returns the buffer holding the result
  auto smooth = [&](const float* x, float* a, float* b) -> const float* {
    const float* src = x;
    float* bufs[2] = {a, b};
    for (int i = 0; i < k; ++i) {
      k_apply_J<<<P, 256, 0, st>>>(src, type, bufs[i % 2], sx, sy, sz);
      src = bufs[i % 2];
    }
    return src;
  };
  k_loss_err<<<P, 256, 0, st>>>(out, target, type, e, V, part);
  const float* je = smooth(e, p0, p1);
  k_apply_A<<<P, 256, 0, st>>>(je, type, p2, sx, sy, sz, part + 2 * P);  // r = A J^k e
  const float* jt = smooth(target, p0, p1);
  k_apply_A<<<P, 256, 0, st>>>(jt, type, p3, sx, sy, sz, part + 4 * P);  // A J^k t (sum only)
  k_apply_A<<<P, 256, 0, st>>>(p2, type, p3, sx, sy, sz, part + 6 * P);  // q = A r
  const float* v = smooth(p3, p0, p1);                                    // J^k q
  k_sum_parts<<<1, 32, 0, st>>>(part, P, 2, sums);
  k_sum_parts<<<1, 32, 0, st>>>(part + 2 * P, P, 2, sums + 2);
  k_sum_parts<<<1, 32, 0, st>>>(part + 4 * P, P, 2, sums + 4);
  cudaError_t err = cudaMemcpyAsync(sums + 3, sums + 4, sizeof(float), cudaMemcpyDeviceToDevice, st);
  if (err != cudaSuccess) return err;
  k_loss_grad<<<ew_grid(V), 256, 0, st>>>(e, v, type, sums, alpha, g, V, head_sums + 17);
  k_head_bwd<<<P, 256, 0, st>>>(g, (const bf16*)h, w, (bf16*)dh, V, head_part);
  k_sum_parts<<<1, 32, 0, st>>>(head_part, P, 17, head_sums);
  return cudaGetLastError();
}

}  // namespace aqb
