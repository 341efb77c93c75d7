// Resident Jacobi pressure solve (stage (c), hot loop #1): the whole solve in
// one cooperative launch whose CTAs keep their tiles' pressure in shared
// memory and right-hand side in registers from the first sweep to the last,
// and exchange only tile halos through L2, once every K = 4 sweeps.
//
// Reference: jacobiImpl (Fluid/Fluid_3D_kernels.cu:460-505), launched
// pressureIterations times by solvePressureJacobi (Fluid/Fluid_3D_common.cu:48-55).
// Per fluid cell
//   p' = (p[x+1] + p[x-1] + p[y+1] + p[y-1] + p[z+1] + p[z-1] + rhs) / 6,
// summed in that order, 0 on non-fluid cells, out-of-domain neighbours
// clamped to the cell itself: the arithmetic of every other sweep kernel of
// the library (jacobi_quad), so the iterates are bit for bit the flat sweep's.
//
// Decomposition.  The grid is cut into tiles of TX x TY x 24 cells (whole 8^3
// activity bricks); a tile takes part when one of its bricks holds fluid
// (cells outside every such tile are non-fluid, 0 in both global buffers,
// and stay 0).  A CTA owns one tile and holds its box, the tile plus a 4-cell
// halo clipped to the domain (at most (TX+8) x (TY+8) x 32 cells), in two
// shared-memory pressure buffers (ping-pong per sweep).  A block of 4 sweeps
// runs on the box with redundant halo work: sweep s updates the cells at
// least s cells inside every face of the box that is not a domain wall, so
// after 4 sweeps the tile's own cells hold exactly what 4 global sweeps give.
// The tile then writes its cells to the global buffer of the block, every
// CTA meets at a bounded grid barrier, and each reloads its box with one TMA
// tensor copy (cp.async.bulk.tensor, the tile's own cells come back
// unchanged; a bounded mbarrier wait).  The
// two global buffers alternate between blocks, so a CTA never overwrites
// cells a slower neighbour may still be reading.  When the active tiles
// outnumber the CTAs, each CTA walks its tiles one after another per block
// and reloads each whole box from L2 (same results, not resident).
//
// Threads.  One per (XS-level x segment, y row, z-quad) of the box (XS = 8,
// 12 or 16 per shape: fewer threads with more registers each, so the rhs of
// every level stays in registers without spills); a warp is 4 whole y rows
// of 8 quads.  A thread keeps the rhs and fluid marks of its XS quads in
// registers and walks its segment in x with a 3-quad window (x-1, x, x+1),
// so a quad costs one shared load for x+1, one each for y+1 and y-1
// (consecutive quads of consecutive rows: conflict-free 16-byte loads), and
// two shuffles for z+1 and z-1.  Levels without fluid in the whole warp are
// skipped (their cells stay 0 in both buffers).  The division by 6 is the
// FMA-corrected reciprocal product; a sweep in which some sum leaves its
// exact range is repeated by the CTA with IEEE divides.
//
// Residual checks (RESIDUAL mode, every `check` sweeps; once at the end in
// FIXED mode): FP64 ||b - A p||^2 over the tiles' fluid cells, per thread in
// x order, per CTA by a fixed tree, then summed over the CTAs' partials in
// index order by every CTA, so all make the same stop decision.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>

#include "aq_kernels.cuh"

namespace aqb {

// RN(s / 6).  On the fast path q0 = RN(s * RN(1/6)) is within an ulp of
// s/6, the FMA remainder s - 6 q0 is exact, and the FMA correction
// q0 + rem * RN(1/6) rounds to the correctly rounded quotient (the
// correction step of Markstein's division).  Checked exhaustively against
// IEEE division: equal for +0 and for every finite s whose quotient is a
// normal number (|s| >= 6 * 2^-126; 4,219,469,824 values, no difference).
// div6_fast_ok(s) accepts +0 and finite s with |s| >= 2^-123, a subset;
// everything else (-0, tiny, Inf, NaN) takes the IEEE divide.
__device__ __forceinline__ float div6_fast(float s) {
  const float r = 0x1.555556p-3f;  // RN(1/6)
  const float q0 = __fmul_rn(s, r);
  const float rem = __fmaf_rn(-q0, 6.0f, s);
  return __fmaf_rn(rem, r, q0);
}
__device__ __forceinline__ bool div6_fast_ok(float s) {
  const unsigned b = __float_as_uint(s);
  return b == 0u || ((b >> 23) & 0xffu) - 4u <= 250u;  // biased exponent in [4, 254]
}
__device__ __forceinline__ float div6(float s) { return div6_fast_ok(s) ? div6_fast(s) : __fdiv_rn(s, 6.f); }

namespace {

template <int TX, int TY, int XS>
struct Res {
  static constexpr int K = 4, TZ = 24;
  static constexpr int EX = TX + 2 * K, EY = TY + 2 * K, EZ = TZ + 2 * K;
  static constexpr int EQ = EZ / 4;        // 8 z-quads per box row
  static constexpr int XSEG = XS;          // x levels per thread
  static constexpr int NXS = EX / XSEG;    // x segments
  static constexpr int THREADS = NXS * EY * EQ;
  static constexpr int PL4 = EY * EQ;      // float4 per x plane of a buffer
  static constexpr int BUF4 = EX * PL4;    // float4 per buffer
  static constexpr int SMEM = 2 * BUF4 * (int)sizeof(float4);
  static_assert(EQ == 8 && EX % XSEG == 0 && EY % 4 == 0, "a warp is 4 whole rows of one x segment");
  static_assert(THREADS <= 1024, "too many threads for one CTA");
  static_assert(SMEM <= 232448, "two buffers must fit in shared memory");
  static_assert(TX % kBrick == 0 && TY % kBrick == 0 && TZ % kBrick == 0, "tiles are whole bricks");
};
// cut (halo inside the domain) rather than domain walls.
struct Box {
  int ex, ey, ez;
  int nx, ny, nz;
  int cx0, cy0, cz0, cx1, cy1, cz1;
  int cut;  // bits: 1 x lo, 2 x hi, 4 y lo, 8 y hi, 16 z lo, 32 z hi
};

template <int TX, int TY, int TZ, int K>
__device__ __forceinline__ Box box_of(const Dims& d, int id) {
  const int nty = (d.sy + TY - 1) / TY, ntz = (d.sz + TZ - 1) / TZ;
  const int tz = id % ntz, t = id / ntz;
  const int ty = t % nty, tx = t / nty;
  Box b;
  const int ox = tx * TX, oy = ty * TY, oz = tz * TZ;
  b.ex = max(ox - K, 0);
  b.ey = max(oy - K, 0);
  b.ez = max(oz - K, 0);
  const int hx = min(ox + TX + K, d.sx), hy = min(oy + TY + K, d.sy), hz = min(oz + TZ + K, d.sz);
  b.nx = hx - b.ex;
  b.ny = hy - b.ey;
  b.nz = hz - b.ez;
  b.cx0 = ox - b.ex;
  b.cy0 = oy - b.ey;
  b.cz0 = oz - b.ez;
  b.cx1 = min(ox + TX, d.sx) - b.ex;
  b.cy1 = min(oy + TY, d.sy) - b.ey;
  b.cz1 = min(oz + TZ, d.sz) - b.ez;
  b.cut = (b.ex > 0 ? 1 : 0) | (hx < d.sx ? 2 : 0) | (b.ey > 0 ? 4 : 0) | (hy < d.sy ? 8 : 0) |
          (b.ez > 0 ? 16 : 0) | (hz < d.sz ? 32 : 0);
  return b;
}

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned int* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// One TMA tensor copy of a (32, EY, EX) box of a pressure buffer at (z, y, x)
// into shared memory, completing on the mbarrier (expected bytes armed by the
// same thread just before).
__device__ __forceinline__ void tma_box_load(uint32_t dst, const CUtensorMap* map, int z, int y, int x,
                                             uint32_t mbar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar), "r"(bytes) : "memory");
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(z), "r"(y), "r"(x), "r"(mbar)
      : "memory");
}

// Bounded wait for phase `parity` of an mbarrier: false after spin_limit
// polls or one second.
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t mbar, uint32_t parity, unsigned spin_limit) {
  const unsigned long long t0 = global_ns();
  for (unsigned i = 0;; ++i) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(done)
        : "r"(mbar), "r"(parity)
        : "memory");
    if (done) return true;
    if (i > spin_limit || ((i & 255u) == 0u && global_ns() - t0 > 1000000000ull)) return false;
  }
}

// Bounded grid barrier on a counter that only grows (arrival e waits for
// e * gridDim.x arrivals): the CTA's writes are published by thread 0's
// release add after the CTA barrier (release is cumulative over what the CTA
// barrier ordered before it) and the others' are seen through the acquire
// poll.  Gives up after spin_limit polls or one second,
// whichever comes first: it then sets *fail and returns false, and after any
// failure every later barrier returns false within 64 polls.
__device__ __forceinline__ bool res_barrier(unsigned int* bar, unsigned target, int* fail, unsigned spin_limit) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    // arrive at once (a failure elsewhere shows in the poll below); the
    // failure flag is read every 64 polls only, as a read after an acquire
    // waits for it
    int ok = 1;
    asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(bar) : "memory");
    unsigned spins = 0;
    const unsigned long long t0 = global_ns();
    while (ld_acquire_u32(bar) < target) {
      ++spins;
      if (spins > spin_limit ||
          ((spins & 63u) == 0u && (*reinterpret_cast<volatile int*>(fail) || global_ns() - t0 > 1000000000ull))) {
        atomicExch(fail, 1);
        ok = 0;
        break;
      }
    }
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// Sum over the CTA in a fixed order: xor tree within warps, warps in order.
template <int THREADS>
__device__ __forceinline__ double cta_sum(double v, double* s_red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < THREADS / 32; ++w) t += s_red[w];
  __syncthreads();
  return t;  // valid in thread 0
}


// FP64 ||b - A p||^2 of the fluid cells (bits 0-3 of f) of a z-quad, in cell
// order, each as b + (x+1 + x-1 + y+1 + y-1 + z+1 + z-1) - 6 p.
__device__ __forceinline__ double quad_residual(const float4& xp, const float4& xm, const float4& yp,
                                                const float4& ym, const float4& pc, float zl, float zh,
                                                const float4& b, unsigned f) {
  const float self[4] = {pc.x, pc.y, pc.z, pc.w};
  const float zp[4] = {pc.y, pc.z, pc.w, zh};
  const float zm[4] = {zl, pc.x, pc.y, pc.z};
  const float vxp[4] = {xp.x, xp.y, xp.z, xp.w}, vxm[4] = {xm.x, xm.y, xm.z, xm.w};
  const float vyp[4] = {yp.x, yp.y, yp.z, yp.w}, vym[4] = {ym.x, ym.y, ym.z, ym.w};
  const float vb[4] = {b.x, b.y, b.z, b.w};
  double acc = 0.0;
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    if (!((f >> c) & 1u)) continue;
    double s = (double)vxp[c];
    s += (double)vxm[c];
    s += (double)vyp[c];
    s += (double)vym[c];
    s += (double)zp[c];
    s += (double)zm[c];
    const double r = (double)vb[c] + s - 6.0 * (double)self[c];
    acc += r * r;
  }
  return acc;
}


// The Jacobi update of one z-quad (cells c..c+3 along z): pn / pm the x + 1
// / x - 1 quads, yp / ym the y neighbours, pc the quad itself, zl / zh the
// z - 1 neighbour of cell 0 and z + 1 of cell 3, b the rhs; f its fluid
// marks (bits 0-3).  Non-fluid cells give 0.  Without IEEE, bad is set when
// some sum leaves the fast quotient's exact range.
template <bool IEEE>
__device__ __forceinline__ float4 quad_update(const float4& pn, const float4& pm, const float4& yp, const float4& ym,
                                              const float4& pc, float zl, float zh, const float4& b, unsigned f,
                                              bool& bad) {
  // per cell: x+1, x-1, y+1, y-1, z+1, z-1, rhs, summed in that order
  float s0 = pn.x + pm.x, s1 = pn.y + pm.y, s2 = pn.z + pm.z, s3 = pn.w + pm.w;
  s0 += yp.x; s1 += yp.y; s2 += yp.z; s3 += yp.w;
  s0 += ym.x; s1 += ym.y; s2 += ym.z; s3 += ym.w;
  s0 += pc.y; s1 += pc.z; s2 += pc.w; s3 += zh;
  s0 += zl;   s1 += pc.x; s2 += pc.y; s3 += pc.z;
  s0 += b.x;  s1 += b.y;  s2 += b.z;  s3 += b.w;
  float q0, q1, q2, q3;
  if (IEEE) {
    q0 = __fdiv_rn(s0, 6.f);
    q1 = __fdiv_rn(s1, 6.f);
    q2 = __fdiv_rn(s2, 6.f);
    q3 = __fdiv_rn(s3, 6.f);
  } else {
    const float mn = fminf(fminf(fabsf(s0), fabsf(s1)), fminf(fabsf(s2), fabsf(s3)));
    const float mx = fmaxf(fmaxf(fabsf(s0), fabsf(s1)), fmaxf(fabsf(s2), fabsf(s3)));
    bad |= !(mn >= 0x1p-123f && mx <= 0x1.fffffep127f);
    q0 = div6_fast(s0);
    q1 = div6_fast(s1);
    q2 = div6_fast(s2);
    q3 = div6_fast(s3);
  }
  return make_float4((f & 1u) ? q0 : 0.f, (f & 2u) ? q1 : 0.f, (f & 4u) ? q2 : 0.f, (f & 8u) ? q3 : 0.f);
}

// One sweep of one thread's x segment: the XSEG z-quads at S, S + PL4, ...
// (levels of jmask only) into D, two levels per step so that their loads and
// sums overlap.  Levels are compile-time (registers only); x neighbours from
// a sliding window, the x + 1 neighbour clamped to level jlast (the box's
// last level, where the x+1 face is a wall: the cell itself), x - 1 of level
// 0 the cell itself at an x = 0 wall (xm_self); y neighbours at offsets ymo
// and ypo; z neighbours by shuffle (the cell itself at the box's z faces).
// Non-fluid cells carry rhs 1 and are written as 0; lanes outside the region
// (act false) write nothing.  Without IEEE the quotient is the FMA-corrected
// reciprocal product, exact while every |sum| of a quad is in [2^-123,
// FLT_MAX]; the return value says that some sum of a lane in the region was
// not (min/max skip a NaN sum, whose quotient is NaN either way).
template <int XSEG, int PL4, bool IEEE>
__device__ __forceinline__ bool res_sweep(const float4* __restrict__ S, float4* __restrict__ D, int ymo, int ypo,
                                          const float4 (&rb)[XSEG], unsigned long long fl, unsigned jmask, int jlast,
                                          bool xm_self, bool act, bool zl_self, bool zh_self) {
  static_assert(XSEG % 2 == 0, "levels go in pairs");
  constexpr unsigned FULL = 0xffffffffu;
  bool bad = false;
  float4 pc = S[0];
  float4 pm = S[xm_self ? 0 : -PL4];
#pragma unroll
  for (int j = 0; j < XSEG; j += 2) {
    const float4 p1 = S[min(j + 1, jlast) * PL4];  // level j + 1 (x + 1 of level j)
    const float4 p2 = S[min(j + 2, jlast) * PL4];  // x + 1 of level j + 1
    const unsigned pair = (jmask >> j) & 3u;
    if (pair) {
      float zl0 = __shfl_up_sync(FULL, pc.w, 1), zh0 = __shfl_down_sync(FULL, pc.x, 1);
      float zl1 = __shfl_up_sync(FULL, p1.w, 1), zh1 = __shfl_down_sync(FULL, p1.x, 1);
      zl0 = zl_self ? pc.x : zl0;
      zh0 = zh_self ? pc.w : zh0;
      zl1 = zl_self ? p1.x : zl1;
      zh1 = zh_self ? p1.w : zh1;
      const float4 ym0 = S[j * PL4 + ymo], yp0 = S[j * PL4 + ypo];
      const float4 ym1 = S[(j + 1) * PL4 + ymo], yp1 = S[(j + 1) * PL4 + ypo];
      bool bad0 = false, bad1 = false;
      const float4 q0 = quad_update<IEEE>(p1, pm, yp0, ym0, pc, zl0, zh0, rb[j], (unsigned)(fl >> (4 * j)), bad0);
      const float4 q1 = quad_update<IEEE>(p2, pc, yp1, ym1, p1, zl1, zh1, rb[j + 1],
                                          (unsigned)(fl >> (4 * (j + 1))), bad1);
      if (act && (pair & 1u)) D[j * PL4] = q0;
      if (act && (pair & 2u)) D[(j + 1) * PL4] = q1;
      bad |= ((pair & 1u) && bad0) || ((pair & 2u) && bad1);
    }
    pm = p1;
    pc = p2;
  }
  return bad && act;
}

template <int TX, int TY, int XS>
__global__ void __launch_bounds__(Res<TX, TY, XS>::THREADS, 1)
    k_resident_solve(Dims d, float* __restrict__ pa, float* __restrict__ pb, const float* __restrict__ rhs,
                     const int8_t* __restrict__ type, const int* __restrict__ tiles, const int* __restrict__ n_tiles,
                     unsigned int* __restrict__ bar, double* __restrict__ part, SolveState* __restrict__ ss,
                     int fixed_sweeps, int check, int max_iters, double tol, BarrierTest bt,
                     const __grid_constant__ CUtensorMap map_a, const __grid_constant__ CUtensorMap map_b) {
  using R = Res<TX, TY, XS>;
  constexpr int EQ = R::EQ, PL4 = R::PL4, XSEG = R::XSEG, K = R::K;
  constexpr unsigned FULL = 0xffffffffu;
  extern __shared__ __align__(128) float4 smem4[];  // [2][EX][EY][EQ]; TMA destinations are 128-byte aligned
  __shared__ double s_red[32];
  __shared__ double s_r2;
  __shared__ Box s_box;  // the resident tile's box (read where used: no registers held across the solve)
  __shared__ __align__(8) uint64_t s_mbar;  // completion of the box's TMA copy

  const int G = gridDim.x, cta = blockIdx.x;
  // test hook: this CTA never arrives at a barrier (a participant that does
  // not join), so the others' bounded waits run out
  if (cta == bt.withhold_cta) return;
  const unsigned spin_limit = bt.spin_limit ? bt.spin_limit : kSpinLimit;
  int* fail = &ss->sync_timeout;
  const int n = *n_tiles;
  const bool resident = n <= G;
  const int tid = threadIdx.x;
  // this thread: z-quad qq of box row ly, x levels [xa, xa + XSEG)
  const int qq = tid % EQ, ly = (tid / EQ) % R::EY, xa = (tid / (EQ * R::EY)) * XSEG;
  const int col = ly * EQ + qq;
  const int it0 = ss->iterations;  // sweeps a warm start already did

  float4 rb[XSEG];  // rhs of this thread's quads (0 on non-fluid cells)
  unsigned long long fl = 0ull;  // bit 4 j + c: cell c of the quad at level xa + j is fluid
  // bit j: some lane of the warp holds fluid at level xa + j.  Resident tiles
  // skip the other levels (their cells are 0 in both shared buffers for the
  // whole solve); tiles that take turns in one CTA sweep every level.
  unsigned wmask = (1u << XSEG) - 1u;
  int cur = 0;  // global buffer of the current iterate (0: pa, 1: pb)
  int par = 0;  // shared buffer of the current iterate

  // both buffers zero once: cells no box covers stay finite
  for (int i = tid; i < 2 * R::BUF4; i += R::THREADS) smem4[i] = make_float4(0.f, 0.f, 0.f, 0.f);
  const uint32_t mbar = smem_addr(&s_mbar);
  uint32_t tma_phase = 0;
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }

  // Box t of global buffer `which` (0: pa, 1: pb) into shared buffer par by
  // one TMA copy of the whole (32, EY, EX) box (the tile's own cells come
  // back as the block stored them; cells past the domain read 0), and with
  // `full` this thread's rhs and fluid marks into registers.  Returns false,
  // CTA-uniformly, if the copy did not complete within the bounded wait.
  auto load = [&](const Box& t, int which, bool full) -> bool {
    if (tid == 0) {
      // order this CTA's earlier shared accesses and the other CTAs' global
      // stores (acquired at the grid barrier) before the async-proxy copy
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      asm volatile("fence.proxy.async.global;" ::: "memory");
      tma_box_load(smem_addr(smem4 + par * R::BUF4), which ? &map_b : &map_a, t.ez, t.ey, t.ex, mbar,
                   (uint32_t)R::BUF4 * 16u);
    }
    if (full) {
      const bool colin = ly < t.ny && 4 * qq < t.nz;
      const int base = (t.ex * d.sy + t.ey + ly) * d.sz + t.ez + 4 * qq;
      fl = 0ull;
#pragma unroll
      for (int j = 0; j < XSEG; ++j) {
        const int x = xa + j;
        rb[j] = make_float4(1.f, 1.f, 1.f, 1.f);
        if (colin && x < t.nx) {
          const int c = base + x * d.sy * d.sz;
          const char4 ty = *reinterpret_cast<const char4*>(type + c);
          const unsigned f = (ty.x == kFluid ? 1u : 0u) | (ty.y == kFluid ? 2u : 0u) | (ty.z == kFluid ? 4u : 0u) |
                             (ty.w == kFluid ? 8u : 0u);
          fl |= (unsigned long long)f << (4 * j);
          if (f) {
            const float4 b = __ldg(reinterpret_cast<const float4*>(rhs + c));
            rb[j] = make_float4((f & 1u) ? b.x : 1.f, (f & 2u) ? b.y : 1.f, (f & 4u) ? b.z : 1.f, (f & 8u) ? b.w : 1.f);
          }
        }
      }
      if (resident) {
        wmask = 0u;
#pragma unroll
        for (int j = 0; j < XSEG; ++j) wmask |= (__any_sync(FULL, (fl >> (4 * j)) & 15u) ? 1u : 0u) << j;
      }
    }
    bool done = mbar_wait_bounded(mbar, tma_phase, spin_limit);
    if (!done) {
      atomicExch(fail, 1);
      done = mbar_wait_bounded(mbar, tma_phase, spin_limit);  // the copy in flight, bounded again
    }
    tma_phase ^= 1u;
    return __syncthreads_and(done) != 0;
  };

  // Sweep s (1-based) of a block on box t: shared buffer par -> par ^ 1, over
  // the region of cells at least s cells inside each cut face (whole quads:
  // a quad's cells outside the region are never read by cells inside it).
  // Wall neighbours are the cell itself.
  auto sweep = [&](const Box& t, int s) {
    const int xlo = (t.cut & 1) ? s : 0, xhi = t.nx - ((t.cut & 2) ? s : 0);
    const int ylo = (t.cut & 4) ? s : 0, yhi = t.ny - ((t.cut & 8) ? s : 0);
    const int zlo = (t.cut & 16) ? s : 0, zhi = t.nz - ((t.cut & 32) ? s : 0);
    const bool act = ly >= ylo && ly < yhi && 4 * qq + 4 > zlo && 4 * qq < zhi;
    // levels of this segment inside the region (and, resident, holding fluid)
    const int jl = max(xlo - xa, 0), jh = min(xhi - xa, XSEG);
    const unsigned jmask = jh > jl ? (((1u << jh) - 1u) & ~((1u << jl) - 1u)) & wmask : 0u;
    const float4* S = smem4 + par * R::BUF4 + col + xa * PL4;
    float4* D = smem4 + (par ^ 1) * R::BUF4 + col + xa * PL4;
    // ly == 0 and ly == ny - 1 are in the region only at walls; rows past the
    // box (clipped boxes) read their own column, so no read leaves the buffer
    const int ymo = ly == 0 ? 0 : -EQ, ypo = ly >= t.ny - 1 ? 0 : EQ;
    const bool zl_self = qq == 0, zh_self = 4 * qq + 4 >= t.nz;
    const int jlast = t.nx - 1 - xa;  // x + 1 of level jlast is outside the box (a wall)
    bool bad = false;
    if (jmask)  // warp-uniform
      bad = res_sweep<XSEG, PL4, false>(S, D, ymo, ypo, rb, fl, jmask, jlast, xa == 0, act, zl_self, zh_self);
    // a sum outside the fast quotient's range anywhere in the CTA's region:
    // the sweep again with IEEE divides (it reads only buffer par, so it can
    // repeat)
    if (__syncthreads_or(bad)) {
      if (jmask) res_sweep<XSEG, PL4, true>(S, D, ymo, ypo, rb, fl, jmask, jlast, xa == 0, act, zl_self, zh_self);
      __syncthreads();
    }
    par ^= 1;
  };

  // ||b - A p||^2 over this thread's own fluid cells of box t (shared buffer
  // par current), FP64, in x order; summed over the CTA in a fixed order.
  auto residual = [&](const Box& t) -> double {
    double acc = 0.0;
    const bool owncol = ly < t.ny && 4 * qq < t.nz && ly >= t.cy0 && ly < t.cy1 && 4 * qq >= t.cz0 && 4 * qq < t.cz1;
    const bool zl_self = qq == 0, zh_self = 4 * qq + 4 >= t.nz;
    const float4* S = smem4 + par * R::BUF4 + col;
    const float4* Sym = S - (ly == 0 ? 0 : EQ);
    const float4* Syp = S + (ly >= t.ny - 1 ? 0 : EQ);
    if (xa < t.cx1 && xa + XSEG > t.cx0) {
      float4 pc = S[xa * PL4];
      float4 pm = xa > 0 ? S[(xa - 1) * PL4] : pc;
#pragma unroll
      for (int j = 0; j < XSEG; ++j) {
        const int x = xa + j;
        const float4 pn = x + 1 < t.nx ? S[(x + 1) * PL4] : pc;
        if (x >= t.cx0 && x < t.cx1) {
          float zl = __shfl_up_sync(FULL, pc.w, 1), zh = __shfl_down_sync(FULL, pc.x, 1);
          if (zl_self) zl = pc.x;
          if (zh_self) zh = pc.w;
          const unsigned f = owncol ? (fl >> (4 * j)) & 15u : 0u;
          if (f) acc += quad_residual(pn, pm, Syp[x * PL4], Sym[x * PL4], pc, zl, zh, rb[j], f);
        }
        pm = pc;
        pc = pn;
      }
    }
    return cta_sum<R::THREADS>(acc, s_red);
  };

  // This thread's own cells of box t from shared buffer par into dst.
  auto store = [&](const Box& t, float* __restrict__ dst) {
    const bool owncol = ly < t.ny && 4 * qq < t.nz && ly >= t.cy0 && ly < t.cy1 && 4 * qq >= t.cz0 && 4 * qq < t.cz1;
    if (owncol) {
      const float4* S = smem4 + par * R::BUF4 + col;
      const int base = (t.ex * d.sy + t.ey + ly) * d.sz + t.ez + 4 * qq;
#pragma unroll
      for (int j = 0; j < XSEG; ++j) {
        const int x = xa + j;
        if (x >= t.cx0 && x < t.cx1) *reinterpret_cast<float4*>(dst + base + x * d.sy * d.sz) = S[x * PL4];
      }
    }
  };

  const bool have = resident && cta < n;
  if (have && tid == 0) s_box = box_of<TX, TY, R::TZ, K>(d, tiles[cta]);
  __syncthreads();
  const Box& T = s_box;
  bool ok = true;
  if (have) ok = load(T, 0, true);
  unsigned epoch = 0;
  int done = 0, checks = 0;
  double r2 = -1.0, rel = -1.0;
  while (ok) {
    const bool due = fixed_sweeps > 0 ? done >= fixed_sweeps : (done > 0 && done % check == 0);
    if (due) {
      double acc = 0.0;
      if (resident) {
        if (have) acc = residual(T);
      } else {
        for (int j = cta; j < n && ok; j += G) {
          const Box t = box_of<TX, TY, R::TZ, K>(d, tiles[j]);
          ok = load(t, cur, true);
          if (ok) acc += residual(t);  // thread 0's running sum, tiles in order
        }
        if (!ok) break;
      }
      if (tid == 0) part[cta] = acc;
      ok = ok && res_barrier(bar, ++epoch * (unsigned)G, fail, spin_limit);
      if (!ok) break;
      if (tid < 32) {
        double t = 0.0;
        for (int k = tid; k < G; k += 32) t += __ldcg(part + k);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
        if (tid == 0) s_r2 = t;
      }
      __syncthreads();
      r2 = s_r2;
      rel = rel_residual_of(r2, ss->b2);
      ++checks;
      if (fixed_sweeps > 0) break;
      if (!(rel > tol) || !isfinite(rel) || it0 + done >= max_iters) break;
    }
    const int next = fixed_sweeps > 0 ? fixed_sweeps : (done / check + 1) * check;
    const int nsw = min(K, next - done);
    if (resident) {
      if (have) {
        for (int s = 1; s <= nsw; ++s) sweep(T, s);
        store(T, cur ? pa : pb);
      }
    } else {
      for (int j = cta; j < n && ok; j += G) {
        const Box t = box_of<TX, TY, R::TZ, K>(d, tiles[j]);
        ok = load(t, cur, true);
        if (!ok) break;
        for (int s = 1; s <= nsw; ++s) sweep(t, s);
        store(t, cur ? pa : pb);
      }
      if (!ok) break;
    }
    done += nsw;
    ok = ok && res_barrier(bar, ++epoch * (unsigned)G, fail, spin_limit);
    if (!ok) break;
    cur ^= 1;
    if (have) ok = load(T, cur, false);  // the box of the new iterate
  }

  // the result belongs in pa
  if (ok && cur == 1) {
    if (resident) {
      if (have) store(T, pa);
    } else {
      for (int j = cta; j < n; j += G) {
        const Box t = box_of<TX, TY, R::TZ, K>(d, tiles[j]);
        const bool owncol =
            ly < t.ny && 4 * qq < t.nz && ly >= t.cy0 && ly < t.cy1 && 4 * qq >= t.cz0 && 4 * qq < t.cz1;
        if (owncol) {
          const int base = (t.ex * d.sy + t.ey + ly) * d.sz + t.ez + 4 * qq;
          for (int jj = 0; jj < XSEG; ++jj) {
            const int x = xa + jj;
            if (x >= t.cx0 && x < t.cx1)
              *reinterpret_cast<float4*>(pa + base + x * d.sy * d.sz) =
                  __ldcg(reinterpret_cast<const float4*>(pb + base + x * d.sy * d.sz));
          }
        }
      }
    }
  }
  if (cta == 0 && tid == 0) {
    ss->iterations = it0 + done;
    ss->bodies += checks;
    ss->total_sweeps += done;
    ss->total_bodies += checks;
    ss->r2 = r2;
    ss->rel_residual = rel;
    const bool finite = isfinite(rel);
    if (!finite) ss->nonfinite = ss->nonfinite_seen = 1;
    ss->converged = (ok && finite && rel >= 0.0 && rel <= tol) ? 1 : 0;
  }
}

// Ordered list of the tiles (tbx x tby x tbz bricks) holding a fluid brick;
// also clears the barrier counter of the solve that follows.
__global__ void __launch_bounds__(1024) k_tile_list(Dims d, int tbx, int tby, int tbz,
                                                   const uint8_t* __restrict__ bact, int* __restrict__ tiles,
                                                   int* __restrict__ n_tiles, unsigned int* __restrict__ bar) {
  __shared__ int s_cnt[32], s_pre[32];
  __shared__ int s_tot, s_base;
  const int ntx = (d.bx + tbx - 1) / tbx, nty = (d.by + tby - 1) / tby, ntz = (d.bz + tbz - 1) / tbz;
  const int total = ntx * nty * ntz;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (threadIdx.x == 0) {
    s_base = 0;
    *bar = 0u;
  }
  __syncthreads();
  for (int base = 0; base < total; base += 1024) {
    const int id = base + threadIdx.x;
    int a = 0;
    if (id < total) {
      const int tz = id % ntz, t = id / ntz;
      const int ty = t % nty, tx = t / nty;
      for (int i = tx * tbx; i < min((tx + 1) * tbx, d.bx) && !a; ++i)
        for (int j = ty * tby; j < min((ty + 1) * tby, d.by) && !a; ++j)
          for (int k = tz * tbz; k < min((tz + 1) * tbz, d.bz) && !a; ++k) a = bact[(i * d.by + j) * d.bz + k];
    }
    const unsigned m = __ballot_sync(0xffffffffu, a != 0);
    const int pre = __popc(m & ((1u << lane) - 1u));
    if (lane == 0) s_cnt[w] = __popc(m);
    __syncthreads();
    if (w == 0) {
      const int v = s_cnt[lane];
      int incl = v;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
      }
      s_pre[lane] = incl - v;
      if (lane == 31) s_tot = incl;
    }
    __syncthreads();
    if (a) tiles[s_base + s_pre[w] + pre] = id;
    __syncthreads();
    if (threadIdx.x == 0) s_base += s_tot;
    __syncthreads();
  }
  if (threadIdx.x == 0) *n_tiles = s_base;
}

struct ShapeInfo {
  int tx, ty, tz;
};
// Tile shapes of the resident plan (plan.xc indexes this table; the x levels
// per thread of each are in dispatch below); z is 24 cells (a 32-cell box)
// for all.
constexpr ShapeInfo kShapes[] = {{8, 40, 24}, {16, 24, 24}, {8, 32, 24}, {16, 16, 24},
                                 {8, 16, 24}, {24, 16, 24}, {8, 40, 24}};
constexpr int kNumShapes = sizeof(kShapes) / sizeof(kShapes[0]);

PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }
  return fn;
}

// Tensor map of a pressure buffer: 3D (z, y, x), fp32, boxes of (32, EY, EX)
// cells, zero fill past the domain.
template <int TX, int TY, int XS>
cudaError_t box_map(CUtensorMap* m, const Dims& d, float* p) {
  using R = Res<TX, TY, XS>;
  const PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
  if (!enc || reinterpret_cast<uintptr_t>(p) % 16 != 0 || d.sz % 4 != 0) return cudaErrorInvalidValue;
  const cuuint64_t dims[3] = {(cuuint64_t)d.sz, (cuuint64_t)d.sy, (cuuint64_t)d.sx};
  const cuuint64_t strides[2] = {(cuuint64_t)d.sz * 4, (cuuint64_t)d.sy * d.sz * 4};
  const cuuint32_t box[3] = {(cuuint32_t)R::EZ, (cuuint32_t)R::EY, (cuuint32_t)R::EX};
  const cuuint32_t es[3] = {1, 1, 1};
  const CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, p, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                         CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

template <int TX, int TY, int XS>
cudaError_t launch_res(cudaStream_t st, const Dims& d, int ctas, float* pa, float* pb, const float* rhs,
                       const int8_t* type, const int* tiles, const int* n_tiles, unsigned int* bar, double* part,
                       SolveState* ss, int fixed_sweeps, int check, int max_iters, double tol, BarrierTest bt) {
  using R = Res<TX, TY, XS>;
  auto fn = &k_resident_solve<TX, TY, XS>;
  CUtensorMap ma, mb;
  cudaError_t e = box_map<TX, TY, XS>(&ma, d, pa);
  if (e == cudaSuccess) e = box_map<TX, TY, XS>(&mb, d, pb);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, R::SMEM);
  if (e != cudaSuccess) return e;
  cudaLaunchConfig_t lc = {};
  lc.gridDim = dim3(ctas);
  lc.blockDim = dim3(R::THREADS);
  lc.dynamicSmemBytes = R::SMEM;
  lc.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeCooperative;  // all CTAs co-resident, or the launch fails
  at[0].val.cooperative = 1;
  lc.attrs = at;
  lc.numAttrs = 1;
  return cudaLaunchKernelEx(&lc, fn, d, pa, pb, rhs, type, tiles, n_tiles, bar, part, ss, fixed_sweeps, check,
                            max_iters, tol, bt, ma, mb);
}

template <int TX, int TY, int XS>
int occupancy_of(int device) {
  using R = Res<TX, TY, XS>;
  auto fn = &k_resident_solve<TX, TY, XS>;
  if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, R::SMEM) != cudaSuccess) return 0;
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, R::THREADS, R::SMEM) != cudaSuccess) return 0;
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  return per_sm >= 1 ? sms : 0;  // one CTA per SM
}

// Dispatch over the shape: calls f.template operator()<TX, TY, XS>().
template <typename F>
auto dispatch(int shape, const F& f) -> decltype(f.template operator()<8, 40, 16>()) {
#define AQ_RES_CASE(S, A, B, X) \
  if (shape == S) return f.template operator()<A, B, X>();
  AQ_RES_CASE(0, 8, 40, 16)
  AQ_RES_CASE(1, 16, 24, 12)
  AQ_RES_CASE(2, 8, 32, 16)
  AQ_RES_CASE(3, 16, 16, 12)
  AQ_RES_CASE(4, 8, 16, 8)
  AQ_RES_CASE(5, 24, 16, 16)
  AQ_RES_CASE(6, 8, 40, 8)
#undef AQ_RES_CASE
  return decltype(f.template operator()<8, 40, 16>())();
}

struct OccupancyOf {
  int device;
  template <int A, int B, int X>
  int operator()() const { return occupancy_of<A, B, X>(device); }
};

struct LaunchRes {
  cudaStream_t st;
  const Dims& d;
  int ctas;
  float *pa, *pb;
  const float* rhs;
  const int8_t* type;
  const int* tiles;
  const int* n_tiles;
  unsigned int* bar;
  double* part;
  SolveState* ss;
  int fixed_sweeps, check, max_iters;
  double tol;
  BarrierTest bt;
  template <int A, int B, int X>
  cudaError_t operator()() const {
    return launch_res<A, B, X>(st, d, ctas, pa, pb, rhs, type, tiles, n_tiles, bar, part, ss, fixed_sweeps, check,
                            max_iters, tol, bt);
  }
};

}  // namespace

bool resident_plan_ok(int shape, int k) { return shape >= 0 && shape < kNumShapes && k == 4; }

int resident_tile_capacity(const Dims& d) {
  int cap = 1;
  for (const ShapeInfo& s : kShapes) {
    const int n = ((d.sx + s.tx - 1) / s.tx) * ((d.sy + s.ty - 1) / s.ty) * ((d.sz + s.tz - 1) / s.tz);
    cap = std::max(cap, n);
  }
  return cap;
}

int resident_ctas(int device, int shape, int k) {
  if (!resident_plan_ok(shape, k)) return 0;
  return dispatch(shape, OccupancyOf{device});
}

long long resident_cells_updated(const Dims& d, int shape, const uint8_t* bact_host) {
  if (shape < 0 || shape >= kNumShapes) return 0;
  const ShapeInfo s = kShapes[shape];
  const int tbx = s.tx / kBrick, tby = s.ty / kBrick, tbz = s.tz / kBrick;
  const int ntx = (d.bx + tbx - 1) / tbx, nty = (d.by + tby - 1) / tby, ntz = (d.bz + tbz - 1) / tbz;
  long long cells = 0;
  for (int tx = 0; tx < ntx; ++tx)
    for (int ty = 0; ty < nty; ++ty)
      for (int tz = 0; tz < ntz; ++tz) {
        bool a = false;
        for (int i = tx * tbx; i < std::min((tx + 1) * tbx, d.bx) && !a; ++i)
          for (int j = ty * tby; j < std::min((ty + 1) * tby, d.by) && !a; ++j)
            for (int k = tz * tbz; k < std::min((tz + 1) * tbz, d.bz) && !a; ++k)
              a = bact_host[(i * d.by + j) * d.bz + k] != 0;
        if (a)
          cells += (long long)(std::min((tx + 1) * s.tx, d.sx) - tx * s.tx) *
                   (std::min((ty + 1) * s.ty, d.sy) - ty * s.ty) * (std::min((tz + 1) * s.tz, d.sz) - tz * s.tz);
      }
  return cells;
}

cudaError_t launch_resident_solve(cudaStream_t st, const Dims& d, int shape, int k, int ctas, float* pa, float* pb,
                                  const float* rhs, const int8_t* type, const uint8_t* bact, int* tiles,
                                  int* n_tiles, unsigned int* bar, double* part, SolveState* ss, int fixed_sweeps,
                                  int check, int max_iters, double tol, BarrierTest bt) {
  if (!resident_plan_ok(shape, k) || ctas <= 0 || (fixed_sweeps <= 0 && check <= 0)) return cudaErrorInvalidValue;
  const ShapeInfo s = kShapes[shape];
  k_tile_list<<<1, 1024, 0, st>>>(d, s.tx / kBrick, s.ty / kBrick, s.tz / kBrick, bact, tiles, n_tiles, bar);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  return dispatch(shape,
                  LaunchRes{st, d, ctas, pa, pb, rhs, type, tiles, n_tiles, bar, part, ss, fixed_sweeps, check,
                            max_iters, tol, bt});
}

// Self-check of div6 against the IEEE divide over all 2^32 bit patterns
// (NaN results compare equal as NaN); writes the number of differences.
__global__ void k_div6_check(unsigned long long* bad) {
  unsigned long long local = 0;
  const unsigned stride = gridDim.x * blockDim.x;
  for (unsigned long long i = blockIdx.x * blockDim.x + threadIdx.x; i <= 0xffffffffull; i += stride) {
    const float x = __uint_as_float((unsigned)i);
    const float a = div6(x), e = __fdiv_rn(x, 6.f);
    if (!(isnan(a) && isnan(e)) && __float_as_uint(a) != __float_as_uint(e)) ++local;
  }
  if (local) atomicAdd(bad, local);
}

cudaError_t launch_div6_check(cudaStream_t st, unsigned long long* bad) {
  k_div6_check<<<148 * 8, 256, 0, st>>>(bad);
  return cudaGetLastError();
}

}  // namespace aqb
