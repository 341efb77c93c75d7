// Resident Jacobi pressure solve (stage (c), hot loop #1): the whole solve in
// one cooperative launch whose CTAs keep their tiles' pressure in shared
// memory and right-hand side in registers from the first sweep to the last,
// and exchange only tile halos through L2, once every K sweeps.
//
// Reference: jacobiImpl (Fluid/Fluid_3D_kernels.cu:460-505), launched
// pressureIterations times by solvePressureJacobi (Fluid/Fluid_3D_common.cu:48-55).
// Per fluid cell
//   p' = (p[x+1] + p[x-1] + p[y+1] + p[y-1] + p[z+1] + p[z-1] + rhs) / 6,
// summed in that order, 0 on non-fluid cells, out-of-domain neighbours
// clamped to the cell itself: the arithmetic of every other sweep kernel of
// the library (jacobi_quad), so the iterates are bit for bit the flat sweep's.
//
// Decomposition.  The grid is cut into tiles of TX x TY x TZ cells (whole 8^3
// activity bricks); a tile takes part when one of its bricks holds fluid
// (cells outside every such tile are non-fluid, 0 in both global buffers,
// and stay 0).  A CTA owns one tile and holds its box, the tile plus a K-cell
// halo clipped to the domain, in shared memory.  A block of K sweeps runs on
// the box with redundant halo work: sweep s updates the cells at least s
// cells inside every face of the box that is not a domain wall, so after K
// sweeps the tile's own cells hold exactly what K global sweeps give.  The
// tile then writes its cells to the global buffer of the block, every CTA
// meets at a bounded grid barrier, and each reloads only its halo.  The two
// global buffers alternate between blocks, so a CTA never overwrites cells a
// slower neighbour may still be reading.  When the active tiles outnumber
// the CTAs, each CTA walks its tiles one after another per block and
// reloads each whole box from L2 (same results, not resident).
//
// Threads.  One per (8-level y segment, x, z-quad) of the box: a thread
// keeps its segment's pressure quads in registers (y neighbours inside the
// segment are its own), takes the z neighbours from the lanes holding the
// adjacent quads (shuffles), and reads x neighbours, segment-end y
// neighbours and the rhs from shared memory; the new iterate goes to the
// other shared buffer (ping-pong per sweep).  The x stride of the shared
// arrays is padded to EZ mod 32, so the lanes of a warp, consecutive quads of
// one or two x rows, read 16-byte quads from distinct banks.
//
// Residual checks (RESIDUAL mode, every `check` sweeps; once at the end in
// FIXED mode): FP64 ||b - A p||^2 over the tiles' fluid cells, per thread in
// y order, per CTA by a fixed tree, then summed over the CTAs' partials in
// index order by every CTA, so all make the same stop decision.
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

template <int TX, int TY, int TZ, int K, int SEG_>
struct Res {
  static constexpr int EX = TX + 2 * K, EY = TY + 2 * K, EZ = TZ + 2 * K;
  static constexpr int EQ = EZ / 4;                   // z-quads per box row
  static constexpr int SEG = SEG_;                    // y levels per thread
  static constexpr int NSEG = (EY + SEG - 1) / SEG;
  static constexpr int NT = NSEG * EX * EQ;           // one thread per (y segment, x, z-quad)
  static constexpr int THREADS = (NT + 31) / 32 * 32;
  static constexpr int XS0 = EY * EZ;
  static constexpr int XS = XS0 + ((EZ % 32) - (XS0 % 32) + 64) % 32;  // x stride = EZ (mod 32)
  static constexpr int BUF = EX * XS;                 // floats per shared buffer
  // two pressure buffers (ping-pong) and the right-hand side
  static constexpr int SMEM = 3 * BUF * (int)sizeof(float);
  static_assert(K % 4 == 0 && TZ % 4 == 0, "z-quads stay aligned to the grid");
  static_assert(THREADS <= 1024, "too many threads for one CTA");
  static_assert(TX % kBrick == 0 && TY % kBrick == 0 && TZ % kBrick == 0, "tiles are whole bricks");
  static_assert(XS % 32 == EZ % 32 && XS % 4 == 0, "padding");
  static_assert(4 * SEG <= 64, "the fluid mask holds 16 levels of quads");
};

// A tile's box: origin (ex, ey, ez) and extent n* (clipped to the domain),
// the tile's own cells [c*0, c*1) in box coordinates, and which faces are
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

// Bounded grid barrier on a counter that only grows (arrival e waits for
// e * gridDim.x arrivals).  Gives up after spin_limit polls or one second,
// whichever comes first: it then sets *fail and returns false, and after any
// failure every barrier returns false at once.
__device__ __forceinline__ bool res_barrier(unsigned int* bar, unsigned target, int* fail, unsigned spin_limit) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    if (*reinterpret_cast<volatile int*>(fail)) {
      ok = 0;
    } else {
      __threadfence();
      atomicAdd(bar, 1u);
      unsigned spins = 0;
      const unsigned long long t0 = global_ns();
      while (ld_acquire_u32(bar) < target) {
        if (++spins > spin_limit || *reinterpret_cast<volatile int*>(fail) ||
            ((spins & 255u) == 0u && global_ns() - t0 > 1000000000ull)) {
          atomicExch(fail, 1);
          ok = 0;
          break;
        }
      }
      __threadfence();
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

// The quotients of a quad whose sums leave the fast path: IEEE divides, out
// of line so the common path carries no predicated copy of them.
__device__ __noinline__ float4 div6_quad_slow(float4 s, unsigned f) {
  return make_float4((f & 1u) ? __fdiv_rn(s.x, 6.f) : 0.f, (f & 2u) ? __fdiv_rn(s.y, 6.f) : 0.f,
                     (f & 4u) ? __fdiv_rn(s.z, 6.f) : 0.f, (f & 8u) ? __fdiv_rn(s.w, 6.f) : 0.f);
}

// The rhs of a non-fluid cell in the resident solve's shared copy: a NaN
// payload no arithmetic produces (the GPU's NaN results are the canonical
// 0x7fffffff, and the rhs comes from the divergence stage's arithmetic).
constexpr unsigned kNotFluidBits = 0x7fc0a11au;
#define kNotFluid __uint_as_float(kNotFluidBits)
__device__ __forceinline__ unsigned fluid_bits(const float4& b) {
  return (__float_as_uint(b.x) != kNotFluidBits ? 1u : 0u) | (__float_as_uint(b.y) != kNotFluidBits ? 2u : 0u) |
         (__float_as_uint(b.z) != kNotFluidBits ? 4u : 0u) | (__float_as_uint(b.w) != kNotFluidBits ? 8u : 0u);
}

// One Jacobi update of a z-quad: p' = (x+1, x-1, y+1, y-1, z+1, z-1 summed in
// that order, + rhs) / 6 on fluid cells (bits 0-3 of f), 0 elsewhere.
__device__ __forceinline__ float4 quad_update(const float4& xp, const float4& xm, const float4& yp, const float4& ym,
                                              const float4& pc, float zl, float zh, const float4& b, unsigned f) {
  float4 s;
  s.x = xp.x + xm.x; s.x += yp.x; s.x += ym.x; s.x += pc.y; s.x += zl; s.x += b.x;
  s.y = xp.y + xm.y; s.y += yp.y; s.y += ym.y; s.y += pc.z; s.y += pc.x; s.y += b.y;
  s.z = xp.z + xm.z; s.z += yp.z; s.z += ym.z; s.z += pc.w; s.z += pc.y; s.z += b.z;
  s.w = xp.w + xm.w; s.w += yp.w; s.w += ym.w; s.w += zh; s.w += pc.z; s.w += b.w;
  // one warp-uniform test: the rare quads leaving the fast path take the IEEE divides
  const bool slow = ((f & 1u) && !div6_fast_ok(s.x)) || ((f & 2u) && !div6_fast_ok(s.y)) ||
                    ((f & 4u) && !div6_fast_ok(s.z)) || ((f & 8u) && !div6_fast_ok(s.w));
  if (__any_sync(__activemask(), slow)) {
    if (slow) return div6_quad_slow(s, f);
  }
  return make_float4((f & 1u) ? div6_fast(s.x) : 0.f, (f & 2u) ? div6_fast(s.y) : 0.f,
                     (f & 4u) ? div6_fast(s.z) : 0.f, (f & 8u) ? div6_fast(s.w) : 0.f);
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

template <int TX, int TY, int TZ, int K, int SEG_>
__global__ void __launch_bounds__(Res<TX, TY, TZ, K, SEG_>::THREADS, 1)
    k_resident_solve(Dims d, float* __restrict__ pa, float* __restrict__ pb, const float* __restrict__ rhs,
                     const int8_t* __restrict__ type, const int* __restrict__ tiles, const int* __restrict__ n_tiles,
                     unsigned int* __restrict__ bar, double* __restrict__ part, SolveState* __restrict__ ss,
                     int fixed_sweeps, int check, int max_iters, double tol, BarrierTest bt) {
  using R = Res<TX, TY, TZ, K, SEG_>;
  constexpr int SEG = R::SEG, EQ = R::EQ, XS4 = R::XS / 4;
  extern __shared__ float4 smem4[];  // [3][EX][XS / 4]: p, p, rhs; x; (y * EZ + z) / 4
  __shared__ double s_red[32];
  __shared__ double s_r2;

  const int G = gridDim.x, cta = blockIdx.x;
  // test hook: this CTA never arrives at a barrier (a participant that does
  // not join), so the others' bounded waits run out
  if (cta == bt.withhold_cta) return;
  const unsigned spin_limit = bt.spin_limit ? bt.spin_limit : kSpinLimit;
  int* fail = &ss->sync_timeout;
  const int n = *n_tiles;
  const bool resident = n <= G;
  const int tid = threadIdx.x;
  const bool thr = tid < R::NT;
  // this thread: z-quad q of box row cx, levels [y0, y0 + SEG) of the box
  const int q = tid % EQ, cx = (tid / EQ) % R::EX, y0 = (tid / (EQ * R::EX)) * SEG;
  const int it0 = ss->iterations;  // sweeps a warm start already did

  unsigned long long fl = 0ull;  // bit 4(ly - y0) + c: cell c of the quad at level ly is fluid
  float4* RB = smem4 + 2 * (R::BUF / 4);  // the rhs of the box
  float* g[2] = {pa, pb};
  int cur = 0;  // global buffer of the current iterate
  int par = 0;  // shared buffer of the current iterate
  const int col_i = cx * XS4 + q;  // shared index of level 0 of this thread's quad column

  // This thread's quads of box t from global buffer src into shared buffer
  // par (all of them, with rhs and fluid bits, when `full`; else those
  // outside the tile's own cells, whose current values are already there).
  auto load = [&](const Box& t, const float* __restrict__ src, bool full) {
    const bool col = thr && cx < t.nx && 4 * q < t.nz;
    const bool ownq = col && cx >= t.cx0 && cx < t.cx1 && 4 * q >= t.cz0 && 4 * q < t.cz1;
    if (full) fl = 0ull;
    if (col) {
      const int base = ((t.ex + cx) * d.sy + t.ey + y0) * d.sz + t.ez + 4 * q;
      float4* S = smem4 + par * (R::BUF / 4) + col_i;
#pragma unroll
      for (int j = 0; j < SEG; ++j) {
        const int ly = y0 + j;
        if (ly < t.ny) {
          const int c = base + j * d.sz;
          if (full || !ownq || ly < t.cy0 || ly >= t.cy1) S[ly * EQ] = __ldcg(reinterpret_cast<const float4*>(src + c));
          if (full) {
            // non-fluid cells carry a NaN sentinel instead of their rhs (which
            // they never use): the sweep reads the fluid mark with the rhs
            float4 rb = __ldg(reinterpret_cast<const float4*>(rhs + c));
            const char4 ty = *reinterpret_cast<const char4*>(type + c);
            if (ty.x != kFluid) rb.x = kNotFluid;
            if (ty.y != kFluid) rb.y = kNotFluid;
            if (ty.z != kFluid) rb.z = kNotFluid;
            if (ty.w != kFluid) rb.w = kNotFluid;
            RB[col_i + ly * EQ] = rb;
            fl |= (unsigned long long)((ty.x == kFluid ? 1u : 0u) | (ty.y == kFluid ? 2u : 0u) |
                                       (ty.z == kFluid ? 4u : 0u) | (ty.w == kFluid ? 8u : 0u))
                  << (4 * j);
          }
        }
      }
    }
    __syncthreads();
  };

  // Sweep s (1-based) of a block on box t: shared buffer par -> par ^ 1.  The
  // sweep's region (every cell at least s cells inside each cut face) is cut
  // into rows of z-quads; the CTA's lanes take consecutive quads of
  // consecutive rows, so every lane has work and a warp's loads of a level
  // are contiguous.  A wall neighbour is the cell itself (offset 0).
  auto sweep = [&](const Box& t, int s) {
    const int xlo = (t.cut & 1) ? s : 0, xhi = t.nx - ((t.cut & 2) ? s : 0);
    const int ylo = (t.cut & 4) ? s : 0, yhi = t.ny - ((t.cut & 8) ? s : 0);
    const int zlo = (t.cut & 16) ? s : 0, zhi = t.nz - ((t.cut & 32) ? s : 0);
    // quads holding a cell of [zlo, zhi); their other cells are invalid and never read by valid ones
    const int qlo = zlo / 4, qhi = (zhi + 3) / 4;
    const int nq = qhi - qlo, ny = yhi - ylo;
    const int total = (xhi - xlo) * ny * nq;
    const float inv_nq = 1.f / (float)nq, inv_ny = 1.f / (float)ny;
    const bool ywall_lo = t.ey == 0, ywall_hi = t.ey + t.ny == d.sy;
    const float4* S = smem4 + par * (R::BUF / 4);
    float4* D = smem4 + (par ^ 1) * (R::BUF / 4);
    for (int it = tid; it < total; it += R::THREADS) {
      // it = (xr * ny + yr) * nq + qr; small integers, so the float quotients are exact
      const int rq = __float2int_rz(((float)it + 0.5f) * inv_nq);
      const int qr = it - rq * nq;
      const int xr = __float2int_rz(((float)rq + 0.5f) * inv_ny);
      const int yr = rq - xr * ny;
      const int x = xlo + xr, ly = ylo + yr, qq = qlo + qr;
      const int i = x * XS4 + ly * EQ + qq;
      const int gx = t.ex + x, gz = t.ez + 4 * qq;
      const float4 pc = S[i];
      const float4 xm = S[i + (gx == 0 ? 0 : -XS4)];
      const float4 xp = S[i + (gx == d.sx - 1 ? 0 : XS4)];
      const float4 ym = (ly == 0 && ywall_lo) ? pc : S[i - (ly > 0 ? EQ : 0)];
      const float4 yp = (ly == t.ny - 1 && ywall_hi) ? pc : S[i + EQ];
      const float* Sf = reinterpret_cast<const float*>(S + i);
      const float zl = Sf[(gz == 0 || qq == 0) ? 0 : -1];
      const float zh = Sf[(gz + 4 == d.sz || qq == EQ - 1) ? 3 : 4];
      const float4 b = RB[i];
      D[i] = quad_update(xp, xm, yp, ym, pc, zl, zh, b, fluid_bits(b));
    }
    __syncthreads();
    par ^= 1;
  };

  // ||b - A p||^2 over this thread's own fluid cells of box t (shared buffer
  // par current), FP64, in level order; summed over the CTA in a fixed order.
  auto residual = [&](const Box& t) -> double {
    double acc = 0.0;
    const bool ownq = thr && cx >= t.cx0 && cx < t.cx1 && 4 * q >= t.cz0 && 4 * q < t.cz1;
    const int lo = max(t.cy0, y0), hi = min(t.cy1, y0 + SEG);
    if (ownq && lo < hi) {
      const int gx = t.ex + cx, gz = t.ez + 4 * q;
      const int oxm = gx == 0 ? 0 : -XS4, oxp = gx == d.sx - 1 ? 0 : XS4;
      const int ozl = (gz == 0 || q == 0) ? 0 : -1, ozh = (gz + 4 == d.sz || q == EQ - 1) ? 3 : 4;
      const float4* S = smem4 + par * (R::BUF / 4) + col_i;
      const float4* Rb = RB + col_i;
      for (int ly = lo; ly < hi; ++ly) {
        const unsigned f = (unsigned)(fl >> (4 * (ly - y0))) & 15u;
        if (!f) continue;
        const int i = ly * EQ, gy = t.ey + ly;
        const float4 pc = S[i];
        const float4 ym = gy == 0 ? pc : S[i - EQ];
        const float4 yp = gy == d.sy - 1 ? pc : S[i + EQ];
        const float zl = reinterpret_cast<const float*>(S + i)[ozl];
        const float zh = reinterpret_cast<const float*>(S + i)[ozh];
        acc += quad_residual(S[i + oxp], S[i + oxm], yp, ym, pc, zl, zh, Rb[i], f);
      }
    }
    return cta_sum<R::THREADS>(acc, s_red);
  };

  // This thread's own cells of box t from shared buffer par into dst.
  auto store = [&](const Box& t, float* __restrict__ dst) {
    const bool ownq = thr && cx >= t.cx0 && cx < t.cx1 && 4 * q >= t.cz0 && 4 * q < t.cz1;
    const int lo = max(t.cy0, y0), hi = min(t.cy1, y0 + SEG);
    if (ownq) {
      const float4* S = smem4 + par * (R::BUF / 4) + col_i;
      const int base = ((t.ex + cx) * d.sy + t.ey) * d.sz + t.ez + 4 * q;
      for (int ly = lo; ly < hi; ++ly) *reinterpret_cast<float4*>(dst + base + ly * d.sz) = S[ly * EQ];
    }
  };

  Box T{};
  const bool have = resident && cta < n;
  if (have) {
    T = box_of<TX, TY, TZ, K>(d, tiles[cta]);
    load(T, g[cur], true);
  }
  unsigned epoch = 0;
  int done = 0, checks = 0;
  bool ok = true;
  double r2 = -1.0, rel = -1.0;
  for (;;) {
    const bool due = fixed_sweeps > 0 ? done >= fixed_sweeps : (done > 0 && done % check == 0);
    if (due) {
      double acc = 0.0;
      if (resident) {
        if (have) acc = residual(T);
      } else {
        for (int j = cta; j < n; j += G) {
          const Box t = box_of<TX, TY, TZ, K>(d, tiles[j]);
          load(t, g[cur], true);
          acc += residual(t);  // thread 0's running sum, tiles in order
        }
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
        store(T, g[cur ^ 1]);
      }
    } else {
      for (int j = cta; j < n; j += G) {
        const Box t = box_of<TX, TY, TZ, K>(d, tiles[j]);
        load(t, g[cur], true);
        for (int s = 1; s <= nsw; ++s) sweep(t, s);
        store(t, g[cur ^ 1]);
      }
    }
    done += nsw;
    ok = ok && res_barrier(bar, ++epoch * (unsigned)G, fail, spin_limit);
    if (!ok) break;
    cur ^= 1;
    if (have) load(T, g[cur], false);  // the halo of the new iterate
  }

  // the result belongs in pa
  if (ok && cur == 1) {
    if (resident) {
      if (have) store(T, pa);
    } else {
      for (int j = cta; j < n; j += G) {
        const Box t = box_of<TX, TY, TZ, K>(d, tiles[j]);
        const bool ownq = thr && cx >= t.cx0 && cx < t.cx1 && 4 * q >= t.cz0 && 4 * q < t.cz1;
        if (ownq) {
          const int base = ((t.ex + cx) * d.sy + t.ey + y0) * d.sz + t.ez + 4 * q;
          for (int jj = 0; jj < SEG; ++jj) {
            const int ly = y0 + jj;
            if (ly >= t.cy0 && ly < t.cy1)
              *reinterpret_cast<float4*>(pa + base + jj * d.sz) =
                  __ldcg(reinterpret_cast<const float4*>(pb + base + jj * d.sz));
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
// Tile shapes of the resident plan (plan.xc indexes this table).
// (6, 7: shape 0 with 8- and 5-level y segments: 576 and 960 threads)
constexpr ShapeInfo kShapes[] = {{8, 40, 16}, {8, 32, 16}, {16, 16, 16}, {8, 24, 16}, {8, 16, 16},
                                 {16, 24, 16}, {8, 40, 16}, {8, 40, 16}};
constexpr int kNumShapes = sizeof(kShapes) / sizeof(kShapes[0]);

template <int TX, int TY, int TZ, int K, int SEG>
cudaError_t launch_res(cudaStream_t st, const Dims& d, int ctas, float* pa, float* pb, const float* rhs,
                       const int8_t* type, const int* tiles, const int* n_tiles, unsigned int* bar, double* part,
                       SolveState* ss, int fixed_sweeps, int check, int max_iters, double tol, BarrierTest bt) {
  using R = Res<TX, TY, TZ, K, SEG>;
  auto fn = &k_resident_solve<TX, TY, TZ, K, SEG>;
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, R::SMEM);
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
                            max_iters, tol, bt);
}

template <int TX, int TY, int TZ, int K, int SEG>
int occupancy_of(int device) {
  using R = Res<TX, TY, TZ, K, SEG>;
  auto fn = &k_resident_solve<TX, TY, TZ, K, SEG>;
  if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, R::SMEM) != cudaSuccess) return 0;
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, R::THREADS, R::SMEM) != cudaSuccess) return 0;
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  return per_sm >= 1 ? sms : 0;  // one CTA per SM
}

// Dispatch over (shape, K): calls f.template operator()<TX, TY, TZ, K, SEG>().
template <typename F>
auto dispatch(int shape, int k, const F& f) -> decltype(f.template operator()<8, 40, 16, 4, 12>()) {
#define AQ_RES_CASE(S, A, B, C, G) \
  if (shape == S && k == 4) return f.template operator()<A, B, C, 4, G>();
  AQ_RES_CASE(0, 8, 40, 16, 12)
  AQ_RES_CASE(1, 8, 32, 16, 12)
  AQ_RES_CASE(2, 16, 16, 16, 8)
  AQ_RES_CASE(3, 8, 24, 16, 8)
  AQ_RES_CASE(4, 8, 16, 16, 8)
  AQ_RES_CASE(5, 16, 24, 16, 12)
  AQ_RES_CASE(6, 8, 40, 16, 8)
  AQ_RES_CASE(7, 8, 40, 16, 5)
#undef AQ_RES_CASE
  return decltype(f.template operator()<8, 40, 16, 4, 12>())();
}

struct OccupancyOf {
  int device;
  template <int A, int B, int C, int D, int E>
  int operator()() const { return occupancy_of<A, B, C, D, E>(device); }
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
  template <int A, int B, int C, int D, int E>
  cudaError_t operator()() const {
    return launch_res<A, B, C, D, E>(st, d, ctas, pa, pb, rhs, type, tiles, n_tiles, bar, part, ss, fixed_sweeps, check,
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
  return dispatch(shape, k, OccupancyOf{device});
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
  return dispatch(shape, k,
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
