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
// Threads.  One per (x, z) column of the box: a thread keeps its column's
// pressure and rhs in registers, so y neighbours are its own, and reads the
// x and z neighbours from the other shared buffer (ping-pong per sweep).
// The x stride of the shared arrays is padded to EZ mod 32, so the 32 lanes
// of a warp, consecutive columns of one or two x rows, load one y level from
// 32 distinct banks.
//
// Residual checks (RESIDUAL mode, every `check` sweeps; once at the end in
// FIXED mode): FP64 ||b - A p||^2 over the tiles' fluid cells, per thread in
// y order, per CTA by a fixed tree, then summed over the CTAs' partials in
// index order by every CTA, so all make the same stop decision.
#include <algorithm>

#include "aq_kernels.cuh"

namespace aqb {

// RN(s / 6) for every float s.  On the fast path q0 = RN(s * RN(1/6)) is
// within an ulp of s/6, the FMA remainder s - 6 q0 is exact, and the FMA
// correction q0 + rem * RN(1/6) rounds to the correctly rounded quotient
// (the correction step of Markstein's division); checked exhaustively
// against IEEE division for every float whose quotient is a normal number
// (|s| >= 6 * 2^-126, finite: 4,219,469,824 values, no difference).  Zeros,
// subnormal quotients, infinities and NaN take the IEEE divide.
__device__ __forceinline__ float div6(float s) {
  const float a = fabsf(s);
  if (a >= 0x1.8p-124f && a <= 0x1.fffffep127f) {
    const float r = 0x1.555556p-3f;  // RN(1/6)
    const float q0 = __fmul_rn(s, r);
    const float rem = __fmaf_rn(-q0, 6.0f, s);
    return __fmaf_rn(rem, r, q0);
  }
  return __fdiv_rn(s, 6.f);
}

namespace {

template <int TX, int TY, int TZ, int K>
struct Res {
  static constexpr int EX = TX + 2 * K, EY = TY + 2 * K, EZ = TZ + 2 * K;
  static constexpr int NT = EX * EZ;                  // one thread per (x, z) column
  static constexpr int THREADS = (NT + 31) / 32 * 32;
  static constexpr int XS0 = EY * EZ;
  static constexpr int XS = XS0 + ((EZ % 32) - (XS0 % 32) + 64) % 32;  // x stride = EZ (mod 32)
  static constexpr int BUF = EX * XS;                 // floats per shared buffer
  static constexpr int SMEM = 2 * BUF * (int)sizeof(float);
  static_assert(THREADS <= 1024, "too many columns for one CTA");
  static_assert(EY <= 64, "the fluid mask holds 64 levels");
  static_assert(TX % kBrick == 0 && TY % kBrick == 0 && TZ % kBrick == 0, "tiles are whole bricks");
  static_assert(XS % 32 == EZ % 32, "padding");
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

// Bounded grid barrier on a counter that only grows (arrival e waits for
// e * gridDim.x arrivals); on timeout it sets *fail and returns false, and
// after any failure every barrier returns false at once.
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
      while (ld_acquire_u32(bar) < target) {
        if (++spins > spin_limit || *reinterpret_cast<volatile int*>(fail)) {
          atomicExch(fail, 1);
          ok = 0;
          break;
        }
        __nanosleep(32);
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

template <int TX, int TY, int TZ, int K>
__global__ void __launch_bounds__(Res<TX, TY, TZ, K>::THREADS, 1)
    k_resident_solve(Dims d, float* __restrict__ pa, float* __restrict__ pb, const float* __restrict__ rhs,
                     const int8_t* __restrict__ type, const int* __restrict__ tiles, const int* __restrict__ n_tiles,
                     unsigned int* __restrict__ bar, double* __restrict__ part, SolveState* __restrict__ ss,
                     int fixed_sweeps, int check, int max_iters, double tol, BarrierTest bt) {
  using R = Res<TX, TY, TZ, K>;
  constexpr int EY = R::EY, EZ = R::EZ, XS = R::XS;
  extern __shared__ float smem[];  // [2][EX][XS]: buffer, x, y * EZ + z
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
  const int cx = tid / EZ, cz = tid % EZ;  // this thread's column in the box
  const int it0 = ss->iterations;          // sweeps a warm start already did

  float p[EY], b[EY];
  unsigned long long fl = 0ull;  // bit ly: cell (cx, ly, cz) is fluid
#pragma unroll
  for (int ly = 0; ly < EY; ++ly) p[ly] = b[ly] = 0.f;
  float* g[2] = {pa, pb};
  int cur = 0;  // global buffer of the current iterate
  int par = 0;  // shared buffer of the current iterate

  // This thread's column of box t from global buffer src into p (every level
  // when `full`, with rhs and fluid mask; else the levels outside the tile's
  // own cells), then the whole column into shared buffer par.
  auto load = [&](const Box& t, const float* __restrict__ src, bool full) {
    const bool col = thr && cx < t.nx && cz < t.nz;
    const bool own = col && cx >= t.cx0 && cx < t.cx1 && cz >= t.cz0 && cz < t.cz1;
    if (full) fl = 0ull;
    if (col) {
      const int base = ((t.ex + cx) * d.sy + t.ey) * d.sz + t.ez + cz;
#pragma unroll
      for (int ly = 0; ly < EY; ++ly) {
        if (ly < t.ny) {
          const int c = base + ly * d.sz;
          if (full || !own || ly < t.cy0 || ly >= t.cy1) p[ly] = __ldcg(src + c);
          if (full) {
            b[ly] = __ldg(rhs + c);
            if (type[c] == kFluid) fl |= 1ull << ly;
          }
        }
      }
      float* S = smem + par * R::BUF + cx * XS + cz;
#pragma unroll
      for (int ly = 0; ly < EY; ++ly)
        if (ly < t.ny) S[ly * EZ] = p[ly];
    }
    __syncthreads();
  };

  // Sweep s of a block (1-based) on box t: shared buffer par -> par ^ 1.
  auto sweep = [&](const Box& t, int s) {
    const int xlo = (t.cut & 1) ? s : 0, xhi = t.nx - ((t.cut & 2) ? s : 0);
    const int ylo = (t.cut & 4) ? s : 0, yhi = t.ny - ((t.cut & 8) ? s : 0);
    const int zlo = (t.cut & 16) ? s : 0, zhi = t.nz - ((t.cut & 32) ? s : 0);
    const bool act = thr && cx >= xlo && cx < xhi && cz >= zlo && cz < zhi;
    if (act) {
      const int gx = t.ex + cx, gz = t.ez + cz;
      const int oxm = gx == 0 ? 0 : -XS, oxp = gx == d.sx - 1 ? 0 : XS;
      const int ozm = gz == 0 ? 0 : -1, ozp = gz == d.sz - 1 ? 0 : 1;
      const float* S = smem + par * R::BUF + cx * XS + cz;
      float* D = smem + (par ^ 1) * R::BUF + cx * XS + cz;
      const bool ywall_lo = t.ey == 0, ywall_hi = t.ey + t.ny == d.sy;
      float last = 0.f;  // level ly - 1 before this sweep
#pragma unroll
      for (int ly = 0; ly < EY; ++ly) {
        const float old = p[ly];
        if (ly >= ylo && ly < yhi) {
          const int i = ly * EZ;
          const float xm = S[i + oxm], xp = S[i + oxp], zm = S[i + ozm], zp = S[i + ozp];
          const float ym = (ly == 0 && ywall_lo) ? old : last;
          const float yp = (ly + 1 < EY && !(ly == t.ny - 1 && ywall_hi)) ? p[ly + 1 < EY ? ly + 1 : ly] : old;
          float sum = xp + xm;
          sum += yp;
          sum += ym;
          sum += zp;
          sum += zm;
          sum += b[ly];
          const float nv = ((fl >> ly) & 1ull) ? div6(sum) : 0.f;
          p[ly] = nv;
          D[i] = nv;
        }
        last = old;
        // the levels are independent; without this fence the compiler hoists
        // every level's shared loads at once and runs out of registers
        if ((ly & 7) == 7) asm volatile("" ::: "memory");
      }
    }
    __syncthreads();
    par ^= 1;
  };

  // ||b - A p||^2 over this thread's own fluid cells of box t (shared buffer
  // par and p current), FP64, in y order; summed over the CTA.
  auto residual = [&](const Box& t) -> double {
    double acc = 0.0;
    const bool own = thr && cx >= t.cx0 && cx < t.cx1 && cz >= t.cz0 && cz < t.cz1;
    if (own) {
      const int gx = t.ex + cx, gz = t.ez + cz;
      const int oxm = gx == 0 ? 0 : -XS, oxp = gx == d.sx - 1 ? 0 : XS;
      const int ozm = gz == 0 ? 0 : -1, ozp = gz == d.sz - 1 ? 0 : 1;
      const float* S = smem + par * R::BUF + cx * XS + cz;
#pragma unroll
      for (int ly = 0; ly < EY; ++ly) {
        if (ly >= t.cy0 && ly < t.cy1 && ((fl >> ly) & 1ull)) {
          const int gy = t.ey + ly;
          const int i = ly * EZ;
          const float self = p[ly];
          const float ym = (gy == 0 || ly == 0) ? self : p[ly > 0 ? ly - 1 : 0];
          const float yp = (gy == d.sy - 1 || ly + 1 >= EY) ? self : p[ly + 1 < EY ? ly + 1 : ly];
          double s = (double)S[i + oxp];
          s += (double)S[i + oxm];
          s += (double)yp;
          s += (double)ym;
          s += (double)S[i + ozp];
          s += (double)S[i + ozm];
          const double r = (double)b[ly] + s - 6.0 * (double)self;
          acc += r * r;
        }
        if ((ly & 7) == 7) asm volatile("" ::: "memory");
      }
    }
    return cta_sum<R::THREADS>(acc, s_red);
  };

  // This thread's own cells of box t from p into dst.
  auto store = [&](const Box& t, float* __restrict__ dst) {
    const bool own = thr && cx >= t.cx0 && cx < t.cx1 && cz >= t.cz0 && cz < t.cz1;
    if (own) {
      const int base = ((t.ex + cx) * d.sy + t.ey) * d.sz + t.ez + cz;
#pragma unroll
      for (int ly = 0; ly < EY; ++ly)
        if (ly >= t.cy0 && ly < t.cy1) dst[base + ly * d.sz] = p[ly];
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
        const bool own = thr && cx >= t.cx0 && cx < t.cx1 && cz >= t.cz0 && cz < t.cz1;
        if (own) {
          const int base = ((t.ex + cx) * d.sy + t.ey) * d.sz + t.ez + cz;
          for (int ly = t.cy0; ly < t.cy1; ++ly) pa[base + ly * d.sz] = __ldcg(pb + base + ly * d.sz);
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
constexpr ShapeInfo kShapes[] = {{8, 40, 16}, {8, 32, 16}, {16, 16, 16}, {8, 24, 16}, {8, 16, 16}, {16, 24, 16}};
constexpr int kNumShapes = sizeof(kShapes) / sizeof(kShapes[0]);

template <int TX, int TY, int TZ, int K>
cudaError_t launch_res(cudaStream_t st, const Dims& d, int ctas, float* pa, float* pb, const float* rhs,
                       const int8_t* type, const int* tiles, const int* n_tiles, unsigned int* bar, double* part,
                       SolveState* ss, int fixed_sweeps, int check, int max_iters, double tol, BarrierTest bt) {
  using R = Res<TX, TY, TZ, K>;
  auto fn = &k_resident_solve<TX, TY, TZ, K>;
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

template <int TX, int TY, int TZ, int K>
int occupancy_of(int device) {
  using R = Res<TX, TY, TZ, K>;
  auto fn = &k_resident_solve<TX, TY, TZ, K>;
  if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, R::SMEM) != cudaSuccess) return 0;
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, R::THREADS, R::SMEM) != cudaSuccess) return 0;
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  return per_sm >= 1 ? sms : 0;  // one CTA per SM
}

// Dispatch over (shape, K): calls f.template operator()<TX, TY, TZ, K>().
template <typename F>
auto dispatch(int shape, int k, const F& f) -> decltype(f.template operator()<8, 40, 16, 4>()) {
#define AQ_RES_CASE(S, A, B, C)                                   \
  if (shape == S && k == 4) return f.template operator()<A, B, C, 4>(); \
  if (shape == S && k == 2) return f.template operator()<A, B, C, 2>();
  AQ_RES_CASE(0, 8, 40, 16)
  AQ_RES_CASE(1, 8, 32, 16)
  AQ_RES_CASE(2, 16, 16, 16)
  AQ_RES_CASE(3, 8, 24, 16)
  AQ_RES_CASE(4, 8, 16, 16)
  AQ_RES_CASE(5, 16, 24, 16)
#undef AQ_RES_CASE
  return decltype(f.template operator()<8, 40, 16, 4>())();
}

struct OccupancyOf {
  int device;
  template <int A, int B, int C, int D>
  int operator()() const { return occupancy_of<A, B, C, D>(device); }
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
  template <int A, int B, int C, int D>
  cudaError_t operator()() const {
    return launch_res<A, B, C, D>(st, d, ctas, pa, pb, rhs, type, tiles, n_tiles, bar, part, ss, fixed_sweeps, check,
                                  max_iters, tol, bt);
  }
};

}  // namespace

bool resident_plan_ok(int shape, int k) { return shape >= 0 && shape < kNumShapes && (k == 2 || k == 4); }

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
