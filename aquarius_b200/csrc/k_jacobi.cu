// Pressure Jacobi sweeps, temporally blocked (stage (c), hot loop #1).
//
// Reference: jacobiImpl (Fluid/Fluid_3D_kernels.cu:460-505), launched
// pressureIterations times (Fluid/Fluid_3D_common.cu:48-55).  Per fluid cell
//   p' = (p[x+1] + p[x-1] + p[y+1] + p[y-1] + p[z+1] + p[z-1] + rhs) / 6,
// rhs = -div*rho, air cells 0, out-of-domain neighbours clamped to the cell
// itself (Neumann walls), summed in that order.  The reference updates in
// place; this is the race-free Jacobi reading of it (ping-pong buffers).
//
// Blocking: a CTA of 32 x BY threads owns one (y,z) column each of a tile
// with an H-cell halo and streams along x over `xc` output planes.  Level 0
// loads a plane; level l = 1..L computes plane xi-l from level l-1.  Each
// thread keeps the three x-neighbours of every level in registers; the four
// in-plane neighbours come from a double-buffered shared-memory plane per
// level.  Only level L is written back, so HBM/L2 traffic per sweep is about
// 1/L of a plain sweep.  With RESID an extra level evaluates the FP64
// residual b - A p of the written iterate on the CTA's output cells.
#include <algorithm>
#include <type_traits>

#include "aq_kernels.cuh"

namespace aqb {
namespace {

template <int L, bool RESID, int BY>
__global__ void __launch_bounds__(32 * BY) k_jacobi(Dims d, int xc, const float* __restrict__ pin,
                                                   float* __restrict__ pout, const float* __restrict__ rhs,
                                                   const int8_t* __restrict__ type,
                                                   const uint8_t* __restrict__ bact, double* __restrict__ part) {
  constexpr int H = L + (RESID ? 1 : 0);
  constexpr int TZ = 32 - 2 * H;
  constexpr int TY = BY - 2 * H;
  static_assert(TZ > 0 && TY > 0, "tile too small for the halo");
  extern __shared__ float smem[];  // [2][H][BY][32]
  __shared__ int s_active;
  __shared__ double s_red[BY];

  const int tz = threadIdx.x, ty = threadIdx.y;
  const int tid = ty * 32 + tz;
  const int z0 = blockIdx.x * TZ, y0 = blockIdx.y * TY, x0 = blockIdx.z * xc;
  const int z = z0 - H + tz, y = y0 - H + ty;
  const int x_end = min(x0 + xc, d.sx);
  const bool col_in = z >= 0 && z < d.sz && y >= 0 && y < d.sy;
  const bool col_out = col_in && tz >= H && tz < H + TZ && ty >= H && ty < H + TY;
  const int bid = (blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;

  // Skip tiles whose output region holds no fluid: it is all air, 0 in both
  // buffers, and stays so for the whole solve.
  if (tid == 0) s_active = 0;
  __syncthreads();
  {
    const int bx0 = x0 / kBrick, bx1 = (x_end - 1) / kBrick;
    const int by0 = y0 / kBrick, by1 = (min(y0 + TY, d.sy) - 1) / kBrick;
    const int bz0 = z0 / kBrick, bz1 = (min(z0 + TZ, d.sz) - 1) / kBrick;
    const int nbz = bz1 - bz0 + 1, nby = by1 - by0 + 1, nbx = bx1 - bx0 + 1;
    const int total = nbx * nby * nbz;
    for (int k = tid; k < total; k += 32 * BY) {
      const int kz = k % nbz, ky = (k / nbz) % nby, kx = k / (nbz * nby);
      if (bact[((bx0 + kx) * d.by + (by0 + ky)) * d.bz + (bz0 + kz)]) s_active = 1;
    }
  }
  __syncthreads();
  if (!s_active) {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;");
    if (RESID && tid == 0) part[bid] = 0.0;
    return;
  }

  // programmatic dependent launch: the previous sweep must be complete (and
  // done reading the buffer this launch writes) before any buffer access
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;");

  float R[H][3];
  float rq[H + 1];
  unsigned tq = 0;
#pragma unroll
  for (int l = 0; l < H; ++l) R[l][0] = R[l][1] = R[l][2] = 0.f;
#pragma unroll
  for (int k = 0; k <= H; ++k) rq[k] = 0.f;
  double racc = 0.0;

  const int tym = max(ty - 1, 0), typ = min(ty + 1, BY - 1);
  const int tzm = max(tz - 1, 0), tzp = min(tz + 1, 31);
  const bool has_ym = y - 1 >= 0, has_yp = y + 1 < d.sy;
  const bool has_zm = z - 1 >= 0, has_zp = z + 1 < d.sz;
  const int plane = d.sy * d.sz;
  const int colofs = y * d.sz + z;

  const int xs = max(x0 - H, 0);
  const int xlast = x_end - 1 + H;
  int par = 0;
  for (int xi = xs; xi <= xlast; ++xi, par ^= 1) {
    float pv = 0.f, rv = 0.f;
    unsigned tv = 0;
    if (col_in && xi < d.sx) {
      const int c = xi * plane + colofs;
      pv = pin[c];
      rv = rhs[c];
      tv = type[c] == kFluid ? 1u : 0u;
    }
    R[0][0] = R[0][1];
    R[0][1] = R[0][2];
    R[0][2] = pv;
#pragma unroll
    for (int k = H; k > 0; --k) rq[k] = rq[k - 1];
    rq[0] = rv;
    tq = (tq << 1) | tv;

#pragma unroll
    for (int l = 1; l <= H; ++l) {
      float* E = smem + ((par * H + (l - 1)) * BY) * 32;
      E[ty * 32 + tz] = R[l - 1][1];
      __syncthreads();
      const int c = xi - l;
      const float self = R[l - 1][1];
      const float xm = c - 1 >= 0 ? R[l - 1][0] : self;
      const float xp = c + 1 < d.sx ? R[l - 1][2] : self;
      const float ym = has_ym ? E[tym * 32 + tz] : self;
      const float yp = has_yp ? E[typ * 32 + tz] : self;
      const float zm = has_zm ? E[ty * 32 + tzm] : self;
      const float zp = has_zp ? E[ty * 32 + tzp] : self;
      const bool fl = (tq >> l) & 1u;
      if (l <= L) {
        float s = xp + xm;
        s += yp;
        s += ym;
        s += zp;
        s += zm;
        s += rq[l];
        const float nv = fl ? __fdiv_rn(s, 6.f) : 0.f;
        if (l < H) {
          R[l][0] = R[l][1];
          R[l][1] = R[l][2];
          R[l][2] = nv;
        }
        if (l == L && col_out && c >= x0 && c < x_end) pout[c * plane + colofs] = nv;
      } else if (RESID) {
        if (fl && col_out && c >= x0 && c < x_end) {
          double s = (double)xp;
          s += (double)xm;
          s += (double)yp;
          s += (double)ym;
          s += (double)zp;
          s += (double)zm;
          const double r = (double)rq[l] + s - 6.0 * (double)self;
          racc += r * r;
        }
      }
    }
  }

  if (RESID) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) racc += __shfl_xor_sync(0xffffffffu, racc, o);
    if (tz == 0) s_red[ty] = racc;
    __syncthreads();
    if (tid == 0) {
      double t = 0.0;
      for (int k = 0; k < BY; ++k) t += s_red[k];
      part[bid] = t;
    }
  }
}


// One sweep per launch, 4 consecutive z cells per thread (float4).  A block
// is 8 warps (rows y) x 32 lanes (z-quads, 128 cells) and streams XS
// consecutive x planes, keeping the x-1, x, x+1 planes of its quads in
// registers and prefetching the next one; y neighbours come from L1/L2, z
// neighbours across lanes by warp shuffle.  Each warp checks the activity
// bricks of its own rows itself (no block barrier) and leaves if none holds
// fluid.  Needs sz % 4 == 0.
__device__ __forceinline__ bool warp_active(const Dims& d, const uint8_t* __restrict__ bact, int x0, int x1, int y,
                                            int zb0) {
  // bricks: x in [x0/8, (x1-1)/8], one y brick, z bricks zb0 .. zb0+15
  const int lane = threadIdx.x;
  int a = 0;
  if (lane < 16 && zb0 + lane < d.bz)
    for (int bx = x0 / kBrick; bx <= (x1 - 1) / kBrick; ++bx)
      a |= bact[(bx * d.by + y / kBrick) * d.bz + zb0 + lane];
  return __any_sync(0xffffffffu, a) != 0;
}

__device__ __forceinline__ float4 ld4(const float* p) { return __ldg(reinterpret_cast<const float4*>(p)); }

__host__ __device__ __forceinline__ int resid_flat_parts_dev(const Dims& d) {
  return ((d.sz / 4 + 31) / 32) * ((d.sy + 7) / 8) * d.sx;
}

// One Jacobi update of 4 consecutive z cells: p' = (x+1, x-1, y+1, y-1, z+1,
// z-1 summed in that order, + rhs) / 6 on fluid cells, 0 elsewhere.  Every
// sweep kernel uses this function, so they agree bit for bit.
__device__ __forceinline__ float4 jacobi_quad(const float4& xm, const float4& xp, const float4& ym, const float4& yp,
                                              const float4& pc, float zlo, float zhi, const float4& b,
                                              const char4& t) {
  float4 o;
  {
    float s = xp.x + xm.x; s += yp.x; s += ym.x; s += pc.y; s += zlo; s += b.x;
    o.x = t.x == kFluid ? __fdiv_rn(s, 6.f) : 0.f;
  }
  {
    float s = xp.y + xm.y; s += yp.y; s += ym.y; s += pc.z; s += pc.x; s += b.y;
    o.y = t.y == kFluid ? __fdiv_rn(s, 6.f) : 0.f;
  }
  {
    float s = xp.z + xm.z; s += yp.z; s += ym.z; s += pc.w; s += pc.y; s += b.z;
    o.z = t.z == kFluid ? __fdiv_rn(s, 6.f) : 0.f;
  }
  {
    float s = xp.w + xm.w; s += yp.w; s += ym.w; s += zhi; s += pc.z; s += b.w;
    o.w = t.w == kFluid ? __fdiv_rn(s, 6.f) : 0.f;
  }
  return o;
}

// (bx, by, bz) = (z-quad block, row block, x-plane group) of the flat grid;
// the caller has checked that the warp's rows hold fluid (warp_active).
template <int XS>
__device__ __forceinline__ void jacobi_row(const Dims& d, const float* __restrict__ pin, float* __restrict__ pout,
                                           const float* __restrict__ rhs, const int8_t* __restrict__ type, int bx,
                                           int y, int bz) {
  const int lane = threadIdx.x;
  const int z = (bx * 32 + lane) * 4;
  const int x0 = bz * XS;
  const int x1 = min(x0 + XS, d.sx);
  const bool in = z < d.sz;
  const int plane = d.sy * d.sz;
  const int col = y * d.sz + z;
  const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f);
  // p at x-1, x, x+1 and the rest of plane x; with XS > 1 the loads of plane
  // x+1 are issued before plane x's arithmetic (software pipelining along x)
  float4 pm = zero, pc = zero, pp = zero, ym = zero, yp = zero, b = zero;
  char4 t = make_char4(0, 0, 0, 0);
  if (in) {
    const int c = x0 * plane + col;
    pc = ld4(pin + c);
    pm = x0 > 0 ? ld4(pin + c - plane) : pc;
    pp = x0 + 1 < d.sx ? ld4(pin + c + plane) : pc;
    ym = y > 0 ? ld4(pin + c - d.sz) : pc;
    yp = y + 1 < d.sy ? ld4(pin + c + d.sz) : pc;
    b = ld4(rhs + c);
    t = *reinterpret_cast<const char4*>(type + c);
  }
  for (int x = x0; x < x1; ++x) {
    const int c = x * plane + col;
    float4 pn = pp, nym = pp, nyp = pp, nb = zero;
    char4 nt = make_char4(0, 0, 0, 0);
    if (in && x + 1 < x1) {
      const int cn = c + plane;
      if (x + 2 < d.sx) pn = ld4(pin + cn + plane);
      if (y > 0) nym = ld4(pin + cn - d.sz);
      if (y + 1 < d.sy) nyp = ld4(pin + cn + d.sz);
      nb = ld4(rhs + cn);
      nt = *reinterpret_cast<const char4*>(type + cn);
    }
    float zlo = __shfl_up_sync(0xffffffffu, pc.w, 1);
    float zhi = __shfl_down_sync(0xffffffffu, pc.x, 1);
    if (in) {
      if (lane == 0) zlo = z > 0 ? pin[c - 1] : pc.x;
      if (lane == 31 || z + 4 >= d.sz) zhi = z + 4 < d.sz ? pin[c + 4] : pc.w;
      *reinterpret_cast<float4*>(pout + c) = jacobi_quad(pm, pp, ym, yp, pc, zlo, zhi, b, t);
    }
    pm = pc;
    pc = pp;
    pp = (x + 2 < d.sx) ? pn : pc;
    ym = nym;
    yp = nyp;
    b = nb;
    t = nt;
  }
}

template <int XS>
__device__ __forceinline__ void jacobi_flat_body(const Dims& d, const float* __restrict__ pin,
                                                 float* __restrict__ pout, const float* __restrict__ rhs,
                                                 const int8_t* __restrict__ type, int bx, int by, int bz) {
  jacobi_row<XS>(d, pin, pout, rhs, type, bx, by * 8 + threadIdx.y, bz);
}

// jacobi_row<1> of row (x, y, z block zb) with its rhs and types loaded.
__device__ __forceinline__ void jacobi_row_pre(const Dims& d, const float* __restrict__ pin, float* __restrict__ pout,
                                               int x, int y, int zb, const float4& b, const char4& t) {
  const int lane = threadIdx.x;
  const int z = (zb * 32 + lane) * 4;
  const bool in = z < d.sz;
  const int plane = d.sy * d.sz;
  const int c = (x * d.sy + y) * d.sz + z;
  float4 pc = make_float4(0.f, 0.f, 0.f, 0.f), pm = pc, pp = pc, ym = pc, yp = pc;
  if (in) {
    pc = ld4(pin + c);
    pm = x > 0 ? ld4(pin + c - plane) : pc;
    pp = x + 1 < d.sx ? ld4(pin + c + plane) : pc;
    ym = y > 0 ? ld4(pin + c - d.sz) : pc;
    yp = y + 1 < d.sy ? ld4(pin + c + d.sz) : pc;
  }
  float zlo = __shfl_up_sync(0xffffffffu, pc.w, 1);
  float zhi = __shfl_down_sync(0xffffffffu, pc.x, 1);
  if (in) {
    if (lane == 0) zlo = z > 0 ? pin[c - 1] : pc.x;
    if (lane == 31 || z + 4 >= d.sz) zhi = z + 4 < d.sz ? pin[c + 4] : pc.w;
    *reinterpret_cast<float4*>(pout + c) = jacobi_quad(pm, pp, ym, yp, pc, zlo, zhi, b, t);
  }
}

// List plan: one sweep of the warp rows (x, y, 128-wide z block) that hold
// fluid, from a list built once per solve (k_row_items).  A resident wave of
// CTAs walks the list, so no CTA is scheduled only to find its rows empty.
// Same arithmetic as the flat sweep (jacobi_quad).
__global__ void __launch_bounds__(256, 6) k_jacobi_list(Dims d, const float* __restrict__ pin, float* __restrict__ pout,
                                                    const float* __restrict__ rhs, const int8_t* __restrict__ type,
                                                    const int* __restrict__ items, const int* __restrict__ n_items,
                                                    int early) {
  const int W = blockDim.y;
  const int gz = (d.sz / 4 + 31) / 32;
  int it = blockIdx.x * W + threadIdx.y;
  int n = 0;
  // early (every sweep of a block but the first): the list, rhs and types
  // were written before the previous sweep was launched, so the warp's first
  // row is decoded and its rhs and types loaded before waiting for that sweep
  bool pre = false;
  int x0 = 0, y0 = 0, zb0 = 0;
  float4 b0 = make_float4(0.f, 0.f, 0.f, 0.f);
  char4 t0 = make_char4(0, 0, 0, 0);
  if (early) {
    n = *n_items;
    if (it < n) {
      const int id = __ldg(items + it);
      zb0 = id % gz;
      const int t = id / gz;
      y0 = t % d.sy;
      x0 = t / d.sy;
      const int z = (zb0 * 32 + threadIdx.x) * 4;
      if (z < d.sz) {
        const int c = (x0 * d.sy + y0) * d.sz + z;
        b0 = ld4(rhs + c);
        t0 = *reinterpret_cast<const char4*>(type + c);
      }
      pre = true;
    }
  }
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;");
  if (!early) n = *n_items;
  if (pre) {
    jacobi_row_pre(d, pin, pout, x0, y0, zb0, b0, t0);
    it += gridDim.x * W;
  }
  for (; it < n; it += gridDim.x * W) {
    const int id = __ldg(items + it);
    const int zb = id % gz, t = id / gz;
    jacobi_row<1>(d, pin, pout, rhs, type, zb, t % d.sy, t / d.sy);
  }
}

// Ordered list of the active warp rows: id = (x * sy + y) * gz + zb for every
// row whose 8^3 bricks (x/8, y/8, 16 z bricks of block zb) hold fluid.
__global__ void __launch_bounds__(1024) k_row_items(Dims d, const uint8_t* __restrict__ bact, int* __restrict__ items,
                                                   int* __restrict__ n_items) {
  __shared__ int s_cnt[32], s_pre[32];
  __shared__ int s_tot, s_base;
  const int gz = (d.sz / 4 + 31) / 32;
  const int total = d.sx * d.sy * gz;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (threadIdx.x == 0) s_base = 0;
  __syncthreads();
  for (int base = 0; base < total; base += 1024) {
    const int id = base + threadIdx.x;
    int a = 0;
    if (id < total) {
      const int zb = id % gz, t = id / gz, y = t % d.sy, x = t / d.sy;
      for (int k = 0; k < 16 && zb * 16 + k < d.bz && !a; ++k)
        a = bact[((x / kBrick) * d.by + y / kBrick) * d.bz + zb * 16 + k] ? 1 : 0;
    }
    const unsigned m = __ballot_sync(0xffffffffu, a);
    const int pre = __popc(m & ((1u << lane) - 1u));
    if (lane == 0) s_cnt[w] = __popc(m);
    __syncthreads();
    if (w == 0) {
      const int v = s_cnt[lane];
      int incl = v;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int tt = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += tt;
      }
      s_pre[lane] = incl - v;
      if (lane == 31) s_tot = incl;
    }
    __syncthreads();
    if (a) items[s_base + s_pre[w] + pre] = id;
    __syncthreads();
    if (threadIdx.x == 0) s_base += s_tot;
    __syncthreads();
  }
  if (threadIdx.x == 0) *n_items = s_base;
}

// Programmatic dependent launch: the activity bricks were written two or more
// launches earlier, so only the pressure reads wait for the previous sweep.
template <int XS>
__global__ void __launch_bounds__(256) k_jacobi_flat(Dims d, const float* __restrict__ pin,
                                                    float* __restrict__ pout, const float* __restrict__ rhs,
                                                    const int8_t* __restrict__ type,
                                                    const uint8_t* __restrict__ bact) {
  const int y = blockIdx.y * 8 + threadIdx.y;
  const int x0 = blockIdx.z * XS;
  const bool act = y < d.sy && warp_active(d, bact, x0, min(x0 + XS, d.sx), y, blockIdx.x * 16);
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;");
  if (!act) return;
  jacobi_flat_body<XS>(d, pin, pout, rhs, type, blockIdx.x, blockIdx.y, blockIdx.z);
}

// FP64 residual ||b - A p||^2 of one iterate over fluid cells, in the flat
// layout (one x plane x 8 rows x 128 z per block); per-block partial sums in
// a fixed order.
__device__ __forceinline__ void resid_flat_body(const Dims& d, const float* __restrict__ p,
                                                const float* __restrict__ rhs, const int8_t* __restrict__ type,
                                                const uint8_t* __restrict__ bact, double* __restrict__ part, int bx,
                                                int by, int bz) {
  const int lane = threadIdx.x;
  const int z = (bx * 32 + lane) * 4;
  const int y = by * 8 + threadIdx.y;
  const int x = bz;
  const int bid = (bz * ((d.sy + 7) / 8) + by) * ((d.sz / 4 + 31) / 32) + bx;
  const bool act = y < d.sy && warp_active(d, bact, x, x + 1, y, bx * 16);
  double acc = 0.0;
  const bool in = act && z < d.sz;
  const int plane = d.sy * d.sz;
  const int c = x * plane + y * d.sz + z;
  float4 pc = make_float4(0.f, 0.f, 0.f, 0.f);
  if (in) pc = ld4(p + c);
  float zlo = __shfl_up_sync(0xffffffffu, pc.w, 1);
  float zhi = __shfl_down_sync(0xffffffffu, pc.x, 1);
  if (in) {
    if (lane == 0) zlo = z > 0 ? p[c - 1] : pc.x;
    if (lane == 31 || z + 4 >= d.sz) zhi = z + 4 < d.sz ? p[c + 4] : pc.w;
    const float4 xm = x > 0 ? ld4(p + c - plane) : pc;
    const float4 xp = x + 1 < d.sx ? ld4(p + c + plane) : pc;
    const float4 ym = y > 0 ? ld4(p + c - d.sz) : pc;
    const float4 yp = y + 1 < d.sy ? ld4(p + c + d.sz) : pc;
    const float4 b = ld4(rhs + c);
    const char4 t = *reinterpret_cast<const char4*>(type + c);
    const float self[4] = {pc.x, pc.y, pc.z, pc.w};
    const float zp[4] = {pc.y, pc.z, pc.w, zhi};
    const float zm[4] = {zlo, pc.x, pc.y, pc.z};
    const float vxp[4] = {xp.x, xp.y, xp.z, xp.w}, vxm[4] = {xm.x, xm.y, xm.z, xm.w};
    const float vyp[4] = {yp.x, yp.y, yp.z, yp.w}, vym[4] = {ym.x, ym.y, ym.z, ym.w};
    const float vb[4] = {b.x, b.y, b.z, b.w};
    const signed char vt[4] = {t.x, t.y, t.z, t.w};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      if (vt[k] != kFluid) continue;
      double s = (double)vxp[k];
      s += (double)vxm[k];
      s += (double)vyp[k];
      s += (double)vym[k];
      s += (double)zp[k];
      s += (double)zm[k];
      const double r = (double)vb[k] + s - 6.0 * (double)self[k];
      acc += r * r;
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  __shared__ double s_red[8];
  if (lane == 0) s_red[threadIdx.y] = acc;
  __syncthreads();
  if (threadIdx.x == 0 && threadIdx.y == 0) {
    double t = 0.0;
    for (int k = 0; k < 8; ++k) t += s_red[k];
    part[bid] = t;
  }
}

__global__ void __launch_bounds__(256) k_resid_flat(Dims d, const float* __restrict__ p,
                                                   const float* __restrict__ rhs, const int8_t* __restrict__ type,
                                                   const uint8_t* __restrict__ bact, double* __restrict__ part) {
  resid_flat_body(d, p, rhs, type, bact, part, blockIdx.x, blockIdx.y, blockIdx.z);
}


// ------------------------------------------------------------- cube tiles
// Temporally blocked sweep on 3D tiles held in shared memory: a CTA loads a
// (TX+2L) x (TX+2L) x 32 block of cells (its core TX x TX x (32-2L) plus an
// L-cell halo), runs L sweeps on it and writes the core.  Sweep s updates the
// cells at distance >= s from the block faces, whose neighbours were all
// updated by sweep s-1, so the core ends exactly as after L separate sweeps
// (same arithmetic, jacobi_quad's summation order).  Warps own block rows
// (x, y) with lanes along z: a lane keeps its cells' pressure, rhs and
// fluid/in-grid bits in registers across the sweeps; x and y neighbours come
// from a shared-memory ping-pong, z neighbours by warp shuffle.
template <int L, int TX>
struct CubeShape {
  static constexpr int E = TX + 2 * L;  // block rows per axis (x, y)
  static constexpr int TZ = 32 - 2 * L;  // core along z
  static constexpr int ROWS = E * E;
};

template <int L, int TX, int WARPS>
__global__ void __launch_bounds__(WARPS * 32) k_jacobi_cube(Dims d, const float* __restrict__ pin,
                                                           float* __restrict__ pout, const float* __restrict__ rhs,
                                                           const int8_t* __restrict__ type,
                                                           const uint8_t* __restrict__ bact) {
  using S = CubeShape<L, TX>;
  constexpr int E = S::E, TZ = S::TZ, ROWS = S::ROWS;
  constexpr int R = (ROWS + WARPS - 1) / WARPS;
  using Mask = typename std::conditional<(R > 32), unsigned long long, unsigned>::type;
  extern __shared__ __align__(16) float cube_smem[];  // [2][ROWS][32]
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int x0 = blockIdx.z * TX, y0 = blockIdx.y * TX, z0 = blockIdx.x * TZ;
  // skip blocks whose core holds no fluid (their cells stay 0 in both buffers)
  int a = 0;
  {
    const int bx0 = x0 / kBrick, bx1 = (min(x0 + TX, d.sx) - 1) / kBrick;
    const int by0 = y0 / kBrick, by1 = (min(y0 + TX, d.sy) - 1) / kBrick;
    const int bz0 = z0 / kBrick, bz1 = (min(z0 + TZ, d.sz) - 1) / kBrick;
    const int nbx = bx1 - bx0 + 1, nby = by1 - by0 + 1, nbz = bz1 - bz0 + 1;
    for (int k = threadIdx.x; k < nbx * nby * nbz; k += WARPS * 32) {
      const int iz = k % nbz, t = k / nbz, iy = t % nby, ix = t / nby;
      a |= bact[((bx0 + ix) * d.by + by0 + iy) * d.bz + bz0 + iz];
    }
  }
  const bool active = __syncthreads_or(a) != 0;
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;");
  if (!active) return;
  const int gz = z0 - L + lane;
  const bool zin = gz >= 0 && gz < d.sz;
  float p[R], b[R];
  Mask fluid = 0, ing = 0;
  float* buf0 = cube_smem;
#pragma unroll
  for (int k = 0; k < R; ++k) {
    const int r = warp + WARPS * k;
    p[k] = 0.f;
    b[k] = 0.f;
    if (r < ROWS) {
      const int gx = x0 - L + r / E, gy = y0 - L + r % E;
      if (zin && gx >= 0 && gx < d.sx && gy >= 0 && gy < d.sy) {
        const int c = (gx * d.sy + gy) * d.sz + gz;
        p[k] = pin[c];
        b[k] = rhs[c];
        ing |= Mask(1) << k;
        if (type[c] == kFluid) fluid |= Mask(1) << k;
      }
      buf0[r * 32 + lane] = p[k];
    }
  }
  __syncthreads();
#pragma unroll 1
  for (int s = 1; s <= L; ++s) {
    const float* src = cube_smem + ((s - 1) & 1) * ROWS * 32;
    float* dst = cube_smem + (s & 1) * ROWS * 32;
    const bool zok = lane >= s && lane < 32 - s;
#pragma unroll
    for (int k = 0; k < R; ++k) {
      const int r = warp + WARPS * k;
      if (r >= ROWS) continue;
      const int lx = r / E, ly = r % E;
      if (lx < s || lx >= E - s || ly < s || ly >= E - s) continue;  // warp-uniform
      const float c = p[k];
      const float zmv = __shfl_up_sync(0xffffffffu, c, 1);
      const float zpv = __shfl_down_sync(0xffffffffu, c, 1);
      if (zok && ((ing >> k) & 1)) {
        const int gx = x0 - L + lx, gy = y0 - L + ly;
        const float xp = gx + 1 < d.sx ? src[(r + E) * 32 + lane] : c;
        const float xm = gx > 0 ? src[(r - E) * 32 + lane] : c;
        const float yp = gy + 1 < d.sy ? src[(r + 1) * 32 + lane] : c;
        const float ym = gy > 0 ? src[(r - 1) * 32 + lane] : c;
        const float zp = gz + 1 < d.sz ? zpv : c;
        const float zm = gz > 0 ? zmv : c;
        float sum = xp + xm;
        sum += yp;
        sum += ym;
        sum += zp;
        sum += zm;
        sum += b[k];
        const float v = ((fluid >> k) & 1) ? __fdiv_rn(sum, 6.f) : 0.f;
        p[k] = v;
        dst[r * 32 + lane] = v;
      }
    }
    __syncthreads();
  }
  if (lane < L || lane >= L + TZ || !zin) return;
#pragma unroll
  for (int k = 0; k < R; ++k) {
    const int r = warp + WARPS * k;
    if (r >= ROWS) continue;
    const int lx = r / E, ly = r % E;
    if (lx < L || lx >= L + TX || ly < L || ly >= L + TX) continue;
    if ((ing >> k) & 1) pout[((x0 - L + lx) * d.sy + (y0 - L + ly)) * d.sz + gz] = p[k];
  }
}

template <int L, int TX, int WARPS>
cudaError_t launch_cube(cudaStream_t st, const Dims& d, const float* pin, float* pout, const float* rhs,
                        const int8_t* type, const uint8_t* bact) {
  using S = CubeShape<L, TX>;
  constexpr size_t smem = (size_t)2 * S::ROWS * 32 * sizeof(float);
  static const cudaError_t attr = cudaFuncSetAttribute(
      k_jacobi_cube<L, TX, WARPS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (attr != cudaSuccess) return attr;
  cudaLaunchConfig_t lc = {};
  lc.gridDim = dim3((d.sz + S::TZ - 1) / S::TZ, (d.sy + TX - 1) / TX, (d.sx + TX - 1) / TX);
  lc.blockDim = dim3(WARPS * 32);
  lc.dynamicSmemBytes = smem;
  lc.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  lc.attrs = at;
  lc.numAttrs = 1;
  return cudaLaunchKernelEx(&lc, k_jacobi_cube<L, TX, WARPS>, d, pin, pout, rhs, type, bact);
}

// Cube plans: (levels, TX) -> warps per CTA.
cudaError_t dispatch_cube(cudaStream_t st, const Dims& d, int levels, int tx, const float* pin, float* pout,
                          const float* rhs, const int8_t* type, const uint8_t* bact) {
  if (levels == 1 && tx == 8) return launch_cube<1, 8, 4>(st, d, pin, pout, rhs, type, bact);
  if (levels == 2 && tx == 8) return launch_cube<2, 8, 8>(st, d, pin, pout, rhs, type, bact);
  if (levels == 3 && tx == 8) return launch_cube<3, 8, 8>(st, d, pin, pout, rhs, type, bact);
  if (levels == 4 && tx == 8) return launch_cube<4, 8, 16>(st, d, pin, pout, rhs, type, bact);
  if (levels == 1 && tx == 16) return launch_cube<1, 16, 16>(st, d, pin, pout, rhs, type, bact);
  if (levels == 2 && tx == 16) return launch_cube<2, 16, 16>(st, d, pin, pout, rhs, type, bact);
  if (levels == 4 && tx == 16) return launch_cube<4, 16, 16>(st, d, pin, pout, rhs, type, bact);
  return cudaErrorInvalidValue;
}


// ---------------------------------------------------------------- persistent
// Flat work item id = (x * gy + yb) * gz + zb, gy = ceil(sy/8), gz = ceil(sz/128).
__device__ __forceinline__ void item_coords(const Dims& d, int id, int& x, int& yb, int& zb) {
  const int gz = (d.sz / 4 + 31) / 32, gy = (d.sy + 7) / 8;
  zb = id % gz;
  const int t = id / gz;
  yb = t % gy;
  x = t / gy;
}

// One Jacobi sweep of one item by a 256-thread CTA (8 warps = 8 rows).  The
// ping-pong buffers are rewritten by other SMs between sweeps of the same
// launch, so their loads bypass L1 (ld.global.cg); rhs and type are constant.
__device__ __forceinline__ void sweep_item(const Dims& d, int id, const float* __restrict__ pin,
                                           float* __restrict__ pout, const float* __restrict__ rhs,
                                           const int8_t* __restrict__ type) {
  int x, yb, zb;
  item_coords(d, id, x, yb, zb);
  const int lane = threadIdx.x & 31, row = (threadIdx.x & 255) >> 5;
  const int y = yb * 8 + row;
  if (y >= d.sy) return;  // warp-uniform
  const int z = (zb * 32 + lane) * 4;
  const bool in = z < d.sz;
  const int plane = d.sy * d.sz;
  const int c = x * plane + y * d.sz + z;
  float4 p = make_float4(0.f, 0.f, 0.f, 0.f);
  if (in) p = __ldcg(reinterpret_cast<const float4*>(pin + c));
  float zlo = __shfl_up_sync(0xffffffffu, p.w, 1);
  float zhi = __shfl_down_sync(0xffffffffu, p.x, 1);
  if (!in) return;
  if (lane == 0) zlo = z > 0 ? __ldcg(pin + c - 1) : p.x;
  if (lane == 31 || z + 4 >= d.sz) zhi = z + 4 < d.sz ? __ldcg(pin + c + 4) : p.w;
  const float4 xp = x + 1 < d.sx ? __ldcg(reinterpret_cast<const float4*>(pin + c + plane)) : p;
  const float4 xm = x > 0 ? __ldcg(reinterpret_cast<const float4*>(pin + c - plane)) : p;
  const float4 yp = y + 1 < d.sy ? __ldcg(reinterpret_cast<const float4*>(pin + c + d.sz)) : p;
  const float4 ym = y > 0 ? __ldcg(reinterpret_cast<const float4*>(pin + c - d.sz)) : p;
  const float4 b = __ldg(reinterpret_cast<const float4*>(rhs + c));
  const char4 t = *reinterpret_cast<const char4*>(type + c);
  float4 o;
  {
    float s = xp.x + xm.x; s += yp.x; s += ym.x; s += p.y; s += zlo; s += b.x;
    o.x = t.x == kFluid ? __fdiv_rn(s, 6.f) : 0.f;
  }
  {
    float s = xp.y + xm.y; s += yp.y; s += ym.y; s += p.z; s += p.x; s += b.y;
    o.y = t.y == kFluid ? __fdiv_rn(s, 6.f) : 0.f;
  }
  {
    float s = xp.z + xm.z; s += yp.z; s += ym.z; s += p.w; s += p.y; s += b.z;
    o.z = t.z == kFluid ? __fdiv_rn(s, 6.f) : 0.f;
  }
  {
    float s = xp.w + xm.w; s += yp.w; s += ym.w; s += zhi; s += p.z; s += b.w;
    o.w = t.w == kFluid ? __fdiv_rn(s, 6.f) : 0.f;
  }
  *reinterpret_cast<float4*>(pout + c) = o;
}

// ||b - A p||^2 of one item's fluid cells (per thread).
__device__ __forceinline__ double resid_item(const Dims& d, int id, const float* __restrict__ pv,
                                             const float* __restrict__ rhs, const int8_t* __restrict__ type) {
  int x, yb, zb;
  item_coords(d, id, x, yb, zb);
  const int lane = threadIdx.x & 31, row = (threadIdx.x & 255) >> 5;
  const int y = yb * 8 + row;
  if (y >= d.sy) return 0.0;
  const int z = (zb * 32 + lane) * 4;
  const bool in = z < d.sz;
  const int plane = d.sy * d.sz;
  const int c = x * plane + y * d.sz + z;
  float4 pc = make_float4(0.f, 0.f, 0.f, 0.f);
  if (in) pc = __ldcg(reinterpret_cast<const float4*>(pv + c));
  float zlo = __shfl_up_sync(0xffffffffu, pc.w, 1);
  float zhi = __shfl_down_sync(0xffffffffu, pc.x, 1);
  if (!in) return 0.0;
  if (lane == 0) zlo = z > 0 ? __ldcg(pv + c - 1) : pc.x;
  if (lane == 31 || z + 4 >= d.sz) zhi = z + 4 < d.sz ? __ldcg(pv + c + 4) : pc.w;
  const float4 xm = x > 0 ? __ldcg(reinterpret_cast<const float4*>(pv + c - plane)) : pc;
  const float4 xp = x + 1 < d.sx ? __ldcg(reinterpret_cast<const float4*>(pv + c + plane)) : pc;
  const float4 ym = y > 0 ? __ldcg(reinterpret_cast<const float4*>(pv + c - d.sz)) : pc;
  const float4 yp = y + 1 < d.sy ? __ldcg(reinterpret_cast<const float4*>(pv + c + d.sz)) : pc;
  const float4 b = __ldg(reinterpret_cast<const float4*>(rhs + c));
  const char4 t = *reinterpret_cast<const char4*>(type + c);
  const float self[4] = {pc.x, pc.y, pc.z, pc.w};
  const float zp[4] = {pc.y, pc.z, pc.w, zhi};
  const float zm[4] = {zlo, pc.x, pc.y, pc.z};
  const float vxp[4] = {xp.x, xp.y, xp.z, xp.w}, vxm[4] = {xm.x, xm.y, xm.z, xm.w};
  const float vyp[4] = {yp.x, yp.y, yp.z, yp.w}, vym[4] = {ym.x, ym.y, ym.z, ym.w};
  const float vb[4] = {b.x, b.y, b.z, b.w};
  const signed char vt[4] = {t.x, t.y, t.z, t.w};
  double acc = 0.0;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    if (vt[k] != kFluid) continue;
    double s = (double)vxp[k];
    s += (double)vxm[k];
    s += (double)vyp[k];
    s += (double)vym[k];
    s += (double)zp[k];
    s += (double)zm[k];
    const double r = (double)vb[k] + s - 6.0 * (double)self[k];
    acc += r * r;
  }
  return acc;
}

__device__ __forceinline__ unsigned ld_acquire(const unsigned int* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Grid barrier on a counter that only grows: arrival e of every CTA waits for
// e * gridDim.x arrivals.  Bounded: after spin_limit polls (kSpinLimit, about
// a second, unless a test shortens it) it sets *fail and returns false; after
// any failure every barrier returns false at once.
__device__ __forceinline__ bool grid_barrier(unsigned int* bar, unsigned target, int* fail, unsigned spin_limit) {
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
      while (ld_acquire(bar) < target) {
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

__global__ void __launch_bounds__(1024) k_items_compact(Dims d, const uint8_t* __restrict__ bact, int* __restrict__ items,
                                                        int* __restrict__ n_items, unsigned int* __restrict__ bar) {
  __shared__ int s_cnt[32], s_pre[32];
  __shared__ int s_tot, s_base;
  const int gz = (d.sz / 4 + 31) / 32, gy = (d.sy + 7) / 8;
  const int total = gz * gy * d.sx;
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
      int x, yb, zb;
      item_coords(d, id, x, yb, zb);
      for (int k = 0; k < 16 && zb * 16 + k < d.bz && !a; ++k)
        a = bact[((x / kBrick) * d.by + yb) * d.bz + zb * 16 + k] ? 1 : 0;
    }
    // ordered compaction: block-wide exclusive scan of the flags
    const unsigned m = __ballot_sync(0xffffffffu, a);
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
    if (a) items[s_base + s_pre[w] + pre] = id;
    __syncthreads();
    if (threadIdx.x == 0) s_base += s_tot;
    __syncthreads();
  }
  if (threadIdx.x == 0) *n_items = s_base;
}

__global__ void __launch_bounds__(1024) k_persist_solve(Dims d, float* __restrict__ pa, float* __restrict__ pb,
                                                      const float* __restrict__ rhs, const int8_t* __restrict__ type,
                                                      const int* __restrict__ items, const int* __restrict__ n_items,
                                                      unsigned int* __restrict__ bar, double* __restrict__ part,
                                                      SolveState* __restrict__ ss, int fixed_sweeps, int check,
                                                      int max_iters, double tol, BarrierTest bt) {
  __shared__ double s_red[32];
  __shared__ double s_r2;
  // one CTA per SM; four groups of 256 threads each sweep one item at a time
  const int P = gridDim.x, cta = blockIdx.x;
  // test hook: this CTA never arrives (a participant that does not join), so
  // the others' bounded barrier waits run out
  if (cta == bt.withhold_cta) return;
  const unsigned spin_limit = bt.spin_limit ? bt.spin_limit : kSpinLimit;
  const int G = 4, grp = threadIdx.x >> 8;
  const int first = cta * G + grp, stride = P * G;
  const int n = *n_items;
  int* fail = &ss->sync_timeout;
  unsigned epoch = 0;
  float* bufs[2] = {pa, pb};
  int cur = 0;
  int it = 0, checks = 0;
  bool ok = true;
  double r2 = -1.0, rel = -1.0;

  auto sweep = [&]() {
    for (int i = first; i < n; i += stride) sweep_item(d, items[i], bufs[cur], bufs[cur ^ 1], rhs, type);
    cur ^= 1;
    ++epoch;
    ok = ok && grid_barrier(bar, epoch * (unsigned)P, fail, spin_limit);
  };
  // residual of the current iterate; every CTA ends with the same r2
  auto residual = [&]() {
    double acc = 0.0;
    for (int i = first; i < n; i += stride) acc += resid_item(d, items[i], bufs[cur], rhs, type);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int k = 0; k < 32; ++k) t += s_red[k];
      part[cta] = t;
    }
    ++epoch;
    ok = ok && grid_barrier(bar, epoch * (unsigned)P, fail, spin_limit);
    if (threadIdx.x < 32) {
      double t = 0.0;
      for (int k = threadIdx.x; k < P; k += 32) t += *reinterpret_cast<volatile double*>(part + k);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
      if (threadIdx.x == 0) s_r2 = t;
    }
    __syncthreads();
    r2 = s_r2;
    rel = rel_residual_of(r2, ss->b2);
    ++checks;
  };

  if (fixed_sweeps > 0) {
    for (int k = 0; k < fixed_sweeps && ok; ++k) sweep();
    it = fixed_sweeps;
    if (ok) residual();
  } else {
    while (ok) {
      for (int k = 0; k < check && ok; ++k) sweep();
      it += check;
      if (!ok) break;
      residual();
      if (!(rel > tol) || !isfinite(rel) || it >= max_iters) break;
    }
  }
  // the result belongs in pa: copy this CTA's items when it ended in pb
  if (cur == 1) {
    for (int i = first; i < n; i += stride) {
      int x, yb, zb;
      item_coords(d, items[i], x, yb, zb);
      const int y = yb * 8 + ((threadIdx.x & 255) >> 5);
      const int z = (zb * 32 + (threadIdx.x & 31)) * 4;
      if (y < d.sy && z < d.sz) {
        const int c = x * d.sy * d.sz + y * d.sz + z;
        *reinterpret_cast<float4*>(pa + c) = __ldcg(reinterpret_cast<const float4*>(pb + c));
      }
    }
  }
  if (cta == 0 && threadIdx.x == 0) {
    ss->iterations = it;
    ss->bodies = checks;
    ss->total_sweeps += it;
    ss->total_bodies += checks;
    ss->r2 = r2;
    ss->rel_residual = rel;
    const bool finite = isfinite(rel);
    if (!finite) ss->nonfinite = ss->nonfinite_seen = 1;
    ss->converged = (ok && finite && rel >= 0.0 && rel <= tol) ? 1 : 0;
  }
}

// The solve state after a residual check of r2; whether the solve goes on.
__device__ __forceinline__ bool finalize_state(double r2, SolveState* __restrict__ ss, int sweeps, double tol,
                                               int max_iters);

// Returns (in thread 0) whether the solve should continue.
__device__ __forceinline__ bool resid_finalize_body(const double* __restrict__ part, int nparts,
                                                    SolveState* __restrict__ ss, int sweeps, double tol,
                                                    int max_iters) {
  __shared__ double sb[1024];
  double a = 0.0;
  for (int i = threadIdx.x; i < nparts; i += 1024) a += part[i];
  sb[threadIdx.x] = a;
  __syncthreads();
  for (int o = 512; o > 0; o >>= 1) {
    if (threadIdx.x < o) sb[threadIdx.x] += sb[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) return finalize_state(sb[0], ss, sweeps, tol, max_iters);
  return false;
}

__device__ __forceinline__ bool finalize_state(double r2, SolveState* __restrict__ ss, int sweeps, double tol,
                                               int max_iters) {
  ss->iterations += sweeps;
  ss->bodies += 1;
  ss->total_sweeps += sweeps;
  ss->total_bodies += 1;
  ss->r2 = r2;
  const double rel = rel_residual_of(r2, ss->b2);
  ss->rel_residual = rel;
  const bool finite = isfinite(rel);
  if (!finite) ss->nonfinite = ss->nonfinite_seen = 1;
  const bool conv = finite && rel <= tol;
  ss->converged = conv ? 1 : 0;
  return finite && !conv && ss->iterations < max_iters;
}

__global__ void __launch_bounds__(1024) k_resid_finalize(const double* __restrict__ part, int nparts,
                                                        SolveState* __restrict__ ss, int sweeps, double tol,
                                                        int max_iters, int set_cond,
                                                        cudaGraphConditionalHandle handle) {
  const bool more = resid_finalize_body(part, nparts, ss, sweeps, tol, max_iters);
  if (threadIdx.x == 0 && set_cond) cudaGraphSetConditional(handle, more ? 1u : 0u);
}

// The residual check of the list plan in one launch: each warp sums the
// FP64 residual of its listed rows (in list order), each CTA its warps in
// order, and the last CTA to finish (a ticket) sums the CTA partials as
// k_resid_finalize does and updates the solve state.
__device__ __forceinline__ double resid_row(const Dims& d, const float* __restrict__ p, const float* __restrict__ rhs,
                                            const int8_t* __restrict__ type, int x, int y, int zb) {
  const int lane = threadIdx.x;
  const int z = (zb * 32 + lane) * 4;
  const bool in = z < d.sz;
  const int plane = d.sy * d.sz;
  const int c = x * plane + y * d.sz + z;
  float4 pc = make_float4(0.f, 0.f, 0.f, 0.f);
  if (in) pc = ld4(p + c);
  float zlo = __shfl_up_sync(0xffffffffu, pc.w, 1);
  float zhi = __shfl_down_sync(0xffffffffu, pc.x, 1);
  double acc = 0.0;
  if (in) {
    if (lane == 0) zlo = z > 0 ? p[c - 1] : pc.x;
    if (lane == 31 || z + 4 >= d.sz) zhi = z + 4 < d.sz ? p[c + 4] : pc.w;
    const float4 xm = x > 0 ? ld4(p + c - plane) : pc;
    const float4 xp = x + 1 < d.sx ? ld4(p + c + plane) : pc;
    const float4 ym = y > 0 ? ld4(p + c - d.sz) : pc;
    const float4 yp = y + 1 < d.sy ? ld4(p + c + d.sz) : pc;
    const float4 b = ld4(rhs + c);
    const char4 t = *reinterpret_cast<const char4*>(type + c);
    const float self[4] = {pc.x, pc.y, pc.z, pc.w};
    const float zp[4] = {pc.y, pc.z, pc.w, zhi};
    const float zm[4] = {zlo, pc.x, pc.y, pc.z};
    const float vxp[4] = {xp.x, xp.y, xp.z, xp.w}, vxm[4] = {xm.x, xm.y, xm.z, xm.w};
    const float vyp[4] = {yp.x, yp.y, yp.z, yp.w}, vym[4] = {ym.x, ym.y, ym.z, ym.w};
    const float vb[4] = {b.x, b.y, b.z, b.w};
    const signed char vt[4] = {t.x, t.y, t.z, t.w};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      if (vt[k] != kFluid) continue;
      double s = (double)vxp[k];
      s += (double)vxm[k];
      s += (double)vyp[k];
      s += (double)vym[k];
      s += (double)zp[k];
      s += (double)zm[k];
      const double r = (double)vb[k] + s - 6.0 * (double)self[k];
      acc += r * r;
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  return acc;
}

__global__ void __launch_bounds__(256) k_resid_list_fin(Dims d, const float* __restrict__ p,
                                                       const float* __restrict__ rhs,
                                                       const int8_t* __restrict__ type,
                                                       const int* __restrict__ items, const int* __restrict__ n_items,
                                                       double* __restrict__ part, unsigned int* __restrict__ ticket,
                                                       SolveState* __restrict__ ss, int sweeps, double tol,
                                                       int max_iters, int set_cond,
                                                       cudaGraphConditionalHandle handle) {
  const int n = *n_items;
  const int gz = (d.sz / 4 + 31) / 32;
  double wsum = 0.0;
  for (int it = blockIdx.x * 8 + threadIdx.y; it < n; it += gridDim.x * 8) {
    const int id = __ldg(items + it);
    const int zb = id % gz, t = id / gz;
    wsum += resid_row(d, p, rhs, type, t / d.sy, t % d.sy, zb);
  }
  __shared__ double s_red[8];
  __shared__ bool s_last;
  const int tid = threadIdx.y * 32 + threadIdx.x;
  if (threadIdx.x == 0) s_red[threadIdx.y] = wsum;
  __syncthreads();
  if (tid == 0) {
    double t = 0.0;
    for (int k = 0; k < 8; ++k) t += s_red[k];
    part[blockIdx.x] = t;
    __threadfence();  // the partial before the ticket
    s_last = atomicAdd(ticket, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  __shared__ double sb[1024];
  const int nparts = (int)gridDim.x;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int v = tid + 256 * q;
    double a = 0.0;
    for (int i = v; i < nparts; i += 1024) a += __ldcg(part + i);
    sb[v] = a;
  }
  __syncthreads();
  for (int o = 512; o > 0; o >>= 1) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int v = tid + 256 * q;
      if (v < o) sb[v] += sb[v + o];
    }
    __syncthreads();
  }
  if (tid == 0) {
    *ticket = 0u;
    const bool more = finalize_state(sb[0], ss, sweeps, tol, max_iters);
    if (set_cond) cudaGraphSetConditional(handle, more ? 1u : 0u);
  }
}

// k_resid_flat and k_resid_finalize in one launch: the last block to write
// its partial (a ticket counter) sums the partials exactly as
// k_resid_finalize does (1024 strided sums, then the same pairwise tree,
// here four sums per thread), so the solve state and the loop decision are
// the same, with one launch fewer per residual check.
__global__ void __launch_bounds__(256) k_resid_flat_fin(Dims d, const float* __restrict__ p,
                                                       const float* __restrict__ rhs,
                                                       const int8_t* __restrict__ type,
                                                       const uint8_t* __restrict__ bact, double* __restrict__ part,
                                                       unsigned int* __restrict__ ticket, SolveState* __restrict__ ss,
                                                       int sweeps, double tol, int max_iters, int set_cond,
                                                       cudaGraphConditionalHandle handle) {
  resid_flat_body(d, p, rhs, type, bact, part, blockIdx.x, blockIdx.y, blockIdx.z);
  __shared__ bool s_last;
  const int tid = threadIdx.y * 32 + threadIdx.x;
  const unsigned nblocks = gridDim.x * gridDim.y * gridDim.z;
  if (tid == 0) {
    __threadfence();  // this block's partial before its ticket
    s_last = atomicAdd(ticket, 1u) == nblocks - 1;
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  __shared__ double sb[1024];
  const int nparts = (int)nblocks;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int v = tid + 256 * q;
    double a = 0.0;
    for (int i = v; i < nparts; i += 1024) a += __ldcg(part + i);
    sb[v] = a;
  }
  __syncthreads();
  for (int o = 512; o > 0; o >>= 1) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int v = tid + 256 * q;
      if (v < o) sb[v] += sb[v + o];
    }
    __syncthreads();
  }
  if (tid == 0) {
    *ticket = 0u;
    const bool more = finalize_state(sb[0], ss, sweeps, tol, max_iters);
    if (set_cond) cudaGraphSetConditional(handle, more ? 1u : 0u);
  }
}

// ------------------------------------------------------------------- batched
// One flat sweep over every scene whose solve is still running (live[s]);
// a finished scene's pressure is left as it is.
__device__ __forceinline__ void flat_block_coords(const Dims& d, int local, int& bx, int& by, int& bz) {
  const int gz = (d.sz / 4 + 31) / 32, gy = (d.sy + 7) / 8;
  bx = local % gz;
  const int t = local / gz;
  by = t % gy;
  bz = t / gy;
}

// Packed-row sweep for batches of small grids.  A warp work item is XS x
// planes x R rows x up to 128 z cells of one scene: with zw = min(sz/4, 32)
// z-quads per row, lane l covers row l / zw, quad l % zw, and R = 32 / zw rows
// share the warp, so a 24-wide grid still fills 30 of 32 lanes.  Items are
// numbered per scene as ((xg * ygroups) + yg) * zblocks + zb; a CTA's 8 warps
// take consecutive items.  Same arithmetic as the flat kernel (jacobi_quad),
// so results are bitwise those of the single-scene sweep.
struct RowItem {
  int zw, R, ygroups, zblocks;
};

__host__ __device__ __forceinline__ RowItem row_item_shape(const Dims& d) {
  RowItem r;
  const int zq = d.sz / 4;
  r.zw = zq < 32 ? zq : 32;
  r.R = 32 / r.zw;
  r.ygroups = (d.sy + r.R - 1) / r.R;
  r.zblocks = (zq + 31) / 32;
  return r;
}

__host__ __device__ __forceinline__ int row_items(const Dims& d, int xs) {
  const RowItem r = row_item_shape(d);
  return ((d.sx + xs - 1) / xs) * r.ygroups * r.zblocks;
}

// Does any 8^3 brick under x in [x0,x1), y in [y0,y1), z in [z0,z1) hold fluid?
__device__ __forceinline__ bool range_active(const Dims& d, const uint8_t* __restrict__ bact, int x0, int x1, int y0,
                                             int y1, int z0, int z1) {
  const int bx0 = x0 / kBrick, nbx = (x1 - 1) / kBrick - bx0 + 1;
  const int by0 = y0 / kBrick, nby = (y1 - 1) / kBrick - by0 + 1;
  const int bz0 = z0 / kBrick, nbz = (z1 - 1) / kBrick - bz0 + 1;
  const int nb = nbx * nby * nbz;
  int a = 0;
  for (int k = threadIdx.x & 31; k < nb; k += 32) {
    const int iz = k % nbz, t = k / nbz, iy = t % nby, ix = t / nby;
    a |= bact[((bx0 + ix) * d.by + by0 + iy) * d.bz + bz0 + iz];
  }
  return __any_sync(0xffffffffu, a) != 0;
}

// LIST: walk a list of (scene, local item) pairs whose bricks hold fluid
// (kb_row_list), built once per step, instead of every item.
template <int XS, bool PIPE, bool LIST>
__global__ void __launch_bounds__(256) kb_jacobi_rows(BatchIndex bi, int total, const int* __restrict__ live,
                                                     const float* __restrict__ pin_all, float* __restrict__ pout_all,
                                                     const float* __restrict__ rhs_all,
                                                     const int8_t* __restrict__ type_all,
                                                     const uint8_t* __restrict__ bact_all,
                                                     const int2* __restrict__ list, const int* __restrict__ n_list) {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;");
  const int lane = threadIdx.x & 31;
  const int warps = gridDim.x * (blockDim.x >> 5);
  const int n = LIST ? *n_list : total;
  for (int item = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); item < n; item += warps) {
    int s, local;
    if (LIST) {
      const int2 e = __ldg(list + item);
      s = e.x;
      local = e.y;
    } else {
      s = find_scene(bi.rows, bi.n_scenes, item);
      local = item - bi.rows[s];
    }
    if (!live[s]) continue;
    const SceneDesc& S = bi.scenes[s];
    const Dims& d = S.d;
    const RowItem ri = row_item_shape(d);
    const int zb = local % ri.zblocks;
    local /= ri.zblocks;
    const int yg = local % ri.ygroups;
    const int xg = local / ri.ygroups;
    const int x0 = xg * XS, x1 = min(x0 + XS, d.sx);
    const int ylo = yg * ri.R, yhi = min(ylo + ri.R, d.sy);
    const int zlo0 = zb * 128, zhi0 = min(zlo0 + 128, d.sz);
    if (!LIST && !range_active(d, bact_all + S.br_off, x0, x1, ylo, yhi, zlo0, zhi0)) continue;
    const int r = lane / ri.zw, q = lane % ri.zw;
    const int y = ylo + r;
    const int z = (zb * 32 + q) * 4;
    const bool in = r < ri.R && y < d.sy && z < d.sz;
    const float* __restrict__ pin = pin_all + S.c_off;
    float* __restrict__ pout = pout_all + S.c_off;
    const float* __restrict__ rhs = rhs_all + S.c_off;
    const int8_t* __restrict__ type = type_all + S.c_off;
    const int plane = d.sy * d.sz;
    const int col = y * d.sz + z;
    const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f);
    // p at x-1, x, x+1 and the rest of plane x.  PIPE: the loads of plane
    // x+1 are issued before plane x's arithmetic (software pipelining along x,
    // more registers); otherwise only p at x+2 is prefetched.
    float4 pm = zero, pc = zero, pp = zero, ym = zero, yp = zero, b = zero;
    char4 t = make_char4(0, 0, 0, 0);
    if (in) {
      const int c = x0 * plane + col;
      pc = ld4(pin + c);
      pm = x0 > 0 ? ld4(pin + c - plane) : pc;
      pp = x0 + 1 < d.sx ? ld4(pin + c + plane) : pc;
      if (PIPE) {
        ym = y > 0 ? ld4(pin + c - d.sz) : pc;
        yp = y + 1 < d.sy ? ld4(pin + c + d.sz) : pc;
        b = ld4(rhs + c);
        t = *reinterpret_cast<const char4*>(type + c);
      }
    }
    for (int x = x0; x < x1; ++x) {
      const int c = x * plane + col;
      float4 pn = pp, nym = pp, nyp = pp, nb = zero;
      char4 nt = make_char4(0, 0, 0, 0);
      if (PIPE) {
        if (in && x + 1 < x1) {
          const int cn = c + plane;
          if (x + 2 < d.sx) pn = ld4(pin + cn + plane);
          if (y > 0) nym = ld4(pin + cn - d.sz);
          if (y + 1 < d.sy) nyp = ld4(pin + cn + d.sz);
          nb = ld4(rhs + cn);
          nt = *reinterpret_cast<const char4*>(type + cn);
        }
      } else {
        if (in && x + 2 < d.sx && x + 1 < x1) pn = ld4(pin + c + 2 * plane);
        ym = pc;
        yp = pc;
        if (in) {
          if (y > 0) ym = ld4(pin + c - d.sz);
          if (y + 1 < d.sy) yp = ld4(pin + c + d.sz);
          b = ld4(rhs + c);
          t = *reinterpret_cast<const char4*>(type + c);
        }
      }
      float zlo = __shfl_up_sync(0xffffffffu, pc.w, 1);
      float zhi = __shfl_down_sync(0xffffffffu, pc.x, 1);
      if (in) {
        if (q == 0) zlo = z > 0 ? pin[c - 1] : pc.x;
        if (q == ri.zw - 1 || z + 4 >= d.sz) zhi = z + 4 < d.sz ? pin[c + 4] : pc.w;
        *reinterpret_cast<float4*>(pout + c) = jacobi_quad(pm, pp, ym, yp, pc, zlo, zhi, b, t);
      }
      pm = pc;
      pc = pp;
      pp = (x + 2 < d.sx) ? pn : pc;
      if (PIPE) {
        ym = nym;
        yp = nyp;
        b = nb;
        t = nt;
      }
    }
  }
}

// The (scene, local item) pairs of the packed-row sweep whose bricks hold
// fluid.  Warp-aggregated appends: the list order varies from run to run,
// the sweep's results do not (items are independent).
template <int XS>
__global__ void __launch_bounds__(256) kb_row_list(BatchIndex bi, int total, const uint8_t* __restrict__ bact_all,
                                                  int2* __restrict__ list, int* __restrict__ n_list) {
  const int lane = threadIdx.x & 31;
  for (int base = blockIdx.x * blockDim.x; base < total; base += gridDim.x * blockDim.x) {
    const int item = base + threadIdx.x;
    int act = 0, s = 0, local = 0;
    if (item < total) {
      s = find_scene(bi.rows, bi.n_scenes, item);
      local = item - bi.rows[s];
      const SceneDesc& S = bi.scenes[s];
      const Dims& d = S.d;
      const RowItem ri = row_item_shape(d);
      int t = local;
      const int zb = t % ri.zblocks;
      t /= ri.zblocks;
      const int yg = t % ri.ygroups, xg = t / ri.ygroups;
      const int x0 = xg * XS, x1 = min(x0 + XS, d.sx);
      const int y0 = yg * ri.R, y1 = min(y0 + ri.R, d.sy);
      const int z0 = zb * 128, z1 = min(z0 + 128, d.sz);
      const uint8_t* bact = bact_all + S.br_off;
      for (int bx = x0 / kBrick; bx <= (x1 - 1) / kBrick && !act; ++bx)
        for (int by = y0 / kBrick; by <= (y1 - 1) / kBrick && !act; ++by)
          for (int bz = z0 / kBrick; bz <= (z1 - 1) / kBrick && !act; ++bz)
            act = bact[(bx * d.by + by) * d.bz + bz] ? 1 : 0;
    }
    const unsigned m = __ballot_sync(0xffffffffu, act);
    int pos = 0;
    if (lane == 0 && m) pos = atomicAdd(n_list, __popc(m));
    pos = __shfl_sync(0xffffffffu, pos, 0) + __popc(m & ((1u << lane) - 1u));
    if (act) list[pos] = make_int2(s, local);
  }
}

__global__ void __launch_bounds__(256) kb_resid_flat(BatchIndex bi, int total, const int* __restrict__ live,
                                                    const float* __restrict__ p, const float* __restrict__ rhs,
                                                    const int8_t* __restrict__ type, const uint8_t* __restrict__ bact,
                                                    double* __restrict__ part) {
  for (int vb = blockIdx.x; vb < total; vb += gridDim.x) {
    const int s = find_scene(bi.flat, bi.n_scenes, vb);
    if (!live[s]) continue;
    const SceneDesc& S = bi.scenes[s];
    int bx, by, bz;
    flat_block_coords(S.d, vb - bi.flat[s], bx, by, bz);
    const int c = S.c_off;
    resid_flat_body(S.d, p + c, rhs + c, type + c, bact + S.br_off, part + S.rp_off, bx, by, bz);
    __syncthreads();  // s_red is reused by the next virtual block
  }
}

// One CTA per scene; a finished scene keeps its record.
__global__ void __launch_bounds__(1024) kb_resid_finalize(BatchIndex bi, const double* __restrict__ part,
                                                         SolveState* __restrict__ ss, int* __restrict__ live,
                                                         int sweeps, double tol, int max_iters) {
  const int s = blockIdx.x;
  if (!live[s]) return;
  const SceneDesc& S = bi.scenes[s];
  const bool more = resid_finalize_body(part + S.rp_off, resid_flat_parts_dev(S.d), ss + s, sweeps, tol, max_iters);
  if (threadIdx.x == 0) live[s] = more ? 1 : 0;
}

__global__ void __launch_bounds__(1024) kb_solve_condition(const int* __restrict__ live, int n_scenes,
                                                          cudaGraphConditionalHandle handle) {
  int any = 0;
  for (int s = threadIdx.x; s < n_scenes; s += blockDim.x) any |= live[s];
  any = __syncthreads_or(any);
  if (threadIdx.x == 0) cudaGraphSetConditional(handle, any ? 1u : 0u);
}

template <int L, bool RESID, int BY>
cudaError_t launch_one(cudaStream_t st, const Dims& d, int xc, const float* pin, float* pout, const float* rhs,
                       const int8_t* type, const uint8_t* bact, double* part, int* nparts) {
  constexpr int H = L + (RESID ? 1 : 0);
  constexpr int TZ = 32 - 2 * H, TY = BY - 2 * H;
  const dim3 grid((d.sz + TZ - 1) / TZ, (d.sy + TY - 1) / TY, (d.sx + xc - 1) / xc);
  const size_t sm = sizeof(float) * 2 * H * BY * 32;
  if (nparts) *nparts = (int)(grid.x * grid.y * grid.z);
  cudaLaunchConfig_t lc = {};
  lc.gridDim = grid;
  lc.blockDim = dim3(32, BY);
  lc.dynamicSmemBytes = sm;
  lc.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  lc.attrs = at;
  lc.numAttrs = 1;
  return cudaLaunchKernelEx(&lc, k_jacobi<L, RESID, BY>, d, xc, pin, pout, rhs, type, bact, part);
}

template <int L, bool RESID, int BY>
cudaError_t set_smem_attr() {
  constexpr int H = L + (RESID ? 1 : 0);
  if constexpr (BY - 2 * H > 0 && 32 - 2 * H > 0) {
    return cudaFuncSetAttribute(k_jacobi<L, RESID, BY>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)(sizeof(float) * 2 * H * BY * 32));
  }
  return cudaSuccess;
}

template <int BY>
cudaError_t prepare_by() {
  cudaError_t e = cudaSuccess;
  if ((e = set_smem_attr<1, false, BY>()) != cudaSuccess) return e;
  if ((e = set_smem_attr<1, true, BY>()) != cudaSuccess) return e;
  if ((e = set_smem_attr<2, false, BY>()) != cudaSuccess) return e;
  if ((e = set_smem_attr<2, true, BY>()) != cudaSuccess) return e;
  if ((e = set_smem_attr<4, false, BY>()) != cudaSuccess) return e;
  if ((e = set_smem_attr<4, true, BY>()) != cudaSuccess) return e;
  if ((e = set_smem_attr<8, false, BY>()) != cudaSuccess) return e;
  return set_smem_attr<8, true, BY>();
}

template <int L, bool RESID>
cudaError_t dispatch_by(cudaStream_t st, const Dims& d, int by, int xc, const float* pin, float* pout,
                        const float* rhs, const int8_t* type, const uint8_t* bact, double* part, int* np) {
  constexpr int H = L + (RESID ? 1 : 0);
  if (by == 8) {
    if constexpr (8 - 2 * H > 0) return launch_one<L, RESID, 8>(st, d, xc, pin, pout, rhs, type, bact, part, np);
  } else if (by == 16) {
    if constexpr (16 - 2 * H > 0) return launch_one<L, RESID, 16>(st, d, xc, pin, pout, rhs, type, bact, part, np);
  } else if (by == 32) {
    if constexpr (32 - 2 * H > 0) return launch_one<L, RESID, 32>(st, d, xc, pin, pout, rhs, type, bact, part, np);
  }
  return cudaErrorInvalidValue;
}

template <bool RESID>
cudaError_t dispatch_levels(cudaStream_t st, const Dims& d, const JacobiPlan& p, const float* pin, float* pout,
                            const float* rhs, const int8_t* type, const uint8_t* bact, double* part, int* np) {
  switch (p.levels) {
    case 1: return dispatch_by<1, RESID>(st, d, p.by, p.xc, pin, pout, rhs, type, bact, part, np);
    case 2: return dispatch_by<2, RESID>(st, d, p.by, p.xc, pin, pout, rhs, type, bact, part, np);
    case 4: return dispatch_by<4, RESID>(st, d, p.by, p.xc, pin, pout, rhs, type, bact, part, np);
    case 8: return dispatch_by<8, RESID>(st, d, p.by, p.xc, pin, pout, rhs, type, bact, part, np);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace

cudaError_t jacobi_prepare() {
  cudaError_t e = prepare_by<8>();
  if (e == cudaSuccess) e = prepare_by<16>();
  if (e == cudaSuccess) e = prepare_by<32>();
  return e;
}

long long jacobi_cells_updated(const Dims& d, const JacobiPlan& p, const uint8_t* bact_host) {
  if (p.by == 2) {  // cube: core cells of the tiles whose core holds fluid
    const int tx = p.xc, tz = 32 - 2 * p.levels;
    long long cells = 0;
    for (int x0 = 0; x0 < d.sx; x0 += tx)
      for (int y0 = 0; y0 < d.sy; y0 += tx)
        for (int z0 = 0; z0 < d.sz; z0 += tz) {
          const int x1 = std::min(x0 + tx, d.sx), y1 = std::min(y0 + tx, d.sy), z1 = std::min(z0 + tz, d.sz);
          bool act = false;
          for (int bx = x0 / kBrick; bx <= (x1 - 1) / kBrick && !act; ++bx)
            for (int by = y0 / kBrick; by <= (y1 - 1) / kBrick && !act; ++by)
              for (int bz = z0 / kBrick; bz <= (z1 - 1) / kBrick && !act; ++bz)
                act = bact_host[(bx * d.by + by) * d.bz + bz] != 0;
          if (act) cells += (long long)(x1 - x0) * (y1 - y0) * (z1 - z0);
        }
    return cells;
  }
  if (p.by == 0) {
    long long cells = 0;  // flat: xc x planes x 8 rows (one warp per row) x 128 z per block
    for (int x0 = 0; x0 < d.sx; x0 += p.xc)
      for (int y = 0; y < d.sy; ++y)
        for (int z0 = 0; z0 < d.sz; z0 += 128) {
          const int x1 = std::min(x0 + p.xc, d.sx);
          bool act = false;
          for (int bx = x0 / kBrick; bx <= (x1 - 1) / kBrick && !act; ++bx)
            for (int bz = z0 / kBrick; bz < (z0 + 128) / kBrick && bz < d.bz && !act; ++bz)
              act = bact_host[(bx * d.by + y / kBrick) * d.bz + bz] != 0;
          if (act) cells += (long long)(x1 - x0) * std::min(128, d.sz - z0);
        }
    return cells;
  }
  const int H = p.levels;
  const int TZ = 32 - 2 * H, TY = p.by - 2 * H;
  if (TZ <= 0 || TY <= 0 || p.xc <= 0) return -1;
  long long cells = 0;
  for (int x0 = 0; x0 < d.sx; x0 += p.xc)
    for (int y0 = 0; y0 < d.sy; y0 += TY)
      for (int z0 = 0; z0 < d.sz; z0 += TZ) {
        const int x1 = x0 + p.xc < d.sx ? x0 + p.xc : d.sx;
        const int y1 = y0 + TY < d.sy ? y0 + TY : d.sy;
        const int z1 = z0 + TZ < d.sz ? z0 + TZ : d.sz;
        bool act = false;
        for (int bx = x0 / kBrick; bx <= (x1 - 1) / kBrick && !act; ++bx)
          for (int by = y0 / kBrick; by <= (y1 - 1) / kBrick && !act; ++by)
            for (int bz = z0 / kBrick; bz <= (z1 - 1) / kBrick && !act; ++bz)
              act = bact_host[(bx * d.by + by) * d.bz + bz] != 0;
        if (act) cells += (long long)(x1 - x0) * (y1 - y0) * (z1 - z0);
      }
  return cells;
}

int jacobi_parts(const Dims& d, const JacobiPlan& p, bool resid) {
  if (p.by == 0 || p.by == 2) return resid ? -1 : 1;
  const int H = p.levels + (resid ? 1 : 0);
  const int TZ = 32 - 2 * H, TY = p.by - 2 * H;
  if (TZ <= 0 || TY <= 0 || p.xc <= 0) return -1;
  return ((d.sz + TZ - 1) / TZ) * ((d.sy + TY - 1) / TY) * ((d.sx + p.xc - 1) / p.xc);
}

cudaError_t launch_jacobi(cudaStream_t st, const Dims& d, const JacobiPlan& plan, bool resid, const float* pin,
                          float* pout, const float* rhs, const int8_t* type, const uint8_t* brick_active,
                          double* part, int* nparts_out) {
  if (plan.by == 0) {
    // flat plan: one sweep per launch, XS = plan.xc x planes per block
    if (resid || d.sz % 4 != 0) return cudaErrorInvalidValue;
    cudaLaunchConfig_t lc = {};
    lc.blockDim = dim3(32, 8);
    lc.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    lc.attrs = at;
    lc.numAttrs = 1;
    if (nparts_out) *nparts_out = 0;
    const dim3 g((d.sz / 4 + 31) / 32, (d.sy + 7) / 8, 1);
    switch (plan.xc) {
      case 1: lc.gridDim = dim3(g.x, g.y, d.sx); return cudaLaunchKernelEx(&lc, k_jacobi_flat<1>, d, pin, pout, rhs, type, brick_active);
      case 2: lc.gridDim = dim3(g.x, g.y, (d.sx + 1) / 2); return cudaLaunchKernelEx(&lc, k_jacobi_flat<2>, d, pin, pout, rhs, type, brick_active);
      case 4: lc.gridDim = dim3(g.x, g.y, (d.sx + 3) / 4); return cudaLaunchKernelEx(&lc, k_jacobi_flat<4>, d, pin, pout, rhs, type, brick_active);
      case 8: lc.gridDim = dim3(g.x, g.y, (d.sx + 7) / 8); return cudaLaunchKernelEx(&lc, k_jacobi_flat<8>, d, pin, pout, rhs, type, brick_active);
      default: return cudaErrorInvalidValue;
    }
  }
  if (plan.by == 2) {
    // cube plan: plan.levels sweeps per launch on TX = plan.xc tiles
    if (resid || d.sz % 4 != 0) return cudaErrorInvalidValue;
    if (nparts_out) *nparts_out = 0;
    return dispatch_cube(st, d, plan.levels, plan.xc, pin, pout, rhs, type, brick_active);
  }
  if (resid) return dispatch_levels<true>(st, d, plan, pin, pout, rhs, type, brick_active, part, nparts_out);
  return dispatch_levels<false>(st, d, plan, pin, pout, rhs, type, brick_active, part, nparts_out);
}

bool cube_plan_ok(int levels, int tx) {
  return (tx == 8 && levels >= 1 && levels <= 4) || (tx == 16 && (levels == 1 || levels == 2 || levels == 4));
}

int persist_items(const Dims& d) { return ((d.sz / 4 + 31) / 32) * ((d.sy + 7) / 8) * d.sx; }

int persist_ctas(int device) {
  int sms = 0, occ = 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_persist_solve, 1024, 0) != cudaSuccess) return 0;
  return sms * (occ < 1 ? 0 : 1);
}

cudaError_t launch_items_compact(cudaStream_t st, const Dims& d, const uint8_t* brick_active, int* items,
                                 int* n_items, unsigned int* bar) {
  k_items_compact<<<1, 1024, 0, st>>>(d, brick_active, items, n_items, bar);
  return cudaGetLastError();
}

cudaError_t launch_persist_solve(cudaStream_t st, const Dims& d, int ctas, float* pa, float* pb, const float* rhs,
                                 const int8_t* type, const int* items, const int* n_items, unsigned int* bar,
                                 double* part, SolveState* ss, int fixed_sweeps, int check, int max_iters, double tol,
                                 BarrierTest bt) {
  if (d.sz % 4 != 0 || ctas <= 0) return cudaErrorInvalidValue;
  cudaLaunchConfig_t lc = {};
  lc.gridDim = dim3(ctas);
  lc.blockDim = dim3(1024);
  lc.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeCooperative;  // all CTAs co-resident, or the launch fails
  at[0].val.cooperative = 1;
  lc.attrs = at;
  lc.numAttrs = 1;
  return cudaLaunchKernelEx(&lc, k_persist_solve, d, pa, pb, rhs, type, items, n_items, bar, part, ss, fixed_sweeps,
                            check, max_iters, tol, bt);
}

int resid_flat_parts(const Dims& d) { return ((d.sz / 4 + 31) / 32) * ((d.sy + 7) / 8) * d.sx; }

cudaError_t launch_resid_flat(cudaStream_t st, const Dims& d, const float* p, const float* rhs, const int8_t* type,
                              const uint8_t* brick_active, double* part) {
  if (d.sz % 4 != 0) return cudaErrorInvalidValue;
  k_resid_flat<<<dim3((d.sz / 4 + 31) / 32, (d.sy + 7) / 8, d.sx), dim3(32, 8), 0, st>>>(d, p, rhs, type,
                                                                                        brick_active, part);
  return cudaGetLastError();
}

cudaError_t launch_resid_flat_fin(cudaStream_t st, const Dims& d, const float* p, const float* rhs,
                                  const int8_t* type, const uint8_t* brick_active, double* part, unsigned int* ticket,
                                  SolveState* ss, int sweeps, double tol, int max_iters, bool set_cond,
                                  unsigned long long cond_handle) {
  if (d.sz % 4 != 0) return cudaErrorInvalidValue;
  k_resid_flat_fin<<<dim3((d.sz / 4 + 31) / 32, (d.sy + 7) / 8, d.sx), dim3(32, 8), 0, st>>>(
      d, p, rhs, type, brick_active, part, ticket, ss, sweeps, tol, max_iters, set_cond ? 1 : 0,
      (cudaGraphConditionalHandle)cond_handle);
  return cudaGetLastError();
}

cudaError_t launch_resid_list_fin(cudaStream_t st, const Dims& d, const float* p, const float* rhs,
                                  const int8_t* type, const int* items, const int* n_items, double* part,
                                  unsigned int* ticket, SolveState* ss, int sweeps, double tol, int max_iters,
                                  bool set_cond, unsigned long long cond_handle) {
  if (d.sz % 4 != 0) return cudaErrorInvalidValue;
  const int need = (row_items_capacity(d) + 7) / 8;
  const int grid = std::max(1, std::min(need, resident_ctas(k_resid_list_fin, 256)));
  k_resid_list_fin<<<grid, dim3(32, 8), 0, st>>>(d, p, rhs, type, items, n_items, part, ticket, ss, sweeps, tol,
                                                 max_iters, set_cond ? 1 : 0, (cudaGraphConditionalHandle)cond_handle);
  return cudaGetLastError();
}

cudaError_t launch_resid_finalize(cudaStream_t st, const double* part, int nparts, SolveState* ss,
                                  int sweeps_done_per_call, double tol, int max_iters, bool set_cond,
                                  unsigned long long cond_handle) {
  k_resid_finalize<<<1, 1024, 0, st>>>(part, nparts, ss, sweeps_done_per_call, tol, max_iters, set_cond ? 1 : 0,
                                       (cudaGraphConditionalHandle)cond_handle);
  return cudaGetLastError();
}

}  // namespace aqb

namespace aqb {

int batch_row_items(const Dims& d, int xs) { return row_items(d, xs); }

long long batch_row_cells_updated(const Dims& d, int xs, const uint8_t* bact_host) {
  const RowItem ri = row_item_shape(d);
  long long cells = 0;
  for (int x0 = 0; x0 < d.sx; x0 += xs)
    for (int y0 = 0; y0 < d.sy; y0 += ri.R)
      for (int z0 = 0; z0 < d.sz; z0 += 128) {
        const int x1 = std::min(x0 + xs, d.sx), y1 = std::min(y0 + ri.R, d.sy), z1 = std::min(z0 + 128, d.sz);
        bool act = false;
        for (int bx = x0 / kBrick; bx <= (x1 - 1) / kBrick && !act; ++bx)
          for (int by = y0 / kBrick; by <= (y1 - 1) / kBrick && !act; ++by)
            for (int bz = z0 / kBrick; bz <= (z1 - 1) / kBrick && !act; ++bz)
              act = bact_host[(bx * d.by + by) * d.bz + bz] != 0;
        if (act) cells += (long long)(x1 - x0) * (y1 - y0) * (z1 - z0);
      }
  return cells;
}

cudaError_t launch_batch_jacobi_rows(cudaStream_t st, const BatchIndex& bi, int total, int xs, bool pipelined,
                                     int grid, const int* live, const float* pin, float* pout, const float* rhs,
                                     const int8_t* type, const uint8_t* brick_active, const int2* list,
                                     const int* n_list) {
  cudaLaunchConfig_t lc = {};
  lc.blockDim = dim3(256);
  lc.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  lc.attrs = at;
  lc.numAttrs = 1;
  auto go = [&](auto kern) {
    const int items_per_cta = 8;
    const int need = (total + items_per_cta - 1) / items_per_cta;
    lc.gridDim = dim3(std::max(1, std::min({grid, need, resident_ctas(kern, 256)})));
    return cudaLaunchKernelEx(&lc, kern, bi, total, live, pin, pout, rhs, type, brick_active, list, n_list);
  };
  const bool L = list != nullptr;
#define AQ_ROWS(X, P) return L ? go(kb_jacobi_rows<X, P, true>) : go(kb_jacobi_rows<X, P, false>)
  if (pipelined) {
    switch (xs) {
      case 2: AQ_ROWS(2, true);
      case 4: AQ_ROWS(4, true);
      case 8: AQ_ROWS(8, true);
      default: return cudaErrorInvalidValue;
    }
  }
  switch (xs) {
    case 1: AQ_ROWS(1, false);
    case 2: AQ_ROWS(2, false);
    case 4: AQ_ROWS(4, false);
    case 8: AQ_ROWS(8, false);
    default: return cudaErrorInvalidValue;
  }
#undef AQ_ROWS
}

cudaError_t launch_batch_row_list(cudaStream_t st, const BatchIndex& bi, int total, int xs,
                                  const uint8_t* brick_active, int2* list, int* n_list) {
  cudaError_t e = cudaMemsetAsync(n_list, 0, sizeof(int), st);
  if (e != cudaSuccess) return e;
  const int g = std::max(1, std::min((total + 255) / 256, 148 * 8));
  switch (xs) {
    case 1: kb_row_list<1><<<g, 256, 0, st>>>(bi, total, brick_active, list, n_list); break;
    case 2: kb_row_list<2><<<g, 256, 0, st>>>(bi, total, brick_active, list, n_list); break;
    case 4: kb_row_list<4><<<g, 256, 0, st>>>(bi, total, brick_active, list, n_list); break;
    case 8: kb_row_list<8><<<g, 256, 0, st>>>(bi, total, brick_active, list, n_list); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t launch_batch_resid_flat(cudaStream_t st, const BatchIndex& bi, int total, int grid, const int* live,
                                    const float* p, const float* rhs, const int8_t* type,
                                    const uint8_t* brick_active, double* part) {
  const int g = std::max(1, std::min({grid, total, resident_ctas(kb_resid_flat, 256)}));
  kb_resid_flat<<<g, dim3(32, 8), 0, st>>>(bi, total, live, p, rhs, type, brick_active, part);
  return cudaGetLastError();
}

cudaError_t launch_batch_resid_finalize(cudaStream_t st, const BatchIndex& bi, const double* part, SolveState* ss,
                                        int* live, int sweeps, double tol, int max_iters) {
  kb_resid_finalize<<<bi.n_scenes, 1024, 0, st>>>(bi, part, ss, live, sweeps, tol, max_iters);
  return cudaGetLastError();
}

cudaError_t launch_batch_solve_condition(cudaStream_t st, const int* live, int n_scenes,
                                         unsigned long long cond_handle) {
  kb_solve_condition<<<1, 1024, 0, st>>>(live, n_scenes, (cudaGraphConditionalHandle)cond_handle);
  return cudaGetLastError();
}

}  // namespace aqb

namespace aqb {

int row_items_capacity(const Dims& d) { return d.sx * d.sy * ((d.sz / 4 + 31) / 32); }

cudaError_t launch_row_items(cudaStream_t st, const Dims& d, const uint8_t* brick_active, int* items, int* n_items) {
  k_row_items<<<1, 1024, 0, st>>>(d, brick_active, items, n_items);
  return cudaGetLastError();
}

cudaError_t launch_jacobi_list(cudaStream_t st, const Dims& d, const float* pin, float* pout, const float* rhs,
                               const int8_t* type, const int* items, const int* n_items, bool early) {
  if (d.sz % 4 != 0) return cudaErrorInvalidValue;
  // 8 warps per CTA, one resident wave (4 to 32 warps per CTA and fewer,
  // fatter waves measured the same or slower at 128^3); the kernel is held
  // to 40 registers so 6 CTAs fit per SM (888 CTAs, 7104 warps): every warp
  // of a 128^3 pool's ~6300 rows then has at most one row, and none waits
  // on a second row's loads after the first (3.02 against 3.29 us a sweep)
  const int wy = 8;
  const int need = (row_items_capacity(d) + wy - 1) / wy;
  cudaLaunchConfig_t lc = {};
  lc.gridDim = dim3(std::max(1, std::min(need, resident_ctas(k_jacobi_list, 32 * wy))));
  lc.blockDim = dim3(32, wy);
  lc.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  lc.attrs = at;
  lc.numAttrs = 1;
  return cudaLaunchKernelEx(&lc, k_jacobi_list, d, pin, pout, rhs, type, items, n_items, early ? 1 : 0);
}

}  // namespace aqb
