// Grid kernels: particle-to-grid transfer with forces and wall clamps,
// divergence, pressure-gradient subtract, velocity extrapolation and phase
// diffusion (stages (b), (c) and (e) except the Jacobi sweeps).
//
// Reference: Fluid/Fluid_3D_FLIP.cu:8-186 (P2G, divide, fractions, counts),
// Fluid/Fluid_3D_kernels.cu:4-98 (gravity, fixBoundary), :118-207 (pressure
// update), :210-422 (extrapolation), :426-458 (divergence), :520-556 (diffusion).
#include "aq_kernels.cuh"

namespace aqb {
namespace {

__device__ __forceinline__ float hat1(float r) { return fmaxf(0.f, __fsub_rn(1.f, fabsf(r))); }

// One particle's contributions to node (fx, fy, fz) from the cell at offset
// (DX, DY, DZ) (transferToCellAccumPhase, Fluid/Fluid_3D_FLIP.cu:29-64): hat
// weights of the u, v, w faces in cell units, each sum rounded as written
// (explicit intrinsics, so every P2G kernel produces the same bits).
// dx, dy, dz are constants wherever this is inlined (unrolled loops).
__device__ __forceinline__ void p2g_particle(int DX, int DY, int DZ, float qx, float qy, float qz, float vx, float vy,
                                             float vz, float fx,
                                             float fy, float fz, float fxh, float fyh, float fzh, float& su,
                                             float& sv, float& sw, float& wu, float& wv, float& ww, float& bxyz) {
  const float bx = hat1(__fsub_rn(qx, fxh)), by = hat1(__fsub_rn(qy, fyh)), bz = hat1(__fsub_rn(qz, fzh));
  if (DX < 1) {  // a cell at dx = +1 cannot touch the u face (weight exactly 0)
    const float w = __fmul_rn(__fmul_rn(hat1(__fsub_rn(qx, fx)), by), bz);
    su = __fmaf_rn(w, vx, su);
    wu = __fadd_rn(wu, w);
  }
  if (DY < 1) {
    const float w = __fmul_rn(__fmul_rn(bx, hat1(__fsub_rn(qy, fy))), bz);
    sv = __fmaf_rn(w, vy, sv);
    wv = __fadd_rn(wv, w);
  }
  if (DZ < 1) {
    const float w = __fmul_rn(__fmul_rn(bx, by), hat1(__fsub_rn(qz, fz)));
    sw = __fmaf_rn(w, vz, sw);
    ww = __fadd_rn(ww, w);
  }
  bxyz = __fmul_rn(__fmul_rn(bx, by), bz);
}

// p2g_particle with the x factors already evaluated: ax = hat1(qx - fx) and
// bx = hat1(qx - fxh), the same values (a staged plane shares the node x).
__device__ __forceinline__ void p2g_particle_x(int DX, int DY, int DZ, float ax, float bx, float qy, float qz,
                                               float vx, float vy, float vz, float fy, float fz, float fyh,
                                               float fzh, float& su, float& sv, float& sw, float& wu, float& wv,
                                               float& ww, float& bxyz) {
  const float by = hat1(__fsub_rn(qy, fyh)), bz = hat1(__fsub_rn(qz, fzh));
  if (DX < 1) {
    const float w = __fmul_rn(__fmul_rn(ax, by), bz);
    su = __fmaf_rn(w, vx, su);
    wu = __fadd_rn(wu, w);
  }
  if (DY < 1) {
    const float w = __fmul_rn(__fmul_rn(bx, hat1(__fsub_rn(qy, fy))), bz);
    sv = __fmaf_rn(w, vy, sv);
    wv = __fadd_rn(wv, w);
  }
  if (DZ < 1) {
    const float w = __fmul_rn(__fmul_rn(bx, by), hat1(__fsub_rn(qz, fz)));
    sw = __fmaf_rn(w, vz, sw);
    ww = __fadd_rn(ww, w);
  }
  bxyz = __fmul_rn(__fmul_rn(bx, by), bz);
}

// The fractions' weighted sum of the node's own cell (transferVolumeFractionsToCell).
__device__ __forceinline__ void p2g_fractions(float w, const float4& f, float4& fs, float& fw) {
  fs.x = __fmaf_rn(w, f.x, fs.x);
  fs.y = __fmaf_rn(w, f.y, fs.y);
  fs.z = __fmaf_rn(w, f.z, fs.z);
  fs.w = __fmaf_rn(w, f.w, fs.w);
  fw = __fadd_rn(fw, w);
}

// P2G gather for node (x,y,z) in [0,s)^3.  The reference loops over the 27
// neighbour cells by a flat index with only a [0,C) range check, so rows at
// the y/z edges wrap to far cells; those particles are more than h away and
// add exactly +0 (sizes >= 4 are enforced), so only in-domain cells are
// visited, in the same (dx,dy,dz,j) order.  A cell at dx=+1 cannot touch the
// u-face at x (weight exactly 0 there), likewise dy=+1 for v and dz=+1 for w.
// Weights use positions in cell units, q = p/h; the reference evaluates
// (p - face*h)/h with approximate division (-use_fast_math).
// Accumulated P2G sums of one node.
struct P2gAcc {
  float su, sv, sw, wu, wv, ww;
  float4 fs;
  float fw;
  int own, left, down, back;  // particles in the node's cell and its -x, -y, -z neighbours
};

// transferToCellDividePhase + transferVolumeFractionsToCell + applyGravity +
// fixBoundary (low walls) for node (x, y, z) from its accumulated sums.
template <bool FORCES, bool MULTI>
__device__ __forceinline__ void p2g_finish(const Dims& d, const StepParams& sp, int x, int y, int z, const P2gAcc& a,
                                           float* __restrict__ u0, float* __restrict__ v0, float* __restrict__ w0,
                                           float* __restrict__ un, float* __restrict__ vn, float* __restrict__ wn,
                                           int8_t* __restrict__ type, float* __restrict__ density,
                                           float4* __restrict__ vf, float4* __restrict__ nvf) {
  const float su = a.su, sv = a.sv, sw = a.sw, wu = a.wu, wv = a.wv, ww = a.ww;
  const float4 fs = a.fs;
  const float fw = a.fw;
  const int own = a.own, left = a.left, down = a.down, back = a.back;
  // transferToCellDividePhase
  const float u = wu > 0.f ? __fdiv_rn(su, wu) : 0.f;
  const float v = wv > 0.f ? __fdiv_rn(sv, wv) : 0.f;
  const float w = ww > 0.f ? __fdiv_rn(sw, ww) : 0.f;
  const int ni = node_index(d, x, y, z);
  const int ci = cell_index(d, x, y, z);
  const bool fluid = own > 0;
  u0[ni] = u; v0[ni] = v; w0[ni] = w;
  type[ci] = fluid ? (int8_t)kFluid : (int8_t)kAir;
  // transferVolumeFractionsToCell
  if (MULTI) {
    float4 f = make_float4(0.f, 0.f, 0.f, 0.f);
    if (fw > 0.f) {
      f.x = __fdiv_rn(fs.x, fw); f.y = __fdiv_rn(fs.y, fw); f.z = __fdiv_rn(fs.z, fw); f.w = __fdiv_rn(fs.w, fw);
      const float s = f.x + f.y + f.z + f.w;
      f.x = __fdiv_rn(f.x, s); f.y = __fdiv_rn(f.y, s); f.z = __fdiv_rn(f.z, s); f.w = __fdiv_rn(f.w, s);
    }
    density[ci] = sp.rho[0] * f.x + sp.rho[1] * f.y + sp.rho[2] * f.z + sp.rho[3] * f.w;
    vf[ci] = f;
    nvf[ci] = f;
  } else {
    density[ci] = fluid ? sp.rho[sp.phase] : 0.f;
  }
  float nu = u, nv = v, nw = w;
  if (FORCES) {
    // applyGravityImpl: a fluid cell adds g*dt to its own three faces; an air
    // cell receives g*dt from each fluid neighbour below it along an axis
    // whose gravity component is nonzero.
    if (fluid) {
      nu += sp.gdx; nv += sp.gdy; nw += sp.gdz;
    } else {
      const int adds = (sp.gx_nz && left > 0) + (sp.gy_nz && down > 0) + (sp.gz_nz && back > 0);
      for (int a = 0; a < adds; ++a) { nu += sp.gdx; nv += sp.gdy; nw += sp.gdz; }
    }
    // fixBoundaryX/Y/Z, low walls (the s-th layer is k_slayer's)
    if (x == 0 && covered_x(d, y, z)) nu = fmaxf(0.f, nu);
    if (y == 0 && covered_y(d, x, z)) nv = fmaxf(0.f, nv);
    if (z == 0 && covered_z(d, x, y)) nw = fmaxf(0.f, nw);
  }
  un[ni] = nu; vn[ni] = nv; wn[ni] = nw;
}


template <bool FORCES, bool MULTI>
__device__ __forceinline__ void p2g_body(const Dims& d, const StepParams& sp, const Particles& cur,
                                         const int* __restrict__ off, float* __restrict__ u0, float* __restrict__ v0,
                                         float* __restrict__ w0, float* __restrict__ un, float* __restrict__ vn,
                                         float* __restrict__ wn, int8_t* __restrict__ type,
                                         float* __restrict__ density, float4* __restrict__ vf,
                                         float4* __restrict__ nvf, int bx, int by, int bz) {
  const int z = bx * 32 + threadIdx.x;
  const int y = by * 8 + threadIdx.y;
  const int x = bz;
  if (z >= d.sz || y >= d.sy) return;
  const float fx = (float)x, fy = (float)y, fz = (float)z;
  const float fxh = fx + 0.5f, fyh = fy + 0.5f, fzh = fz + 0.5f;
  const float inv_h = d.inv_h;
  float su = 0.f, sv = 0.f, sw = 0.f, wu = 0.f, wv = 0.f, ww = 0.f;
  float4 fs = make_float4(0.f, 0.f, 0.f, 0.f);
  float fw = 0.f;
  int own = 0, left = 0, down = 0, back = 0;
#pragma unroll
  for (int dx = -1; dx <= 1; ++dx) {
    const int X = x + dx;
    if (X < 0 || X >= d.sx) continue;
#pragma unroll
    for (int dy = -1; dy <= 1; ++dy) {
      const int Y = y + dy;
      if (Y < 0 || Y >= d.sy) continue;
#pragma unroll
      for (int dz = -1; dz <= 1; ++dz) {
        const int Z = z + dz;
        if (Z < 0 || Z >= d.sz) continue;
        const int c = (X * d.sy + Y) * d.sz + Z;
        const int b = __ldg(off + c), e = __ldg(off + c + 1);
        if (dx == 0 && dy == 0 && dz == 0) own = e - b;
        if (dx == -1 && dy == 0 && dz == 0) left = e - b;
        if (dx == 0 && dy == -1 && dz == 0) down = e - b;
        if (dx == 0 && dy == 0 && dz == -1) back = e - b;
        for (int j = b; j < e; ++j) {
          const float qx = __fmul_rn(__ldg(cur.px + j), inv_h);
          const float qy = __fmul_rn(__ldg(cur.py + j), inv_h);
          const float qz = __fmul_rn(__ldg(cur.pz + j), inv_h);
          const float vx = dx < 1 ? __ldg(cur.vx + j) : 0.f;
          const float vy = dy < 1 ? __ldg(cur.vy + j) : 0.f;
          const float vz = dz < 1 ? __ldg(cur.vz + j) : 0.f;
          float bxyz;
          p2g_particle(dx, dy, dz, qx, qy, qz, vx, vy, vz, fx, fy, fz, fxh, fyh, fzh, su, sv, sw, wu, wv, ww, bxyz);
          if (MULTI && dx == 0 && dy == 0 && dz == 0) p2g_fractions(bxyz, cur.frac[j], fs, fw);
        }
      }
    }
  }
  P2gAcc a;
  a.su = su; a.sv = sv; a.sw = sw; a.wu = wu; a.wv = wv; a.ww = ww;
  a.fs = fs; a.fw = fw;
  a.own = own; a.left = left; a.down = down; a.back = back;
  p2g_finish<FORCES, MULTI>(d, sp, x, y, z, a, u0, v0, w0, un, vn, wn, type, density, vf, nvf);
}

template <bool FORCES, bool MULTI>
__global__ void __launch_bounds__(256) k_p2g(Dims d, StepParams sp, Particles cur, const int* __restrict__ off,
                                            float* __restrict__ u0, float* __restrict__ v0,
                                            float* __restrict__ w0, float* __restrict__ un,
                                            float* __restrict__ vn, float* __restrict__ wn,
                                            int8_t* __restrict__ type, float* __restrict__ density,
                                            float4* __restrict__ vf, float4* __restrict__ nvf) {
  p2g_body<FORCES, MULTI>(d, sp, cur, off, u0, v0, w0, un, vn, wn, type, density, vf, nvf, blockIdx.x, blockIdx.y,
                          blockIdx.z);
}

// ------------------------------------------------------- shared-memory P2G
// The gather of p2g_body (same arithmetic, same (dx, dy, dz, j) order, same
// epilogue) with the particles staged in shared memory.  A CTA owns the
// nodes of one x plane, 8 y rows and 32 z columns, one per thread.  For each
// dx it stages, once and coalesced, the particles of the cells it reads in
// plane x + dx (10 rows of 34 cells: its own rows and columns and a one-cell
// rim), into cell-major slots: slot k of cell c sits at k * kP2gCells + c.
// A slot holds the particle's two x hat factors (the CTA's nodes share one
// x, so they are the particle's for the whole plane), its y and z in cell
// units and its velocity.  The 32 lanes of a warp read the k-th
// particle of 32 consecutive cells, i.e. 32 consecutive words and 32
// distinct banks, where the one-thread-per-node kernel's lanes gathered from
// scattered addresses through L1.  A cell holding more than kP2gSlots
// particles reads the rest from global memory.
constexpr int kP2gCols = 34, kP2gRows = 10, kP2gCells = kP2gCols * kP2gRows;
constexpr int p2g_smem(int slots) { return 7 * slots * kP2gCells * (int)sizeof(float); }

template <bool FORCES, bool MULTI, int kP2gSlots>
__global__ void __launch_bounds__(256, kP2gSlots <= 7 ? 3 : (kP2gSlots <= 11 ? 2 : 1)) k_p2g_tiled(Dims d, StepParams sp, Particles cur, const int* __restrict__ off,
                                                     float* __restrict__ u0, float* __restrict__ v0,
                                                     float* __restrict__ w0, float* __restrict__ un,
                                                     float* __restrict__ vn, float* __restrict__ wn,
                                                     int8_t* __restrict__ type, float* __restrict__ density,
                                                     float4* __restrict__ vf, float4* __restrict__ nvf) {
  // hat1(qx - fx), hat1(qx - fxh), qy, qz, vx, vy, vz: [kP2gSlots][kP2gCells] each (the x
  // factors are per particle: the CTA's nodes share one x)
  extern __shared__ float p2g_sm[];
  __shared__ int s_beg[kP2gCells], s_cnt[kP2gCells];
  constexpr int A = kP2gSlots * kP2gCells;
  float* const sax = p2g_sm;
  float* const sbx = sax + A;
  float* const sqy = sbx + A;
  float* const sqz = sqy + A;
  float* const svx = sqz + A;
  float* const svy = svx + A;
  float* const svz = svy + A;
  const int lane = threadIdx.x, wy = threadIdx.y, tid = wy * 32 + lane;
  const int z0 = blockIdx.x * 32, y0 = blockIdx.y * 8, x = blockIdx.z;
  const int z = z0 + lane, y = y0 + wy;
  const bool node = z < d.sz && y < d.sy;
  const float fx = (float)x, fy = (float)y, fz = (float)z;
  const float fxh = fx + 0.5f, fyh = fy + 0.5f, fzh = fz + 0.5f;
  const float inv_h = d.inv_h;
  float su = 0.f, sv = 0.f, sw = 0.f, wu = 0.f, wv = 0.f, ww = 0.f;
  float4 fs = make_float4(0.f, 0.f, 0.f, 0.f);
  float fw = 0.f;
  int own = 0, left = 0, down = 0, back = 0;
#pragma unroll
  for (int dx = -1; dx <= 1; ++dx) {
    const int X = x + dx;
    if (X < 0 || X >= d.sx) continue;  // the same for the whole CTA
    __syncthreads();                   // the previous plane's slots are consumed
    for (int lc = tid; lc < kP2gCells; lc += 256) {
      const int Y = y0 - 1 + lc / kP2gCols, Z = z0 - 1 + lc % kP2gCols;
      int b = 0, n = 0;
      if (Y >= 0 && Y < d.sy && Z >= 0 && Z < d.sz) {
        const int c = (X * d.sy + Y) * d.sz + Z;
        b = __ldg(off + c);
        n = __ldg(off + c + 1) - b;
      }
      s_beg[lc] = b;
      s_cnt[lc] = n;
      const int m = min(n, kP2gSlots);
      for (int k = 0; k < m; ++k) {
        const int j = b + k, sl = k * kP2gCells + lc;
        const float qx = __fmul_rn(__ldg(cur.px + j), inv_h);
        sax[sl] = hat1(__fsub_rn(qx, fx));
        sbx[sl] = hat1(__fsub_rn(qx, fxh));
        sqy[sl] = __fmul_rn(__ldg(cur.py + j), inv_h);
        sqz[sl] = __fmul_rn(__ldg(cur.pz + j), inv_h);
        svx[sl] = __ldg(cur.vx + j);
        svy[sl] = __ldg(cur.vy + j);
        svz[sl] = __ldg(cur.vz + j);
      }
    }
    __syncthreads();
    if (!node) continue;
    // dy and dz stay loops (the branches on them are uniform across the
    // warp): 27 unrolled copies of the particle loop overflow the
    // instruction cache
#pragma unroll 1
    for (int dy = -1; dy <= 1; ++dy) {
      const int Y = y + dy;
      if (Y < 0 || Y >= d.sy) continue;
#pragma unroll 1
      for (int dz = -1; dz <= 1; ++dz) {
        const int Z = z + dz;
        if (Z < 0 || Z >= d.sz) continue;
        const int lc = (wy + 1 + dy) * kP2gCols + lane + 1 + dz;
        const int b = s_beg[lc], n = s_cnt[lc];
        if (dx == 0 && dy == 0 && dz == 0) own = n;
        if (dx == -1 && dy == 0 && dz == 0) left = n;
        if (dx == 0 && dy == -1 && dz == 0) down = n;
        if (dx == 0 && dy == 0 && dz == -1) back = n;
        const int m = min(n, kP2gSlots);
        for (int k = 0; k < m; ++k) {  // the staged slots
          const int sl = k * kP2gCells + lc;
          float bxyz;
          p2g_particle_x(dx, dy, dz, sax[sl], sbx[sl], sqy[sl], sqz[sl], dx < 1 ? svx[sl] : 0.f,
                         dy < 1 ? svy[sl] : 0.f, dz < 1 ? svz[sl] : 0.f, fy, fz, fyh, fzh, su, sv, sw, wu, wv, ww,
                         bxyz);
          if (MULTI && dx == 0 && dy == 0 && dz == 0) p2g_fractions(bxyz, cur.frac[b + k], fs, fw);
        }
        for (int k = m; k < n; ++k) {  // a crowded cell's particles beyond the slots
          const int j = b + k;
          float bxyz;
          p2g_particle(dx, dy, dz, __fmul_rn(__ldg(cur.px + j), inv_h), __fmul_rn(__ldg(cur.py + j), inv_h),
                       __fmul_rn(__ldg(cur.pz + j), inv_h), dx < 1 ? __ldg(cur.vx + j) : 0.f,
                       dy < 1 ? __ldg(cur.vy + j) : 0.f, dz < 1 ? __ldg(cur.vz + j) : 0.f, fx, fy, fz, fxh, fyh, fzh,
                       su, sv, sw, wu, wv, ww, bxyz);
          if (MULTI && dx == 0 && dy == 0 && dz == 0) p2g_fractions(bxyz, cur.frac[j], fs, fw);
        }
      }
    }
  }
  if (!node) return;
  P2gAcc a;
  a.su = su; a.sv = sv; a.sw = sw; a.wu = wu; a.wv = wv; a.ww = ww;
  a.fs = fs; a.fw = fw;
  a.own = own; a.left = left; a.down = down; a.back = back;
  p2g_finish<FORCES, MULTI>(d, sp, x, y, z, a, u0, v0, w0, un, vn, wn, type, density, vf, nvf);
}

// node-grid virtual block -> (z block, y block, x plane) of one scene
__device__ __forceinline__ void node_block_coords(const Dims& d, int local, int& bx, int& by, int& bz) {
  const int gz = (d.sz + 31) / 32, gy = (d.sy + 7) / 8;
  bx = local % gz;
  const int t = local / gz;
  by = t % gy;
  bz = t / gy;
}

// Nodes with a coordinate equal to s: never reset by resetCellImpl, so they
// persist across steps; gravity reaches them only from the fluid cell below
// along that axis and only where fixBoundary left them AIR.
__device__ __forceinline__ void slayer_body(const Dims& d, const StepParams& sp, const int8_t* __restrict__ type,
                                            const float* __restrict__ su, const float* __restrict__ sv,
                                            const float* __restrict__ sw, float* __restrict__ u1,
                                            float* __restrict__ v1, float* __restrict__ w1, float* __restrict__ u2,
                                            float* __restrict__ v2, float* __restrict__ w2, int block) {
  int t = block * blockDim.x + threadIdx.x;
  const int na = (d.sy + 1) * (d.sz + 1), nb = d.sx * (d.sz + 1), nc = d.sx * d.sy;
  int x, y, z;
  if (t < na) {
    x = d.sx; y = t / (d.sz + 1); z = t % (d.sz + 1);
  } else if ((t -= na) < nb) {
    y = d.sy; x = t / (d.sz + 1); z = t % (d.sz + 1);
  } else if ((t -= nb) < nc) {
    z = d.sz; x = t / d.sy; y = t % d.sy;
  } else {
    return;
  }
  const bool solid = (x == d.sx && covered_x(d, y, z)) || (y == d.sy && covered_y(d, x, z)) ||
                     (z == d.sz && covered_z(d, x, y));
  const int ni = node_index(d, x, y, z);
  float u = su[ni], v = sv[ni], w = sw[ni];
  if (!solid) {
    bool add = false;
    if (x == d.sx && y < d.sy && z < d.sz) add = sp.gx_nz && type[cell_index(d, x - 1, y, z)] == kFluid;
    else if (y == d.sy && x < d.sx && z < d.sz) add = sp.gy_nz && type[cell_index(d, x, y - 1, z)] == kFluid;
    else if (z == d.sz && x < d.sx && y < d.sy) add = sp.gz_nz && type[cell_index(d, x, y, z - 1)] == kFluid;
    if (add) { u += sp.gdx; v += sp.gdy; w += sp.gdz; }
  }
  if (covered_x(d, y, z)) {
    if (x == 0) u = fmaxf(0.f, u);
    if (x == d.sx) u = fminf(0.f, u);
  }
  if (covered_y(d, x, z)) {
    if (y == 0) v = fmaxf(0.f, v);
    if (y == d.sy) v = fminf(0.f, v);
  }
  if (covered_z(d, x, y)) {
    if (z == 0) w = fmaxf(0.f, w);
    if (z == d.sz) w = fminf(0.f, w);
  }
  u1[ni] = u; v1[ni] = v; w1[ni] = w;
  u2[ni] = u; v2[ni] = v; w2[ni] = w;
}

__global__ void __launch_bounds__(256) k_slayer(Dims d, StepParams sp, const int8_t* __restrict__ type,
                                               const float* __restrict__ su, const float* __restrict__ sv,
                                               const float* __restrict__ sw, float* __restrict__ u1,
                                               float* __restrict__ v1, float* __restrict__ w1,
                                               float* __restrict__ u2, float* __restrict__ v2,
                                               float* __restrict__ w2) {
  slayer_body(d, sp, type, su, sv, sw, u1, v1, w1, u2, v2, w2, blockIdx.x);
}

// One 8x8x8 brick per CTA (threads z,y,x); (bx,by,bz) = brick coordinates
// along z, y, x.
__device__ __forceinline__ void divergence_body(const Dims& d, const int* __restrict__ off,
                                                const int8_t* __restrict__ type, const float* __restrict__ density,
                                                const float* __restrict__ un, const float* __restrict__ vn,
                                                const float* __restrict__ wn, int* __restrict__ pcount,
                                                float* __restrict__ div_out, float* __restrict__ rhs,
                                                float* __restrict__ pa, float* __restrict__ pb, int zero_init,
                                                uint8_t* __restrict__ brick_active, double* __restrict__ part_b2,
                                                int* __restrict__ part_nf, int bx, int by, int bz) {
  const int z = bx * kBrick + threadIdx.x;
  const int y = by * kBrick + threadIdx.y;
  const int x = bz * kBrick + threadIdx.z;
  double b2 = 0.0;
  int nf = 0;
  if (x < d.sx && y < d.sy && z < d.sz) {
    const int c = cell_index(d, x, y, z);
    const int ni = node_index(d, x, y, z);
    const int cnt = off[c + 1] - off[c];
    const int pc = cnt > 0 ? cnt - 1 : 0;  // cellEnd - cellStart (inclusive end; -1 - -1 when empty)
    pcount[c] = pc;
    float dv = vn[ni + d.nz] - vn[ni] + un[ni + d.nyz] - un[ni] + wn[ni + 1] - wn[ni];
    dv = (float)__dsub_rn((double)dv, __dmul_rn((double)((float)pc - 8.0f), 0.001));
    div_out[c] = dv;
    const bool fluid = type[c] == kFluid;
    const float b = fluid ? (-dv) * density[c] : 0.f;
    rhs[c] = b;
    if (!fluid || zero_init) { pa[c] = 0.f; pb[c] = 0.f; }
    if (fluid) { b2 = (double)b * (double)b; nf = 1; }
  }
  const int any = __syncthreads_or(nf);
  // deterministic block reduction
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    b2 += __shfl_xor_sync(0xffffffffu, b2, o);
    nf += __shfl_xor_sync(0xffffffffu, nf, o);
  }
  __shared__ double sb[16];
  __shared__ int sn[16];
  const int tid = threadIdx.x + kBrick * (threadIdx.y + kBrick * threadIdx.z);
  if ((tid & 31) == 0) { sb[tid >> 5] = b2; sn[tid >> 5] = nf; }
  __syncthreads();
  if (tid == 0) {
    double tb = 0.0;
    int tn = 0;
    for (int k = 0; k < 16; ++k) { tb += sb[k]; tn += sn[k]; }
    const int bid = (bz * d.by + by) * d.bz + bx;
    part_b2[bid] = tb;
    part_nf[bid] = tn;
    brick_active[bid] = any ? 1 : 0;
  }
}

__global__ void __launch_bounds__(512) k_divergence(Dims d, const int* __restrict__ off,
                                                   const int8_t* __restrict__ type,
                                                   const float* __restrict__ density,
                                                   const float* __restrict__ un, const float* __restrict__ vn,
                                                   const float* __restrict__ wn, int* __restrict__ pcount,
                                                   float* __restrict__ div_out, float* __restrict__ rhs,
                                                   float* __restrict__ pa, float* __restrict__ pb, int zero_init,
                                                   uint8_t* __restrict__ brick_active,
                                                   double* __restrict__ part_b2, int* __restrict__ part_nf) {
  divergence_body(d, off, type, density, un, vn, wn, pcount, div_out, rhs, pa, pb, zero_init, brick_active, part_b2,
                  part_nf, blockIdx.x, blockIdx.y, blockIdx.z);
}

__device__ __forceinline__ void b2_finalize_body(const double* __restrict__ part_b2, const int* __restrict__ part_nf,
                                                 int nb, SolveState* __restrict__ ss) {
  __shared__ double sb[1024];
  __shared__ int sn[1024];
  double b = 0.0;
  int n = 0;
  for (int i = threadIdx.x; i < nb; i += 1024) { b += part_b2[i]; n += part_nf[i]; }
  sb[threadIdx.x] = b;
  sn[threadIdx.x] = n;
  __syncthreads();
  for (int o = 512; o > 0; o >>= 1) {
    if (threadIdx.x < o) { sb[threadIdx.x] += sb[threadIdx.x + o]; sn[threadIdx.x] += sn[threadIdx.x + o]; }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    ss->b2 = sb[0];
    if (!isfinite(sb[0])) ss->nonfinite_seen = 1;
    ss->fluid_cells = sn[0];
    ss->iterations = 0;
    ss->bodies = 0;
    ss->converged = 0;
    ss->nonfinite = 0;
    ss->rel_residual = -1.0;
    ss->r2 = -1.0;
    ss->warm = 0;
    ss->warm_rel = -1.0;
    ss->zero_rel = -1.0;
  }
}

__global__ void __launch_bounds__(1024) k_b2_finalize(const double* __restrict__ part_b2,
                                                     const int* __restrict__ part_nf, int nb,
                                                     SolveState* __restrict__ ss) {
  b2_finalize_body(part_b2, part_nf, nb, ss);
}

// updateVelocityWithPressureImpl (Fluid/Fluid_3D_kernels.cu:118-207).
__device__ __forceinline__ void project_body(const Dims& d, const int8_t* __restrict__ type,
                                             const float* __restrict__ p, const float* __restrict__ dens,
                                             float* __restrict__ u, float* __restrict__ v, float* __restrict__ w,
                                             uint8_t* __restrict__ has, int bx, int by, int bz) {
  const int z = bx * 32 + threadIdx.x;
  const int y = by * 8 + threadIdx.y;
  const int x = bz;
  if (z >= d.sz || y >= d.sy) return;
  const int c = cell_index(d, x, y, z), ni = node_index(d, x, y, z);
  const bool t = type[c] == kFluid;
  const float pc = p[c], dc = dens[c];
  float uu = u[ni], vv = v[ni], ww = w[ni];
  uint8_t hb = 0;
  if (x > 0) {
    const int o = c - d.sy * d.sz;
    const bool lc = type[o] == kFluid;
    if (t || lc) {
      const float ld = dens[o];
      const float du = (t && lc) ? (ld + dc) / 2 : (lc ? ld : dc);
      uu = uu - __fdiv_rn(pc - p[o], du);
      hb |= 1;
    }
  }
  if (y > 0) {
    const int o = c - d.sz;
    const bool lc = type[o] == kFluid;
    if (t || lc) {
      const float ld = dens[o];
      const float du = (t && lc) ? (ld + dc) / 2 : (lc ? ld : dc);
      vv = vv - __fdiv_rn(pc - p[o], du);
      hb |= 2;
    }
  }
  if (z > 0) {
    const int o = c - 1;
    const bool lc = type[o] == kFluid;
    if (t || lc) {
      const float ld = dens[o];
      const float du = (t && lc) ? (ld + dc) / 2 : (lc ? ld : dc);
      ww = ww - __fdiv_rn(pc - p[o], du);
      hb |= 4;
    }
  }
  u[ni] = uu; v[ni] = vv; w[ni] = ww;
  has[ni] = hb;
}

__global__ void __launch_bounds__(256) k_project(Dims d, const int8_t* __restrict__ type,
                                                const float* __restrict__ p, const float* __restrict__ dens,
                                                float* __restrict__ u, float* __restrict__ v,
                                                float* __restrict__ w, uint8_t* __restrict__ has) {
  project_body(d, type, p, dens, u, v, w, has, blockIdx.x, blockIdx.y, blockIdx.z);
}

// extrapolateVelocityByOne (Fluid/Fluid_3D_kernels.cu:210-422), reading the
// previous pass only.  Neighbour order: left, down, back, right, up, front;
// each neighbour counts if it has the component and its velocity along the
// neighbour direction passes the epsilon test.
__device__ __forceinline__ void extrapolate_body(const Dims& d, const float* __restrict__ ui,
                                                 const float* __restrict__ vi, const float* __restrict__ wi,
                                                 const uint8_t* __restrict__ hi, float* __restrict__ uo,
                                                 float* __restrict__ vo, float* __restrict__ wo,
                                                 uint8_t* __restrict__ ho, int bx, int by, int bz) {
  const int z = bx * 32 + threadIdx.x;
  const int y = by * 8 + threadIdx.y;
  const int x = bz;
  if (z >= d.sz || y >= d.sy) return;
  const float eps = (float)(-1 + 1e-6);
  const int ni = node_index(d, x, y, z);
  uint8_t h = hi[ni];
  float val[3] = {ui[ni], vi[ni], wi[ni]};
  if (h != 7) {
    // neighbours: offset, exists, direction component, sign of the test
    const int offs[6] = {-d.nyz, -d.nz, -1, d.nyz, d.nz, 1};
    const bool ok[6] = {x > 0, y > 0, z > 0, x < d.sx - 1, y < d.sy - 1, z < d.sz - 1};
    uint8_t nh[6];
    float nvv[6][3];
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      if (ok[k]) {
        const int o = ni + offs[k];
        nh[k] = hi[o];
        nvv[k][0] = ui[o]; nvv[k][1] = vi[o]; nvv[k][2] = wi[o];
      } else {
        nh[k] = 0;
        nvv[k][0] = nvv[k][1] = nvv[k][2] = 0.f;
      }
    }
    uint8_t hn = h;
#pragma unroll
    for (int comp = 0; comp < 3; ++comp) {
      if (h & (1 << comp)) continue;
      float sum = 0.f;
      int cnt = 0;
#pragma unroll
      for (int k = 0; k < 6; ++k) {
        const int dir = k % 3;
        const bool pass = k < 3 ? nvv[k][dir] > eps : nvv[k][dir] < -eps;
        if (ok[k] && (nh[k] & (1 << comp)) && pass) { sum += nvv[k][comp]; cnt++; }
      }
      if (cnt > 0) {
        val[comp] = __fdiv_rn(sum, (float)cnt);
        hn |= (uint8_t)(1 << comp);
      }
    }
    h = hn;
  }
  uo[ni] = val[0]; vo[ni] = val[1]; wo[ni] = val[2];
  ho[ni] = h;
}

__global__ void __launch_bounds__(256) k_extrapolate(Dims d, const float* __restrict__ ui,
                                                    const float* __restrict__ vi, const float* __restrict__ wi,
                                                    const uint8_t* __restrict__ hi, float* __restrict__ uo,
                                                    float* __restrict__ vo, float* __restrict__ wo,
                                                    uint8_t* __restrict__ ho) {
  extrapolate_body(d, ui, vi, wi, hi, uo, vo, wo, ho, blockIdx.x, blockIdx.y, blockIdx.z);
}

// ------------------------------------------------------------------ batched
// Each batched kernel walks the virtual blocks of all scenes (grid-stride);
// every virtual block belongs to one scene and runs the same body as the
// single-scene kernel on that scene's slice of the batch arrays.

template <bool FORCES>
__global__ void __launch_bounds__(256) kb_p2g(BatchIndex bi, int total, Particles cur, const int* __restrict__ off,
                                             float* __restrict__ u0, float* __restrict__ v0, float* __restrict__ w0,
                                             float* __restrict__ un, float* __restrict__ vn, float* __restrict__ wn,
                                             int8_t* __restrict__ type, float* __restrict__ density) {
  for (int vb = blockIdx.x; vb < total; vb += gridDim.x) {
    const int s = find_scene(bi.nodes, bi.n_scenes, vb);
    const SceneDesc& S = bi.scenes[s];
    int bx, by, bz;
    node_block_coords(S.d, vb - bi.nodes[s], bx, by, bz);
    p2g_body<FORCES, false>(S.d, S.sp, cur, off + S.c_off, u0 + S.f_off, v0 + S.f_off, w0 + S.f_off, un + S.f_off,
                            vn + S.f_off, wn + S.f_off, type + S.c_off, density + S.c_off, nullptr, nullptr, bx, by,
                            bz);
  }
}

__global__ void __launch_bounds__(256) kb_slayer(BatchIndex bi, int total, const int8_t* __restrict__ type,
                                                const float* __restrict__ su, const float* __restrict__ sv,
                                                const float* __restrict__ sw, float* __restrict__ u1,
                                                float* __restrict__ v1, float* __restrict__ w1, float* __restrict__ u2,
                                                float* __restrict__ v2, float* __restrict__ w2) {
  for (int vb = blockIdx.x; vb < total; vb += gridDim.x) {
    const int s = find_scene(bi.slayer, bi.n_scenes, vb);
    const SceneDesc& S = bi.scenes[s];
    const int o = S.f_off;
    slayer_body(S.d, S.sp, type + S.c_off, su + o, sv + o, sw + o, u1 + o, v1 + o, w1 + o, u2 + o, v2 + o, w2 + o,
                vb - bi.slayer[s]);
  }
}

__global__ void __launch_bounds__(512) kb_divergence(BatchIndex bi, int total, const int* __restrict__ off,
                                                    const int8_t* __restrict__ type, const float* __restrict__ density,
                                                    const float* __restrict__ un, const float* __restrict__ vn,
                                                    const float* __restrict__ wn, int* __restrict__ pcount,
                                                    float* __restrict__ div_out, float* __restrict__ rhs,
                                                    float* __restrict__ pa, float* __restrict__ pb, int zero_init,
                                                    uint8_t* __restrict__ brick_active, double* __restrict__ part_b2,
                                                    int* __restrict__ part_nf) {
  for (int vb = blockIdx.x; vb < total; vb += gridDim.x) {
    const int s = find_scene(bi.bricks, bi.n_scenes, vb);
    const SceneDesc& S = bi.scenes[s];
    const int local = vb - bi.bricks[s];
    const int bx = local % S.d.bz, by = (local / S.d.bz) % S.d.by, bz = local / (S.d.bz * S.d.by);
    const int c = S.c_off, f = S.f_off;
    divergence_body(S.d, off + c, type + c, density + c, un + f, vn + f, wn + f, pcount + c, div_out + c, rhs + c,
                    pa + c, pb + c, zero_init, brick_active + S.br_off, part_b2 + S.br_off, part_nf + S.br_off, bx,
                    by, bz);
  }
}

// One CTA per scene; also marks every scene's pressure solve as running.
__global__ void __launch_bounds__(1024) kb_b2_finalize(BatchIndex bi, const double* __restrict__ part_b2,
                                                      const int* __restrict__ part_nf, SolveState* __restrict__ ss,
                                                      int* __restrict__ live) {
  const SceneDesc& S = bi.scenes[blockIdx.x];
  b2_finalize_body(part_b2 + S.br_off, part_nf + S.br_off, S.d.bx * S.d.by * S.d.bz, ss + blockIdx.x);
  if (threadIdx.x == 0) live[blockIdx.x] = 1;
}

__global__ void __launch_bounds__(256) kb_project(BatchIndex bi, int total, const int8_t* __restrict__ type,
                                                 const float* __restrict__ p, const float* __restrict__ dens,
                                                 float* __restrict__ u, float* __restrict__ v, float* __restrict__ w,
                                                 uint8_t* __restrict__ has) {
  for (int vb = blockIdx.x; vb < total; vb += gridDim.x) {
    const int s = find_scene(bi.nodes, bi.n_scenes, vb);
    const SceneDesc& S = bi.scenes[s];
    int bx, by, bz;
    node_block_coords(S.d, vb - bi.nodes[s], bx, by, bz);
    project_body(S.d, type + S.c_off, p + S.c_off, dens + S.c_off, u + S.f_off, v + S.f_off, w + S.f_off,
                 has + S.f_off, bx, by, bz);
  }
}

__global__ void __launch_bounds__(256) kb_extrapolate(BatchIndex bi, int total, const float* __restrict__ ui,
                                                     const float* __restrict__ vi, const float* __restrict__ wi,
                                                     const uint8_t* __restrict__ hi, float* __restrict__ uo,
                                                     float* __restrict__ vo, float* __restrict__ wo,
                                                     uint8_t* __restrict__ ho) {
  for (int vb = blockIdx.x; vb < total; vb += gridDim.x) {
    const int s = find_scene(bi.nodes, bi.n_scenes, vb);
    const SceneDesc& S = bi.scenes[s];
    int bx, by, bz;
    node_block_coords(S.d, vb - bi.nodes[s], bx, by, bz);
    const int o = S.f_off;
    extrapolate_body(S.d, ui + o, vi + o, wi + o, hi + o, uo + o, vo + o, wo + o, ho + o, bx, by, bz);
  }
}

// diffusionJacobiImpl (Fluid/Fluid_3D_kernels.cu:520-556), ping-pong.  Air
// cells keep their fractions (their pressure is already 0 after the solve).
__global__ void __launch_bounds__(256) k_diffuse(Dims d, const int8_t* __restrict__ type, float lambda,
                                                const float4* __restrict__ fin, float4* __restrict__ fout) {
  const int z = blockIdx.x * 32 + threadIdx.x;
  const int y = blockIdx.y * 8 + threadIdx.y;
  const int x = blockIdx.z;
  if (z >= d.sz || y >= d.sy) return;
  const int c = cell_index(d, x, y, z);
  if (type[c] != kFluid) { fout[c] = fin[c]; return; }
  const int nb[6] = {x + 1 < d.sx ? c + d.sy * d.sz : c, x - 1 >= 0 ? c - d.sy * d.sz : c,
                     y + 1 < d.sy ? c + d.sz : c, y - 1 >= 0 ? c - d.sz : c,
                     z + 1 < d.sz ? c + 1 : c, z - 1 >= 0 ? c - 1 : c};
  float4 r = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    const float4 f = fin[nb[k]];
    r.x += f.x * lambda; r.y += f.y * lambda; r.z += f.z * lambda; r.w += f.w * lambda;
  }
  const float4 s0 = fin[c];
  r.x += s0.x; r.y += s0.y; r.z += s0.z; r.w += s0.w;
  const float center = 1.f + 2 * lambda;
  r.x = __fdiv_rn(r.x, center); r.y = __fdiv_rn(r.y, center);
  r.z = __fdiv_rn(r.z, center); r.w = __fdiv_rn(r.w, center);
  const float s = r.x + r.y + r.z + r.w;
  r.x = __fdiv_rn(r.x, s); r.y = __fdiv_rn(r.y, s); r.z = __fdiv_rn(r.z, s); r.w = __fdiv_rn(r.w, s);
  fout[c] = r;
}

inline dim3 node_grid(const Dims& d) { return dim3((d.sz + 31) / 32, (d.sy + 7) / 8, d.sx); }

}  // namespace

cudaError_t launch_batch_p2g(cudaStream_t st, const BatchIndex& bi, int total, int grid, bool forces, Particles cur,
                             const int* off, float* u0, float* v0, float* w0, float* un, float* vn, float* wn,
                             int8_t* type, float* density) {
  if (forces)
    kb_p2g<true><<<batch_grid(kb_p2g<true>, 256, grid, total), dim3(32, 8), 0, st>>>(bi, total, cur, off, u0, v0, w0,
                                                                                   un, vn, wn, type, density);
  else
    kb_p2g<false><<<batch_grid(kb_p2g<false>, 256, grid, total), dim3(32, 8), 0, st>>>(bi, total, cur, off, u0, v0,
                                                                                     w0, un, vn, wn, type, density);
  return cudaGetLastError();
}

cudaError_t launch_batch_slayer(cudaStream_t st, const BatchIndex& bi, int total, int grid, const int8_t* type,
                                const float* su, const float* sv, const float* sw, float* u1, float* v1, float* w1,
                                float* u2, float* v2, float* w2) {
  kb_slayer<<<batch_grid(kb_slayer, 256, grid, total), 256, 0, st>>>(bi, total, type, su, sv, sw, u1, v1, w1, u2, v2, w2);
  return cudaGetLastError();
}

cudaError_t launch_batch_divergence(cudaStream_t st, const BatchIndex& bi, int total, int grid, const int* off,
                                    const int8_t* type, const float* density, const float* un, const float* vn,
                                    const float* wn, int* pcount, float* div, float* rhs, float* pa, float* pb,
                                    bool zero_init, uint8_t* brick_active, double* part_b2, int* part_nf) {
  kb_divergence<<<batch_grid(kb_divergence, 512, grid, total), dim3(kBrick, kBrick, kBrick), 0, st>>>(
      bi, total, off, type, density, un, vn, wn, pcount, div, rhs, pa, pb, zero_init ? 1 : 0, brick_active, part_b2,
      part_nf);
  return cudaGetLastError();
}

cudaError_t launch_batch_b2_finalize(cudaStream_t st, const BatchIndex& bi, const double* part_b2, const int* part_nf,
                                     SolveState* ss, int* live) {
  kb_b2_finalize<<<bi.n_scenes, 1024, 0, st>>>(bi, part_b2, part_nf, ss, live);
  return cudaGetLastError();
}

cudaError_t launch_batch_project(cudaStream_t st, const BatchIndex& bi, int total, int grid, const int8_t* type,
                                 const float* p, const float* density, float* u, float* v, float* w, uint8_t* has) {
  kb_project<<<batch_grid(kb_project, 256, grid, total), dim3(32, 8), 0, st>>>(bi, total, type, p, density, u, v, w, has);
  return cudaGetLastError();
}

cudaError_t launch_batch_extrapolate(cudaStream_t st, const BatchIndex& bi, int total, int grid, const float* ui,
                                     const float* vi, const float* wi, const uint8_t* hi, float* uo, float* vo,
                                     float* wo, uint8_t* ho) {
  kb_extrapolate<<<batch_grid(kb_extrapolate, 256, grid, total), dim3(32, 8), 0, st>>>(bi, total, ui, vi, wi, hi, uo, vo, wo, ho);
  return cudaGetLastError();
}

// 0: one thread per node through L1; 1, 2, 3: shared-memory staged with
// 11, 7 or 16 slots per cell (2, 3 or 1 CTAs per SM; with fewer slots more
// crowded cells read partly from global memory)
static int g_p2g_variant = 1;
void set_p2g_variant(int v) { g_p2g_variant = v; }
int p2g_variant() { return g_p2g_variant; }

template <bool F, bool M, int SLOTS>
static cudaError_t launch_p2g_slots(cudaStream_t st, const Dims& d, const StepParams& sp, Particles cur,
                                    const int* off, float* u0, float* v0, float* w0, float* un, float* vn,
                                    float* wn, int8_t* type, float* density, float4* vf, float4* nvf) {
  constexpr int smem = p2g_smem(SLOTS);
  cudaError_t e = cudaFuncSetAttribute(k_p2g_tiled<F, M, SLOTS>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e != cudaSuccess) return e;
  k_p2g_tiled<F, M, SLOTS><<<node_grid(d), dim3(32, 8), smem, st>>>(d, sp, cur, off, u0, v0, w0, un, vn, wn, type,
                                                                     density, vf, nvf);
  return cudaGetLastError();
}

template <bool F, bool M>
static cudaError_t launch_p2g_tiled(cudaStream_t st, const Dims& d, const StepParams& sp, Particles cur,
                                    const int* off, float* u0, float* v0, float* w0, float* un, float* vn,
                                    float* wn, int8_t* type, float* density, float4* vf, float4* nvf) {
  if (g_p2g_variant == 2)
    return launch_p2g_slots<F, M, 7>(st, d, sp, cur, off, u0, v0, w0, un, vn, wn, type, density, vf, nvf);
  if (g_p2g_variant == 3)
    return launch_p2g_slots<F, M, 16>(st, d, sp, cur, off, u0, v0, w0, un, vn, wn, type, density, vf, nvf);
  return launch_p2g_slots<F, M, 11>(st, d, sp, cur, off, u0, v0, w0, un, vn, wn, type, density, vf, nvf);
}

cudaError_t launch_p2g(cudaStream_t st, const Dims& d, const StepParams& sp, bool forces, Particles cur,
                       const int* off, int n, float* u0, float* v0, float* w0, float* un, float* vn,
                       float* wn, int8_t* type, float* density, float4* vf, float4* nvf) {
  (void)n;
  const dim3 g = node_grid(d), b(32, 8);
  const bool multi = sp.multiphase != 0;
  if (g_p2g_variant >= 1) {
    if (forces && multi)
      return launch_p2g_tiled<true, true>(st, d, sp, cur, off, u0, v0, w0, un, vn, wn, type, density, vf, nvf);
    if (forces)
      return launch_p2g_tiled<true, false>(st, d, sp, cur, off, u0, v0, w0, un, vn, wn, type, density, vf, nvf);
    if (multi)
      return launch_p2g_tiled<false, true>(st, d, sp, cur, off, u0, v0, w0, un, vn, wn, type, density, vf, nvf);
    return launch_p2g_tiled<false, false>(st, d, sp, cur, off, u0, v0, w0, un, vn, wn, type, density, vf, nvf);
  }
  if (forces && multi)
    k_p2g<true, true><<<g, b, 0, st>>>(d, sp, cur, off, u0, v0, w0, un, vn, wn, type, density, vf, nvf);
  else if (forces)
    k_p2g<true, false><<<g, b, 0, st>>>(d, sp, cur, off, u0, v0, w0, un, vn, wn, type, density, vf, nvf);
  else if (multi)
    k_p2g<false, true><<<g, b, 0, st>>>(d, sp, cur, off, u0, v0, w0, un, vn, wn, type, density, vf, nvf);
  else
    k_p2g<false, false><<<g, b, 0, st>>>(d, sp, cur, off, u0, v0, w0, un, vn, wn, type, density, vf, nvf);
  return cudaGetLastError();
}

cudaError_t launch_slayer(cudaStream_t st, const Dims& d, const StepParams& sp, const int8_t* type,
                          const float* su, const float* sv, const float* sw, float* u1, float* v1, float* w1,
                          float* u2, float* v2, float* w2) {
  const int m = d.F - d.C;
  k_slayer<<<(m + 255) / 256, 256, 0, st>>>(d, sp, type, su, sv, sw, u1, v1, w1, u2, v2, w2);
  return cudaGetLastError();
}

cudaError_t launch_divergence(cudaStream_t st, const Dims& d, const int* off, const int8_t* type,
                              const float* density, const float* un, const float* vn, const float* wn,
                              int* pcount, float* div, float* rhs, float* pa, float* pb, bool zero_init,
                              uint8_t* brick_active, double* part_b2, int* part_nf, int* nblocks_out) {
  const dim3 g(d.bz, d.by, d.bx), b(kBrick, kBrick, kBrick);
  if (nblocks_out) *nblocks_out = d.bx * d.by * d.bz;
  k_divergence<<<g, b, 0, st>>>(d, off, type, density, un, vn, wn, pcount, div, rhs, pa, pb, zero_init ? 1 : 0,
                                brick_active, part_b2, part_nf);
  return cudaGetLastError();
}

cudaError_t launch_b2_finalize(cudaStream_t st, const double* part_b2, const int* part_nf, int nblocks,
                               SolveState* ss) {
  k_b2_finalize<<<1, 1024, 0, st>>>(part_b2, part_nf, nblocks, ss);
  return cudaGetLastError();
}

cudaError_t launch_project(cudaStream_t st, const Dims& d, const int8_t* type, const float* p,
                           const float* density, float* u, float* v, float* w, uint8_t* has) {
  k_project<<<node_grid(d), dim3(32, 8), 0, st>>>(d, type, p, density, u, v, w, has);
  return cudaGetLastError();
}

cudaError_t launch_extrapolate(cudaStream_t st, const Dims& d, const float* ui, const float* vi,
                               const float* wi, const uint8_t* hi, float* uo, float* vo, float* wo,
                               uint8_t* ho) {
  k_extrapolate<<<node_grid(d), dim3(32, 8), 0, st>>>(d, ui, vi, wi, hi, uo, vo, wo, ho);
  return cudaGetLastError();
}

cudaError_t launch_diffuse(cudaStream_t st, const Dims& d, const int8_t* type, float lambda,
                           const float4* fin, float4* fout) {
  k_diffuse<<<node_grid(d), dim3(32, 8), 0, st>>>(d, type, lambda, fin, fout);
  return cudaGetLastError();
}

}  // namespace aqb
