// Host side of the B200 FLIP step: configuration, particle seeding, device
// memory, stage sequencing, CUDA-graph capture and the C ABI declared in
// include/aquarius_b200.h.
//
// Reference surface: Fluid_3D_FLIP::Fluid (Fluid/Fluid_3D_FLIP.cuh:53-156),
// init (Fluid/Fluid_3D_FLIP.cu:435-505), simulationStep (:316-352).
#include <cmath>
#include <cstdlib>
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <stdlib.h>
#include <string>
#include <vector>

#include "../../include/aquarius_b200.h"
#include "fluid_impl.cuh"
#include "unet_impl.cuh"

using namespace aqb;

namespace {

thread_local std::string g_last_error;

#define AQ_CUDA(call)                                                                            \
  do {                                                                                           \
    cudaError_t e_ = (call);                                                                     \
    if (e_ != cudaSuccess)                                                                       \
      return fail(e_ == cudaErrorMemoryAllocation ? AQ_ERR_OUT_OF_MEMORY : AQ_ERR_CUDA,          \
                  std::string(#call) + ": " + cudaGetErrorString(e_));                           \
  } while (0)

#define AQ_TRY(expr)              \
  do {                            \
    aq_status s_ = (expr);        \
    if (s_ != AQ_OK) return s_;   \
  } while (0)

__global__ void k_copy_f(const float* __restrict__ a, float* __restrict__ b, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) b[i] = a[i];
}

// Sweeps run from each start of the learned warm start before they are compared.
constexpr int kWarmSweeps = 20;

// Learned warm start: compares the FP64 residuals after kWarmSweeps sweeps
// from the network's prediction and from zero (partial sums summed in the
// fixed order of the residual finaliser); the zero-init path wins when the
// prediction's residual is larger (or not finite).
__global__ void __launch_bounds__(1024) k_pick_start(const double* __restrict__ pl, const double* __restrict__ pz,
                                                     int nparts, SolveState* __restrict__ ss, int* __restrict__ pick,
                                                     double tol) {
  __shared__ double sa[1024], sb[1024];
  double a = 0.0, b = 0.0;
  for (int i = threadIdx.x; i < nparts; i += 1024) {
    a += pl[i];
    b += pz[i];
  }
  sa[threadIdx.x] = a;
  sb[threadIdx.x] = b;
  __syncthreads();
  for (int o = 512; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      sa[threadIdx.x] += sa[threadIdx.x + o];
      sb[threadIdx.x] += sb[threadIdx.x + o];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const double rl = rel_residual_of(sa[0], ss->b2), rz = rel_residual_of(sb[0], ss->b2);
    const bool zero_wins = !(rl <= rz);
    *pick = zero_wins ? 1 : 0;
    ss->warm = zero_wins ? 2 : 1;
    ss->warm_rel = rl;
    ss->zero_rel = rz;
    const double rel = zero_wins ? rz : rl;
    ss->iterations = kWarmSweeps;
    ss->total_sweeps += 2 * kWarmSweeps;
    ss->r2 = zero_wins ? sb[0] : sa[0];
    ss->rel_residual = rel;
    if (!isfinite(rel)) ss->nonfinite = ss->nonfinite_seen = 1;
    ss->converged = (isfinite(rel) && rel <= tol) ? 1 : 0;
  }
}

__global__ void k_copy_if(const int* __restrict__ pick, const float* __restrict__ a, float* __restrict__ b, int n) {
  if (*pick == 0) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) b[i] = a[i];
}

int covered_faces(int s1, int s2) {  // fixBoundary launch coverage (Fluid/Fluid_3D_common.cu:13-41)
  const int total = s1 * s2;
  const int nt = total < 1024 ? total : 1024;
  const int nb = nt == 0 ? 1 : (total % nt != 0 ? total / nt + 1 : total / nt);
  const int t = nb * nt;
  const int faces = (s1 + 1) * (s2 + 1);
  return t < faces ? t : faces;
}

// ------------------------------------------------------------------ seeding
// Fluid::createParticlesAt / createSquareFluid / createSphereFluid
// (Fluid/Fluid_3D_FLIP.cu:508-594).  The jitter comes from glibc rand()
// (Common/Commons.h:3-5); random_r with a 128-byte state replays
// srand(seed); rand() exactly.  Jitter is drawn before the sphere filter, so
// rejected sub-cells consume the sequence too.
struct Seeder {
  const aq_config& cfg;
  int sx, sy, sz;
  float h;
  aqb::HostRand& rng;
  std::vector<float> pos;  // xyz interleaved
  std::vector<int> phase;

  Seeder(const aq_config& c, float h_, aqb::HostRand& r)
      : cfg(c), sx(c.size_x), sy(c.size_y), sz(c.size_z), h(h_), rng(r) {}
  float random0to1() { return rng.random0to1(); }
  void at(float cx, float cy, float cz, bool sphere, float scx, float scy, float scz, float rad, float spacing,
          int ph) {
    const float jit = cfg.particle_jitter;
    for (float dx = 0; dx <= 1; ++dx)
      for (float dy = 0; dy <= 1; ++dy)
        for (float dz = 0; dz <= 1; ++dz) {
          float px = (float)(dx - 0.5) * spacing + cx;
          float py = (float)(dy - 0.5) * spacing + cy;
          float pz = (float)(dz - 0.5) * spacing + cz;
          const float xj = random0to1() - 0.5f, yj = random0to1() - 0.5f, zj = random0to1() - 0.5f;
          px += xj * spacing * jit;
          py += yj * spacing * jit;
          pz += zj * spacing * jit;
          const float md = spacing / 2;
          px = fmaxf(md, fminf((float)sx * h - md, px));
          py = fmaxf(md, fminf((float)sy * h - md, py));
          pz = fmaxf(md, fminf((float)sz * h - md, pz));
          bool keep = true;
          if (sphere) {
            const float ex = px - scx, ey = py - scy, ez = pz - scz;
            const float len = sqrtf(ex * ex + ey * ey + ez * ez);
            keep = len < rad * h * (float)sy;
          }
          if (keep) {
            pos.push_back(px);
            pos.push_back(py);
            pos.push_back(pz);
            phase.push_back(ph);
          }
        }
  }
  static bool valid01(const float* c) {
    return !(c[0] < 0 || c[1] < 0 || c[2] < 0) && !(c[0] > 1 || c[1] > 1 || c[2] > 1);
  }
  void center(int x, int y, int z, float& cx, float& cy, float& cz) const {
    cx = ((float)x + 0.5f) * h;
    cy = ((float)y + 0.5f) * h;
    cz = ((float)z + 0.5f) * h;
  }
  void square(const aq_volume& v) {
    if (!valid01(v.box_min) || !valid01(v.box_max)) return;
    float cx, cy, cz;
    for (int z = (int)(v.box_min[2] * (float)sz); (float)z < v.box_max[2] * (float)sz; ++z)
      for (int x = (int)(v.box_min[0] * (float)sx); (float)x < v.box_max[0] * (float)sx; ++x)
        for (int y = (int)(v.box_min[1] * (float)sy); (float)y < v.box_max[1] * (float)sy; ++y) {
          center(x, y, z, cx, cy, cz);
          at(cx, cy, cz, false, 0, 0, 0, 0, h / 2, v.phase);
        }
  }
  void sphere(const aq_volume& v) {
    if (!valid01(v.ball_center)) return;
    const float scx = (v.ball_center[0] * (float)sx * h);
    const float scy = (v.ball_center[1] * (float)sy * h);
    const float scz = (v.ball_center[2] * (float)sz * h);
    float cx, cy, cz;
    for (int y = 0; y < sy; ++y)
      for (int x = 0; x < sx; ++x)
        for (int z = 0; z < sz; ++z) {
          center(x, y, z, cx, cy, cz);
          at(cx, cy, cz, true, scx, scy, scz, v.ball_radius, h / 2, v.phase);
        }
  }
  // Fluid::createSquareInk (Fluid/Fluid_3D_FLIP.cu:600-640): a lattice of
  // the given spacing from box_min*size + spacing/2 up to box_max*size -
  // (spacing/2 - 1e-3), loops x, y, z, each point jittered by
  // (random0to1() - 0.5) * spacing/2 and clamped spacing/2 off the walls.
  void square_ink(const aq_volume& v, float spacing) {
    const float md = spacing / 2.f;
    const float gx = (float)sx * h, gy = (float)sy * h, gz = (float)sz * h;
    const float shrink = (float)((double)md - 1e-3);
    const float x0 = v.box_min[0] * gx + md, y0 = v.box_min[1] * gy + md, z0 = v.box_min[2] * gz + md;
    const float x1 = v.box_max[0] * gx - shrink, y1 = v.box_max[1] * gy - shrink, z1 = v.box_max[2] * gz - shrink;
    const float mag = spacing / 2.f;
    for (float x = x0; x <= x1; x += spacing)
      for (float y = y0; y <= y1; y += spacing)
        for (float z = z0; z <= z1; z += spacing) {
          // (random0to1() - 0.5) is evaluated in double and stored as float
          float jx = (float)((double)random0to1() - 0.5);
          float jy = (float)((double)random0to1() - 0.5);
          float jz = (float)((double)random0to1() - 0.5);
          jx *= mag; jy *= mag; jz *= mag;
          const float px = fminf(gx - md, fmaxf(md, x + jx));
          const float py = fminf(gy - md, fmaxf(md, y + jy));
          const float pz = fminf(gz - md, fmaxf(md, z + jz));
          pos.push_back(px);
          pos.push_back(py);
          pos.push_back(pz);
          phase.push_back(v.phase);
        }
  }
  // Fluid::createSphereInk (Fluid/Fluid_3D_FLIP.cu:642-664): the particle
  // seeding (8 jittered sub-points at spacing h/2, sphere filter) at every
  // point of a lattice of the given spacing from 0, loops z, y, x.
  void sphere_ink(const aq_volume& v, float spacing) {
    if (!valid01(v.ball_center)) return;
    const float scx = (v.ball_center[0] * (float)sx * h);
    const float scy = (v.ball_center[1] * (float)sy * h);
    const float scz = (v.ball_center[2] * (float)sz * h);
    const float gx = (float)sx * h, gy = (float)sy * h, gz = (float)sz * h;
    for (float z = 0; z < gz; z += spacing)
      for (float y = 0; y < gy; y += spacing)
        for (float x = 0; x < gx; x += spacing) at(x, y, z, true, scx, scy, scz, v.ball_radius, h / 2, v.phase);
  }
};

}  // namespace

aq_status aqb::set_last_error(aq_status st, const std::string& msg) {
  g_last_error = msg;
  return st;
}

// Plans whose residual is a separate pass over the final iterate (flat, cube
// and list); the x-streaming tiled plans (rows 8/16/32) fuse it into their
// last launch as an extra level.
static bool separate_residual(const aqb::JacobiPlan& p) { return p.by == 0 || p.by == 2 || p.by == 3; }

// =================================================================== fluid
// ------------------------------------------------------------- allocation
aq_status aq_fluid::allocate() {
  const size_t N = (size_t)n, C = (size_t)d.C, F = (size_t)d.F;
  AQ_TRY(alloc(&cur.px, N)); AQ_TRY(alloc(&cur.py, N)); AQ_TRY(alloc(&cur.pz, N));
  AQ_TRY(alloc(&cur.vx, N)); AQ_TRY(alloc(&cur.vy, N)); AQ_TRY(alloc(&cur.vz, N));
  AQ_TRY(alloc(&tmp.px, N)); AQ_TRY(alloc(&tmp.py, N)); AQ_TRY(alloc(&tmp.pz, N));
  AQ_TRY(alloc(&tmp.vx, N)); AQ_TRY(alloc(&tmp.vy, N)); AQ_TRY(alloc(&tmp.vz, N));
  AQ_TRY(alloc(&cur.frac, N)); AQ_TRY(alloc(&tmp.frac, N));
  AQ_TRY(alloc(&key, N)); AQ_TRY(alloc(&slot, N)); AQ_TRY(alloc(&perm_u, N)); AQ_TRY(alloc(&sort_index, N));
  AQ_TRY(alloc(&count, C + 1)); AQ_TRY(alloc(&off, C + 1));
  AQ_TRY(alloc(&tile_sums, cell_scan_tiles(d.C)));
  AQ_TRY(alloc(&u0, F)); AQ_TRY(alloc(&v0, F)); AQ_TRY(alloc(&w0, F));
  AQ_TRY(alloc(&un1, F)); AQ_TRY(alloc(&vn1, F)); AQ_TRY(alloc(&wn1, F));
  AQ_TRY(alloc(&un2, F)); AQ_TRY(alloc(&vn2, F)); AQ_TRY(alloc(&wn2, F));
  AQ_TRY(alloc(&h1, F)); AQ_TRY(alloc(&h2, F));
  AQ_TRY(alloc(&type, C)); AQ_TRY(alloc(&density, C)); AQ_TRY(alloc(&div, C)); AQ_TRY(alloc(&rhs, C));
  AQ_TRY(alloc(&pa, C)); AQ_TRY(alloc(&pb, C)); AQ_TRY(alloc(&pcount, C));
  AQ_TRY(alloc(&vf, C)); AQ_TRY(alloc(&nvf, C)); AQ_TRY(alloc(&nvf2, C));
  nbricks = d.bx * d.by * d.bz;
  AQ_TRY(alloc(&bact, (size_t)nbricks)); AQ_TRY(alloc(&part_b2, (size_t)nbricks));
  AQ_TRY(alloc(&part_nf, (size_t)nbricks));
  jpart_cap = 0;
  for (int lv : {1, 2, 4, 8})
    for (int res = 0; res < 2; ++res) {
      JacobiPlan p = plan;
      p.levels = lv;
      const int k = jacobi_parts(d, p, res != 0);
      if (k > jpart_cap) jpart_cap = k;
    }
  if (jpart_cap < 1) jpart_cap = 1;
  AQ_TRY(alloc(&jpart, (size_t)jpart_cap));
  AQ_TRY(alloc(&ss, 1));
  AQ_CUDA(cudaMallocHost(&ss_host, sizeof(SolveState)));
  int sms = 0;
  AQ_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  AQ_TRY(alloc(&bar, 1));
  AQ_TRY(alloc(&tiles, (size_t)resident_tile_capacity(d)));
  AQ_TRY(alloc(&n_tiles, 1));
  if (d.sz % 4 == 0) ctas = persist_ctas(device);
  // partials of the persistent and resident solves: one per CTA (at most one per SM)
  AQ_TRY(alloc(&ppart, (size_t)std::max({ctas, sms, 1})));
  if (d.sz % 4 == 0) {
    AQ_TRY(alloc(&items, (size_t)persist_items(d)));
    AQ_TRY(alloc(&n_items, 1));
    AQ_TRY(alloc(&row_items, (size_t)row_items_capacity(d)));
    AQ_TRY(alloc(&n_row_items, 1));
    AQ_TRY(alloc(&resid_ticket, 1));
  }
  // default Jacobi plan: one vectorised sweep per launch over the listed
  // active warp rows where z allows it, otherwise the tiled kernel with two
  // sweeps per launch
  plan = d.sz % 4 == 0 ? JacobiPlan{1, 3, 1} : JacobiPlan{2, 16, 16};
  // room for the default plan's residual partials: the flat pass, or the
  // fused residual level of every launch size split_sweeps can produce
  int need = d.sz % 4 == 0 ? resid_flat_parts(d) : 0;
  for (int l = plan.levels; l >= 1 && !separate_residual(plan); l >>= 1) {
    JacobiPlan q = plan;
    q.levels = l;
    need = std::max(need, jacobi_parts(d, q, true));
  }
  if (need > jpart_cap) {
    jpart_cap = need;
    AQ_TRY(alloc(&jpart, (size_t)jpart_cap));
  }
  memset(ss_host, 0, sizeof(SolveState));
  return AQ_OK;
}

// ------------------------------------------------------------------ stages
aq_status aq_fluid::enq_particles(bool move) {
  AQ_CUDA(launch_particles_advance(stream, d, sp, move, cur, tmp, u0, v0, w0, un2, vn2, wn2, nvf, key, slot,
                                   count, n));
  AQ_CUDA(launch_cell_scan(stream, d.C, count, off, tile_sums));
  AQ_CUDA(launch_scatter(stream, key, slot, off, perm_u, n));
  AQ_CUDA(launch_rank_gather(stream, multiphase, key, off, perm_u, tmp, cur, sort_index, n));
  return AQ_OK;
}

aq_status aq_fluid::enq_p2g(bool forces) {
  AQ_CUDA(launch_p2g(stream, d, sp, forces, cur, off, n, u0, v0, w0, un1, vn1, wn1, type, density, vf, nvf));
  if (forces) {
    AQ_CUDA(launch_slayer(stream, d, sp, type, un2, vn2, wn2, un1, vn1, wn1, un2, vn2, wn2));
  }
  nv_cur = 1;
  return AQ_OK;
}

aq_status aq_fluid::enq_divergence() {
  int nb = 0;
  AQ_CUDA(launch_divergence(stream, d, off, type, density, nvx(nv_cur), nvy(nv_cur), nvz(nv_cur), pcount, div,
                            rhs, pa, pb, cfg.pressure_init != AQ_PRESSURE_CARRY, bact, part_b2, part_nf, &nb));
  AQ_CUDA(launch_b2_finalize(stream, part_b2, part_nf, nb, ss));
  AQ_TRY(enq_row_items());
  return AQ_OK;
}

// Sweep counts per launch for `sweeps` sweeps with the plan's level count.
static std::vector<int> split_sweeps(int sweeps, int levels) {
  std::vector<int> out;
  int left = sweeps;
  while (left > 0) {
    int l = levels;
    while (l > left) l >>= 1;
    out.push_back(l);
    left -= l;
  }
  return out;
}

static int jacobi_launches(const JacobiPlan& plan, int sweeps) {
  if (plan.by == 1 || plan.by == 4) return 2;  // work list + the cooperative solve
  const int k = (int)split_sweeps(sweeps, plan.levels).size();
  // sweeps, parity copy, finalize, separate residual pass (flat, cube and list plans)
  return k + (k % 2) + 1 + (separate_residual(plan) ? 1 : 0);
}

int aq_fluid::count_jacobi_launches(int sweeps) const { return jacobi_launches(plan, sweeps); }

// `sweeps` Jacobi sweeps from pa; the last launch also writes the residual
// partials of its output; the result ends in pa.
// `sweeps` Jacobi sweeps from pa; the FP64 residual partials of the final
// iterate are written to jpart; the result ends in pa.  Tiled plans fuse the
// residual into their last launch (one extra level); the flat plan computes
// it with one residual pass over the final iterate.
// The same with an explicit plan and buffer pair (result in `a`, residual
// partials in `part`).
static aq_status enqueue_sweeps_on(aq_fluid* f, const JacobiPlan& plan, float* a, float* b, int sweeps,
                                   bool with_residual, double* part) {
  const std::vector<int> parts = split_sweeps(sweeps, plan.levels);
  const bool flat = separate_residual(plan);
  float* bufs[2] = {a, b};
  for (size_t k = 0; k < parts.size(); ++k) {
    if (plan.by == 3) {
      AQ_CUDA(launch_jacobi_list(f->stream, f->d, bufs[k % 2], bufs[(k + 1) % 2], f->rhs, f->type, f->row_items,
                                 f->n_row_items, k > 0));
      continue;
    }
    const bool last = k + 1 == parts.size();
    JacobiPlan p = plan;
    p.levels = parts[k];
    int np = 0;
    AQ_CUDA(launch_jacobi(f->stream, f->d, p, last && with_residual && !flat, bufs[k % 2], bufs[(k + 1) % 2],
                          f->rhs, f->type, f->bact, part, &np));
  }
  if (flat && with_residual && !parts.empty())
    AQ_CUDA(launch_resid_flat(f->stream, f->d, bufs[parts.size() % 2], f->rhs, f->type, f->bact, part));
  if (parts.size() % 2 == 1) {
    k_copy_f<<<(f->d.C + 255) / 256, 256, 0, f->stream>>>(b, a, f->d.C);
    AQ_CUDA(cudaGetLastError());
  }
  return AQ_OK;
}

static aq_status enqueue_sweeps(aq_fluid* f, int sweeps, bool with_residual = true) {
  return enqueue_sweeps_on(f, f->plan, f->pa, f->pb, sweeps, with_residual, f->jpart);
}

static int last_parts_of(const aq_fluid* f, const JacobiPlan& plan, int sweeps) {
  const std::vector<int> parts = split_sweeps(sweeps, plan.levels);
  if (parts.empty()) return 0;
  if (separate_residual(plan)) return resid_flat_parts(f->d);
  JacobiPlan p = plan;
  p.levels = parts.back();
  return jacobi_parts(f->d, p, true);
}

static int last_parts(const aq_fluid* f, int sweeps) { return last_parts_of(f, f->plan, sweeps); }

aq_status aq_fluid::enq_row_items() {
  // the list plan's rows; the resident plan's learned start sweeps them too
  const bool warm_rows = plan.by == 4 && cfg.pressure_init == AQ_PRESSURE_LEARNED && d.sz % 4 == 0;
  if (plan.by != 3 && !warm_rows) return AQ_OK;
  AQ_CUDA(launch_row_items(stream, d, bact, row_items, n_row_items));
  return AQ_OK;
}

int aq_fluid::solve_sweeps_done() const { return cfg.pressure_init == AQ_PRESSURE_LEARNED ? kWarmSweeps : 0; }

// AQ_PRESSURE_LEARNED: pa <- network prediction; kWarmSweeps sweeps from it
// and from zero; the solve continues in pa from the better of the two.
aq_status aq_fluid::enq_learned_start() {
  if (!net || !net_acts) return fail(AQ_ERR_INVALID_CONFIG, "AQ_PRESSURE_LEARNED needs a network (aq_fluid_set_warm_start)");
  AQ_TRY(unet_predict(net, stream, net_acts, rhs, type, pa));
  // the two short starts run one sweep per launch (the list plan) when the
  // solve itself is the resident plan
  const JacobiPlan wp = plan.by == 4 ? JacobiPlan{1, 3, 1} : plan;
  AQ_TRY(enqueue_sweeps_on(this, wp, pa, pb, kWarmSweeps, true, jpart));
  AQ_CUDA(cudaMemsetAsync(za, 0, sizeof(float) * d.C, stream));
  AQ_CUDA(cudaMemsetAsync(zb, 0, sizeof(float) * d.C, stream));
  AQ_TRY(enqueue_sweeps_on(this, wp, za, zb, kWarmSweeps, true, jpart2));
  k_pick_start<<<1, 1024, 0, stream>>>(jpart, jpart2, last_parts_of(this, wp, kWarmSweeps), ss, pick,
                                       cfg.solve_mode == AQ_SOLVE_RESIDUAL ? (double)cfg.rel_residual : 0.0);
  AQ_CUDA(cudaGetLastError());
  k_copy_if<<<std::min((d.C + 255) / 256, 148 * 8), 256, 0, stream>>>(pick, za, pa, d.C);
  AQ_CUDA(cudaGetLastError());
  return AQ_OK;
}

// The whole solve as one cooperative launch (plan.by == 1).
static aq_status enqueue_persistent(aq_fluid* f, int fixed_sweeps) {
  AQ_CUDA(launch_items_compact(f->stream, f->d, f->bact, f->items, f->n_items, f->bar));
  AQ_CUDA(launch_persist_solve(f->stream, f->d, f->ctas, f->pa, f->pb, f->rhs, f->type, f->items, f->n_items, f->bar,
                               f->ppart, f->ss, fixed_sweeps, f->cfg.check_interval, f->cfg.max_iterations,
                               (double)f->cfg.rel_residual, f->barrier_test));
  return AQ_OK;
}

// The whole solve as one cooperative launch of resident tiles (plan.by == 4).
static aq_status enqueue_resident(aq_fluid* f, int fixed_sweeps) {
  AQ_CUDA(launch_resident_solve(f->stream, f->d, f->plan.xc, f->plan.levels, f->res_ctas, f->pa, f->pb, f->rhs,
                                f->type, f->bact, f->tiles, f->n_tiles, f->bar, f->ppart, f->ss, fixed_sweeps,
                                f->cfg.check_interval, f->cfg.max_iterations, (double)f->cfg.rel_residual,
                                f->barrier_test));
  return AQ_OK;
}

aq_status aq_fluid::enq_solve_fixed(int sweeps) {
  if (sweeps <= 0) return AQ_OK;
  if (plan.by == 1) return enqueue_persistent(this, sweeps);
  if (plan.by == 4) return enqueue_resident(this, sweeps);
  AQ_TRY(enqueue_sweeps(this, sweeps));
  AQ_CUDA(launch_resid_finalize(stream, jpart, last_parts(this, sweeps), ss, sweeps, 0.0, 0, false, 0));
  return AQ_OK;
}

aq_status aq_fluid::enq_solve_body(bool set_cond, unsigned long long handle, int* launches) {
  const int m = cfg.check_interval;
  if (separate_residual(plan) && d.sz % 4 == 0) {
    // plans whose residual is a separate pass: pass and check in one launch
    AQ_TRY(enqueue_sweeps(this, m, false));
    if (plan.by == 3)
      AQ_CUDA(launch_resid_list_fin(stream, d, pa, rhs, type, row_items, n_row_items, jpart, resid_ticket, ss, m,
                                    (double)cfg.rel_residual, cfg.max_iterations, set_cond, handle));
    else
      AQ_CUDA(launch_resid_flat_fin(stream, d, pa, rhs, type, bact, jpart, resid_ticket, ss, m,
                                    (double)cfg.rel_residual, cfg.max_iterations, set_cond, handle));
    if (launches) *launches = count_jacobi_launches(m) - 1;
    return AQ_OK;
  }
  AQ_TRY(enqueue_sweeps(this, m));
  AQ_CUDA(launch_resid_finalize(stream, jpart, last_parts(this, m), ss, m, (double)cfg.rel_residual,
                                cfg.max_iterations, set_cond, handle));
  if (launches) *launches = count_jacobi_launches(m);
  return AQ_OK;
}

// Residual mode without a graph: the host reads the solve state after each block.
aq_status aq_fluid::enq_solve_residual_eager() {
  if (plan.by == 1) return enqueue_persistent(this, 0);
  if (plan.by == 4) return enqueue_resident(this, 0);
  for (int guard = 0; guard < 1000000; ++guard) {
    AQ_TRY(enq_solve_body(false, 0, nullptr));
    AQ_CUDA(cudaMemcpyAsync(ss_host, ss, sizeof(SolveState), cudaMemcpyDeviceToHost, stream));
    AQ_CUDA(cudaStreamSynchronize(stream));
    const SolveState& s = *ss_host;
    if (s.converged || s.nonfinite || s.iterations >= cfg.max_iterations) break;
  }
  return AQ_OK;
}

aq_status aq_fluid::enq_project() {
  AQ_CUDA(launch_project(stream, d, type, pa, density, nvx(nv_cur), nvy(nv_cur), nvz(nv_cur), hb(nv_cur)));
  has_cur = nv_cur;
  return AQ_OK;
}

aq_status aq_fluid::enq_extrapolate() {
  // extrapolateVelocity: 3 passes (Fluid/Fluid_3D_common.cu:65-82); ends in buffer 2.
  int a = nv_cur, b = 3 - nv_cur;
  if (has_cur != nv_cur) {
    // has bits must sit beside the velocities they describe
    AQ_CUDA(cudaMemcpyAsync(hb(nv_cur), hb(has_cur), (size_t)d.F, cudaMemcpyDeviceToDevice, stream));
  }
  for (int pass = 0; pass < 3; ++pass) {
    AQ_CUDA(launch_extrapolate(stream, d, nvx(a), nvy(a), nvz(a), hb(a), nvx(b), nvy(b), nvz(b), hb(b)));
    std::swap(a, b);
  }
  nv_cur = a;
  has_cur = a;
  if (nv_cur != 2) {
    // keep the invariant that the step's final newVelocity lives in buffer 2
    AQ_CUDA(cudaMemcpyAsync(un2, un1, sizeof(float) * d.F, cudaMemcpyDeviceToDevice, stream));
    AQ_CUDA(cudaMemcpyAsync(vn2, vn1, sizeof(float) * d.F, cudaMemcpyDeviceToDevice, stream));
    AQ_CUDA(cudaMemcpyAsync(wn2, wn1, sizeof(float) * d.F, cudaMemcpyDeviceToDevice, stream));
    AQ_CUDA(cudaMemcpyAsync(h2, h1, (size_t)d.F, cudaMemcpyDeviceToDevice, stream));
    nv_cur = has_cur = 2;
  }
  return AQ_OK;
}

aq_status aq_fluid::enq_diffuse() {
  // solveDiffusionJacobi (Fluid/Fluid_3D_common.cu:85-91).  With every
  // particle in one phase, each fluid cell holds the same one-hot vector and
  // a sweep maps it to itself exactly (x/x = 1 in IEEE arithmetic), so the
  // sweeps are skipped; air pressure is already 0 after the solve.
  if (!multiphase || cfg.diffusion_iterations <= 0) return AQ_OK;
  const float lambda = cfg.diffusion_coeff * cfg.timestep / (d.h * d.h);
  float4* a = nvf;
  float4* b = nvf2;
  for (int i = 0; i < cfg.diffusion_iterations; ++i) {
    AQ_CUDA(launch_diffuse(stream, d, type, lambda, a, b));
    std::swap(a, b);
  }
  if (a != nvf) AQ_CUDA(cudaMemcpyAsync(nvf, a, sizeof(float4) * d.C, cudaMemcpyDeviceToDevice, stream));
  return AQ_OK;
}

aq_status aq_fluid::run_stage(int stage) {
  if (stage != AQ_STAGE_SORT) sorted_by_stage1 = false;
  switch (stage) {
    case AQ_STAGE_G2P_ADVECT:
      // transferToParticles + moveParticles run fused with the spatial hash
      // and sort, so the particles come out sorted already.
      AQ_TRY(enq_particles(true));
      sorted_by_stage1 = true;
      return AQ_OK;
    case AQ_STAGE_SORT:
      if (!sorted_by_stage1) AQ_TRY(enq_particles(false));
      sorted_by_stage1 = false;
      return AQ_OK;
    case AQ_STAGE_P2G: return enq_p2g(true);
    case AQ_STAGE_DIVERGENCE: return enq_divergence();
    case AQ_STAGE_PRESSURE:
      if (cfg.pressure_init != AQ_PRESSURE_CARRY) {  // done by the divergence kernel inside a step
        AQ_CUDA(cudaMemsetAsync(pa, 0, sizeof(float) * d.C, stream));
        AQ_CUDA(cudaMemsetAsync(pb, 0, sizeof(float) * d.C, stream));
      }
      if (cfg.pressure_init == AQ_PRESSURE_LEARNED) AQ_TRY(enq_learned_start());
      if (cfg.solve_mode == AQ_SOLVE_RESIDUAL) return enq_solve_residual_eager();
      return enq_solve_fixed(cfg.pressure_iterations - solve_sweeps_done());
    case AQ_STAGE_PROJECT: return enq_project();
    case AQ_STAGE_EXTRAPOLATE: return enq_extrapolate();
    case AQ_STAGE_DIFFUSE:
      AQ_TRY(enq_diffuse());
      AQ_TRY(enq_ink());
      time += (double)cfg.timestep;
      return AQ_OK;
    default: return fail(AQ_ERR_INVALID_ARGUMENT, "unknown stage");
  }
}

aq_status aq_fluid::enq_pre_solve() {
  nv_cur = 2;
  AQ_TRY(enq_particles(true));
  AQ_TRY(enq_p2g(true));
  AQ_TRY(enq_divergence());
  if (cfg.pressure_init == AQ_PRESSURE_LEARNED) AQ_TRY(enq_learned_start());
  return AQ_OK;
}

aq_status aq_fluid::enq_post_solve() {
  AQ_TRY(enq_project());
  AQ_TRY(enq_extrapolate());
  AQ_TRY(enq_diffuse());
  return enq_ink();
}

// The step's last calls in the reference, left commented out there
// (transferToInkParticles + moveInkParticles, Fluid/Fluid_3D_FLIP.cu:349-350):
// the ink moves with the step's velocity (P2G) and newVelocity (after
// extrapolation and diffusion).
aq_status aq_fluid::enq_ink() {
  if (!ink_on || n_ink <= 0) return AQ_OK;
  AQ_CUDA(launch_ink_advance(stream, d, cfg.timestep, ink, u0, v0, w0, nvx(nv_cur), nvy(nv_cur), nvz(nv_cur), n_ink));
  return AQ_OK;
}

// Fluid::initInkRenderer (Fluid/Fluid_3D_FLIP.cu:676-709), which Fluid::init
// would run right after the particle seeding (Fluid/Fluid_3D_FLIP.cu:498):
// spacing h/4 over the initial volumes, continuing the seeding's rand()
// sequence; velocities start at zero.
aq_status aq_fluid::enable_ink() {
  if (ink_on) return AQ_OK;
  if (!rng) return fail(AQ_ERR_INVALID_ARGUMENT, "this fluid has no seeding state");
  Seeder s(cfg, d.h, *rng);
  const float spacing = d.h / 4;
  for (int i = 0; i < cfg.volume_count; ++i) {
    const aq_volume& v = cfg.volumes[i];
    if (v.shape == AQ_SHAPE_SQUARE) s.square_ink(v, spacing);
    else if (v.shape == AQ_SHAPE_SPHERE) s.sphere_ink(v, spacing);
  }
  const size_t N = s.phase.size();
  if (N > (size_t)INT32_MAX) return fail(AQ_ERR_INVALID_CONFIG, "too many ink particles");
  AQ_TRY(alloc(&ink.px, N)); AQ_TRY(alloc(&ink.py, N)); AQ_TRY(alloc(&ink.pz, N));
  AQ_TRY(alloc(&ink.vx, N)); AQ_TRY(alloc(&ink.vy, N)); AQ_TRY(alloc(&ink.vz, N));
  ink.frac = nullptr;
  std::vector<float> comp(N);
  float* dst[3] = {ink.px, ink.py, ink.pz};
  for (int k = 0; k < 3; ++k) {
    for (size_t i = 0; i < N; ++i) comp[i] = s.pos[3 * i + k];
    AQ_CUDA(cudaMemcpyAsync(dst[k], comp.data(), sizeof(float) * N, cudaMemcpyHostToDevice, stream));
    AQ_CUDA(cudaStreamSynchronize(stream));
  }
  n_ink = (int)N;
  ink_on = true;
  invalidate_graph();
  return AQ_OK;
}

static aq_status leaves_of(cudaGraph_t g, std::vector<cudaGraphNode_t>& out) {
  size_t nn = 0;
  AQ_CUDA(cudaGraphGetNodes(g, nullptr, &nn));
  std::vector<cudaGraphNode_t> nodes(nn);
  AQ_CUDA(cudaGraphGetNodes(g, nodes.data(), &nn));
  out.clear();
  for (cudaGraphNode_t nd : nodes) {
    size_t k = 0;
    AQ_CUDA(cudaGraphNodeGetDependentNodes(nd, nullptr, &k));
    if (k == 0) out.push_back(nd);
  }
  return AQ_OK;
}

// The whole step as one CUDA graph.  RESIDUAL mode puts the sweeps in a
// conditional WHILE node whose body ends with the residual check that sets
// the loop condition, so a step needs no host round trip.
aq_status aq_fluid::build_graph() {
  invalidate_graph();
  cudaGraph_t g = nullptr;
  AQ_CUDA(cudaGraphCreate(&g, 0));
  int launches = 0;
  auto capture = [&](cudaGraph_t into, const cudaGraphNode_t* deps, size_t nd, auto&& body) -> aq_status {
    AQ_CUDA(cudaStreamBeginCaptureToGraph(stream, into, deps, nullptr, nd, cudaStreamCaptureModeThreadLocal));
    aq_status st = body();
    cudaGraph_t got = nullptr;
    cudaError_t e = cudaStreamEndCapture(stream, &got);
    if (st != AQ_OK) return st;
    if (e != cudaSuccess) return fail(AQ_ERR_CUDA, std::string("capture: ") + cudaGetErrorString(e));
    return AQ_OK;
  };
  aq_status st = AQ_OK;
  launches += (n > 0 ? 6 : 3) + 2 + 2;  // particles (+3 scan kernels), p2g, slayer, divergence, b2
  if (cfg.solve_mode == AQ_SOLVE_RESIDUAL && (plan.by == 1 || plan.by == 4)) {
    st = capture(g, nullptr, 0, [&]() {
      aq_status s2 = enq_pre_solve();
      if (s2 != AQ_OK) return s2;
      s2 = plan.by == 1 ? enqueue_persistent(this, 0) : enqueue_resident(this, 0);
      if (s2 != AQ_OK) return s2;
      return enq_post_solve();
    });
    launches += 2;
    body_launches = 0;
  } else if (cfg.solve_mode == AQ_SOLVE_RESIDUAL) {
    st = capture(g, nullptr, 0, [&]() { return enq_pre_solve(); });
    if (st != AQ_OK) { cudaGraphDestroy(g); return st; }
    std::vector<cudaGraphNode_t> leaves;
    st = leaves_of(g, leaves);
    if (st != AQ_OK) { cudaGraphDestroy(g); return st; }
    cudaGraphConditionalHandle handle;
    cudaError_t e = cudaGraphConditionalHandleCreate(&handle, g, 1, cudaGraphCondAssignDefault);
    if (e != cudaSuccess) { cudaGraphDestroy(g); return fail(AQ_ERR_CUDA, cudaGetErrorString(e)); }
    cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};
    cp.conditional.handle = handle;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t cnode;
    e = cudaGraphAddNode(&cnode, g, leaves.data(), leaves.size(), &cp);
    if (e != cudaSuccess) {
      cudaGraphDestroy(g);
      return fail(AQ_ERR_CUDA, std::string("conditional node: ") + cudaGetErrorString(e));
    }
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    int bl = 0;
    st = capture(body, nullptr, 0, [&]() { return enq_solve_body(true, (unsigned long long)handle, &bl); });
    if (st != AQ_OK) { cudaGraphDestroy(g); return st; }
    body_launches = bl;
    st = capture(g, &cnode, 1, [&]() { return enq_post_solve(); });
  } else {
    st = capture(g, nullptr, 0, [&]() {
      aq_status s2 = enq_pre_solve();
      if (s2 != AQ_OK) return s2;
      s2 = enq_solve_fixed(cfg.pressure_iterations - solve_sweeps_done());
      if (s2 != AQ_OK) return s2;
      return enq_post_solve();
    });
    const int rest = cfg.pressure_iterations - solve_sweeps_done();
    launches += rest > 0 ? count_jacobi_launches(rest) : 0;
    body_launches = 0;
  }
  if (st != AQ_OK) { cudaGraphDestroy(g); return st; }
  if (cfg.pressure_init == AQ_PRESSURE_LEARNED)  // network, two 20-sweep starts, pick, copy
    launches += kUNetForwardLaunches +
                2 * (jacobi_launches(plan.by == 4 ? JacobiPlan{1, 3, 1} : plan, kWarmSweeps) - 1) + 2;
  launches += 1 + 3 + (multiphase ? cfg.diffusion_iterations : 0) + (ink_on && n_ink > 0 ? 1 : 0);
  graph_launches = launches;
  cudaError_t e = cudaGraphInstantiate(&exec, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) { exec = nullptr; return fail(AQ_ERR_CUDA, std::string("instantiate: ") + cudaGetErrorString(e)); }
  return AQ_OK;
}

aq_status aq_fluid::step(int nsteps) {
  if (!use_graph) {
    for (int i = 0; i < nsteps; ++i) {
      AQ_TRY(enq_pre_solve());
      if (cfg.solve_mode == AQ_SOLVE_RESIDUAL) AQ_TRY(enq_solve_residual_eager());
      else AQ_TRY(enq_solve_fixed(cfg.pressure_iterations - solve_sweeps_done()));
      AQ_TRY(enq_post_solve());
      time += (double)cfg.timestep;
    }
    nv_cur = has_cur = 2;
    return AQ_OK;
  }
  if (!exec) AQ_TRY(build_graph());
  for (int i = 0; i < nsteps; ++i) {
    AQ_CUDA(cudaGraphLaunch(exec, stream));
    time += (double)cfg.timestep;
  }
  nv_cur = has_cur = 2;
  return AQ_OK;
}

// ------------------------------------------------------------------ init
aq_status aq_fluid::seed_and_init() {
  rng.reset(new aqb::HostRand((unsigned)cfg.seed));
  Seeder s(cfg, d.h, *rng);
  for (int i = 0; i < cfg.volume_count; ++i) {
    const aq_volume& v = cfg.volumes[i];
    if (v.shape == AQ_SHAPE_SQUARE) s.square(v);
    else if (v.shape == AQ_SHAPE_SPHERE) s.sphere(v);
  }
  n = (int)s.phase.size();
  multiphase = false;
  phase = n > 0 ? s.phase[0] : (cfg.volume_count > 0 ? cfg.volumes[0].phase : 0);
  for (int i = 1; i < n; ++i)
    if (s.phase[i] != phase) { multiphase = true; break; }
  sp.multiphase = multiphase ? 1 : 0;
  sp.phase = phase;
  AQ_TRY(allocate());
  if (n > 0) {
    std::vector<float> comp((size_t)n);
    float* dst[3] = {cur.px, cur.py, cur.pz};
    for (int k = 0; k < 3; ++k) {
      for (int i = 0; i < n; ++i) comp[i] = s.pos[3 * (size_t)i + k];
      AQ_CUDA(cudaMemcpyAsync(dst[k], comp.data(), sizeof(float) * n, cudaMemcpyHostToDevice, stream));
      AQ_CUDA(cudaStreamSynchronize(stream));
    }
    std::vector<float4> fr((size_t)n);
    for (int i = 0; i < n; ++i) {
      const int p = s.phase[i];
      fr[i] = make_float4(p == 0, p == 1, p == 2, p == 3);
    }
    AQ_CUDA(cudaMemcpyAsync(cur.frac, fr.data(), sizeof(float4) * n, cudaMemcpyHostToDevice, stream));
    AQ_CUDA(cudaStreamSynchronize(stream));
  }
  // Fluid::init order: fixBoundary (zero velocities stay zero), seeding,
  // transferToGrid (sort + P2G without forces); newVelocity = velocity.
  AQ_TRY(enq_particles(false));
  AQ_TRY(enq_p2g(false));
  AQ_CUDA(cudaMemcpyAsync(un2, un1, sizeof(float) * d.F, cudaMemcpyDeviceToDevice, stream));
  AQ_CUDA(cudaMemcpyAsync(vn2, vn1, sizeof(float) * d.F, cudaMemcpyDeviceToDevice, stream));
  AQ_CUDA(cudaMemcpyAsync(wn2, wn1, sizeof(float) * d.F, cudaMemcpyDeviceToDevice, stream));
  nv_cur = 2;
  has_cur = 2;
  AQ_CUDA(cudaStreamSynchronize(stream));
  return AQ_OK;
}

// ----------------------------------------------------------- state exchange
aq_status aq_fluid::download(aq_host_state* s) {
  if (s->size_x != d.sx || s->size_y != d.sy || s->size_z != d.sz || s->particle_count != n)
    return fail(AQ_ERR_INVALID_ARGUMENT, "state dimensions do not match the fluid");
  AQ_CUDA(cudaStreamSynchronize(stream));
  const size_t N = (size_t)n, C = (size_t)d.C, F = (size_t)d.F;
  s->physical_time = time;
  auto get = [&](void* dst, const void* src, size_t bytes) -> aq_status {
    AQ_CUDA(cudaMemcpy(dst, src, bytes, cudaMemcpyDeviceToHost));
    return AQ_OK;
  };
  if (s->position && N) {
    AQ_TRY(get(s->position, cur.px, 4 * N)); AQ_TRY(get(s->position + N, cur.py, 4 * N));
    AQ_TRY(get(s->position + 2 * N, cur.pz, 4 * N));
  }
  if (s->velocity_p && N) {
    AQ_TRY(get(s->velocity_p, cur.vx, 4 * N)); AQ_TRY(get(s->velocity_p + N, cur.vy, 4 * N));
    AQ_TRY(get(s->velocity_p + 2 * N, cur.vz, 4 * N));
  }
  std::vector<int8_t> ty(C);
  AQ_TRY(get(ty.data(), type, C));
  if (s->fractions && N) {
    if (multiphase) {
      std::vector<float4> fr(N);
      AQ_TRY(get(fr.data(), cur.frac, sizeof(float4) * N));
      for (size_t i = 0; i < N; ++i) {
        s->fractions[i] = fr[i].x; s->fractions[N + i] = fr[i].y;
        s->fractions[2 * N + i] = fr[i].z; s->fractions[3 * N + i] = fr[i].w;
      }
    } else {
      for (int k = 0; k < 4; ++k)
        for (size_t i = 0; i < N; ++i) s->fractions[k * N + i] = k == phase ? 1.f : 0.f;
    }
  }
  if (s->content) {
    for (int x = 0; x <= d.sx; ++x)
      for (int y = 0; y <= d.sy; ++y)
        for (int z = 0; z <= d.sz; ++z) {
          int v;
          if (x < d.sx && y < d.sy && z < d.sz) v = ty[cell_index(d, x, y, z)];
          else
            v = ((x == d.sx && covered_x(d, y, z)) || (y == d.sy && covered_y(d, x, z)) ||
                 (z == d.sz && covered_z(d, x, y))) ? kSolid : kAir;
          s->content[node_index(d, x, y, z)] = v;
        }
  }
  if (s->velocity) {
    AQ_TRY(get(s->velocity, u0, 4 * F)); AQ_TRY(get(s->velocity + F, v0, 4 * F));
    AQ_TRY(get(s->velocity + 2 * F, w0, 4 * F));
  }
  if (s->new_velocity) {
    AQ_TRY(get(s->new_velocity, nvx(nv_cur), 4 * F)); AQ_TRY(get(s->new_velocity + F, nvy(nv_cur), 4 * F));
    AQ_TRY(get(s->new_velocity + 2 * F, nvz(nv_cur), 4 * F));
  }
  if (s->pressure) AQ_TRY(get(s->pressure, pa, 4 * C));
  if (s->divergence) AQ_TRY(get(s->divergence, div, 4 * C));
  if (s->particle_count_cell) AQ_TRY(get(s->particle_count_cell, pcount, 4 * C));
  if (s->density) AQ_TRY(get(s->density, density, 4 * C));
  if (s->has_velocity) {
    std::vector<uint8_t> hbits(F);
    AQ_TRY(get(hbits.data(), hb(has_cur), F));
    for (int x = 0; x < d.sx; ++x)
      for (int y = 0; y < d.sy; ++y)
        for (int z = 0; z < d.sz; ++z) {
          const uint8_t b = hbits[node_index(d, x, y, z)];
          const size_t c = cell_index(d, x, y, z);
          for (int k = 0; k < 3; ++k) s->has_velocity[k * C + c] = (b >> k) & 1;
        }
  }
  if (s->volume_fractions || s->new_volume_fractions) {
    if (multiphase) {
      std::vector<float4> a(C);
      if (s->volume_fractions) {
        AQ_TRY(get(a.data(), vf, sizeof(float4) * C));
        for (size_t c = 0; c < C; ++c) {
          s->volume_fractions[c] = a[c].x; s->volume_fractions[C + c] = a[c].y;
          s->volume_fractions[2 * C + c] = a[c].z; s->volume_fractions[3 * C + c] = a[c].w;
        }
      }
      if (s->new_volume_fractions) {
        AQ_TRY(get(a.data(), nvf, sizeof(float4) * C));
        for (size_t c = 0; c < C; ++c) {
          s->new_volume_fractions[c] = a[c].x; s->new_volume_fractions[C + c] = a[c].y;
          s->new_volume_fractions[2 * C + c] = a[c].z; s->new_volume_fractions[3 * C + c] = a[c].w;
        }
      }
    } else {
      for (int k = 0; k < 4; ++k)
        for (size_t c = 0; c < C; ++c) {
          const float v = (ty[c] == kFluid && k == phase) ? 1.f : 0.f;
          if (s->volume_fractions) s->volume_fractions[k * C + c] = v;
          if (s->new_volume_fractions) s->new_volume_fractions[k * C + c] = v;
        }
    }
  }
  if (s->cell_start || s->cell_end || s->particle_hash) {
    std::vector<int> o(C + 1);
    AQ_TRY(get(o.data(), off, 4 * (C + 1)));
    for (size_t c = 0; c <= C; ++c) o[c] -= index_base;
    for (size_t c = 0; c < C; ++c) {
      const bool occ = o[c + 1] > o[c];
      if (s->cell_start) s->cell_start[c] = occ ? o[c] : -1;
      if (s->cell_end) s->cell_end[c] = occ ? o[c + 1] - 1 : -1;
      if (s->particle_hash)
        for (int k = o[c]; k < o[c + 1]; ++k) s->particle_hash[k] = (int)c;
    }
  }
  if (s->sort_index && N) {
    AQ_TRY(get(s->sort_index, sort_index, 4 * N));
    if (index_base)
      for (size_t i = 0; i < N; ++i) s->sort_index[i] -= index_base;
  }
  return AQ_OK;
}

// rhs, air pressure, active bricks and ||b||^2 from an injected state, as the
// divergence stage would have left them.
aq_status aq_fluid::derive_from_state(const std::vector<int>& content, const std::vector<float>& divv,
                                      const std::vector<float>& dens) {
  const size_t C = (size_t)d.C;
  std::vector<int8_t> ty(C);
  std::vector<float> r(C);
  std::vector<uint8_t> act((size_t)nbricks, 0);
  double b2 = 0.0;
  int nf = 0;
  for (int x = 0; x < d.sx; ++x)
    for (int y = 0; y < d.sy; ++y)
      for (int z = 0; z < d.sz; ++z) {
        const int c = cell_index(d, x, y, z);
        const bool fl = content[node_index(d, x, y, z)] == kFluid;
        ty[c] = fl ? kFluid : kAir;
        r[c] = fl ? (-divv[c]) * dens[c] : 0.f;
        if (fl) {
          b2 += (double)r[c] * (double)r[c];
          nf++;
          act[brick_index(d, x, y, z)] = 1;
        }
      }
  AQ_CUDA(cudaMemcpy(type, ty.data(), C, cudaMemcpyHostToDevice));
  AQ_CUDA(cudaMemcpy(rhs, r.data(), 4 * C, cudaMemcpyHostToDevice));
  // air pressure is 0 before any sweep (the divergence stage clears it)
  std::vector<float> p(C);
  for (float* buf : {pa, pb}) {
    AQ_CUDA(cudaMemcpy(p.data(), buf, 4 * C, cudaMemcpyDeviceToHost));
    for (size_t c = 0; c < C; ++c)
      if (ty[c] != kFluid) p[c] = 0.f;
    AQ_CUDA(cudaMemcpy(buf, p.data(), 4 * C, cudaMemcpyHostToDevice));
  }
  AQ_CUDA(cudaMemcpy(bact, act.data(), (size_t)nbricks, cudaMemcpyHostToDevice));
  SolveState s0;
  memset(&s0, 0, sizeof(s0));
  s0.b2 = b2;
  s0.fluid_cells = nf;
  s0.rel_residual = -1.0;
  s0.r2 = -1.0;
  AQ_CUDA(cudaMemcpy(ss, &s0, sizeof(s0), cudaMemcpyHostToDevice));
  return AQ_OK;
}

aq_status aq_fluid::upload(const aq_host_state* s) {
  if (s->size_x != d.sx || s->size_y != d.sy || s->size_z != d.sz || s->particle_count != n)
    return fail(AQ_ERR_INVALID_ARGUMENT, "state dimensions do not match the fluid");
  AQ_CUDA(cudaStreamSynchronize(stream));
  // a new state: the sticky health flags start over
  AQ_CUDA(cudaMemsetAsync(&ss->nonfinite_seen, 0, sizeof(int), stream));
  AQ_CUDA(cudaMemsetAsync(&ss->sync_timeout, 0, sizeof(int), stream));
  const size_t N = (size_t)n, C = (size_t)d.C, F = (size_t)d.F;
  if (s->position) {
    const float lim[3] = {d.sx * d.h, d.sy * d.h, d.sz * d.h};
    for (int k = 0; k < 3; ++k)
      for (size_t i = 0; i < N; ++i) {
        const float p = s->position[k * N + i];
        if (!(p >= 0.f && p <= lim[k])) return fail(AQ_ERR_INVALID_ARGUMENT, "particle position outside the domain");
      }
  }
  auto put = [&](void* dst, const void* src, size_t bytes) -> aq_status {
    AQ_CUDA(cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice));
    return AQ_OK;
  };
  time = s->physical_time;
  if (s->position && N) {
    AQ_TRY(put(cur.px, s->position, 4 * N)); AQ_TRY(put(cur.py, s->position + N, 4 * N));
    AQ_TRY(put(cur.pz, s->position + 2 * N, 4 * N));
  }
  if (s->velocity_p && N) {
    AQ_TRY(put(cur.vx, s->velocity_p, 4 * N)); AQ_TRY(put(cur.vy, s->velocity_p + N, 4 * N));
    AQ_TRY(put(cur.vz, s->velocity_p + 2 * N, 4 * N));
  }
  bool mode_changed = false;
  if (s->fractions && N) {
    std::vector<float4> fr(N);
    int ph = -1;
    bool multi = false;
    for (size_t i = 0; i < N; ++i) {
      fr[i] = make_float4(s->fractions[i], s->fractions[N + i], s->fractions[2 * N + i], s->fractions[3 * N + i]);
      const float e[4] = {fr[i].x, fr[i].y, fr[i].z, fr[i].w};
      int hot = -1, nz = 0;
      for (int k = 0; k < 4; ++k)
        if (e[k] != 0.f) { nz++; hot = k; }
      if (nz != 1 || e[hot] != 1.f) multi = true;
      else if (ph < 0) ph = hot;
      else if (ph != hot) multi = true;
    }
    if (!multi && ph >= 0) {
      if (multiphase || phase != ph) mode_changed = true;
      multiphase = false;
      phase = ph;
    } else if (multi) {
      if (!multiphase) mode_changed = true;
      multiphase = true;
    }
    AQ_TRY(put(cur.frac, fr.data(), sizeof(float4) * N));
    sp.multiphase = multiphase ? 1 : 0;
    sp.phase = phase;
  }
  std::vector<int> content;
  if (s->content) content.assign(s->content, s->content + F);
  if (s->velocity) {
    AQ_TRY(put(u0, s->velocity, 4 * F)); AQ_TRY(put(v0, s->velocity + F, 4 * F));
    AQ_TRY(put(w0, s->velocity + 2 * F, 4 * F));
  }
  if (s->new_velocity) {
    for (int which = 1; which <= 2; ++which) {
      AQ_TRY(put(nvx(which), s->new_velocity, 4 * F)); AQ_TRY(put(nvy(which), s->new_velocity + F, 4 * F));
      AQ_TRY(put(nvz(which), s->new_velocity + 2 * F, 4 * F));
    }
  }
  if (s->pressure) {
    AQ_TRY(put(pa, s->pressure, 4 * C));
    AQ_TRY(put(pb, s->pressure, 4 * C));
  }
  if (s->divergence) AQ_TRY(put(div, s->divergence, 4 * C));
  if (s->particle_count_cell) AQ_TRY(put(pcount, s->particle_count_cell, 4 * C));
  if (s->density) AQ_TRY(put(density, s->density, 4 * C));
  if (s->has_velocity) {
    std::vector<uint8_t> hbits(F, 0);
    for (int x = 0; x < d.sx; ++x)
      for (int y = 0; y < d.sy; ++y)
        for (int z = 0; z < d.sz; ++z) {
          const size_t c = cell_index(d, x, y, z);
          uint8_t b = 0;
          for (int k = 0; k < 3; ++k) b |= (s->has_velocity[k * C + c] ? 1 : 0) << k;
          hbits[node_index(d, x, y, z)] = b;
        }
    AQ_TRY(put(h1, hbits.data(), F));
    AQ_TRY(put(h2, hbits.data(), F));
  }
  if (s->volume_fractions || s->new_volume_fractions) {
    std::vector<float4> a(C);
    if (s->volume_fractions) {
      for (size_t c = 0; c < C; ++c)
        a[c] = make_float4(s->volume_fractions[c], s->volume_fractions[C + c], s->volume_fractions[2 * C + c],
                           s->volume_fractions[3 * C + c]);
      AQ_TRY(put(vf, a.data(), sizeof(float4) * C));
    }
    if (s->new_volume_fractions) {
      for (size_t c = 0; c < C; ++c)
        a[c] = make_float4(s->new_volume_fractions[c], s->new_volume_fractions[C + c],
                           s->new_volume_fractions[2 * C + c], s->new_volume_fractions[3 * C + c]);
      AQ_TRY(put(nvf, a.data(), sizeof(float4) * C));
    }
  }
  if (s->cell_start && s->cell_end) {
    std::vector<int> o(C + 1);
    int run = 0;
    for (size_t c = 0; c < C; ++c) {
      o[c] = run;
      if (s->cell_start[c] >= 0) {
        if (s->cell_start[c] != run || s->cell_end[c] < s->cell_start[c])
          return fail(AQ_ERR_INVALID_ARGUMENT, "cell tables are not a sorted partition of the particles");
        run = s->cell_end[c] + 1;
      }
    }
    if (run != n) return fail(AQ_ERR_INVALID_ARGUMENT, "cell tables do not cover every particle");
    o[C] = run;
    AQ_TRY(put(off, o.data(), 4 * (C + 1)));
  }
  if (s->sort_index && N) AQ_TRY(put(sort_index, s->sort_index, 4 * N));
  // derived solver inputs
  if (s->content || s->divergence || s->density) {
    std::vector<int> ct = content;
    if (ct.empty()) {
      aq_host_state q;
      memset(&q, 0, sizeof(q));
      q.size_x = d.sx; q.size_y = d.sy; q.size_z = d.sz; q.particle_count = n;
      ct.resize(F);
      q.content = ct.data();
      AQ_TRY(download(&q));
    }
    std::vector<float> dv(C), dn(C);
    AQ_CUDA(cudaMemcpy(dv.data(), div, 4 * C, cudaMemcpyDeviceToHost));
    AQ_CUDA(cudaMemcpy(dn.data(), density, 4 * C, cudaMemcpyDeviceToHost));
    AQ_TRY(derive_from_state(ct, dv, dn));
    AQ_TRY(enq_row_items());
  }
  nv_cur = has_cur = 2;
  sorted_by_stage1 = false;
  if (mode_changed) invalidate_graph();
  return AQ_OK;
}

// ====================================================================== ABI
namespace {

aq_status validate(const aq_config* c) {
  if (!c) return fail(AQ_ERR_INVALID_ARGUMENT, "config is NULL");
  if (c->size_x < 4 || c->size_y < 4 || c->size_z < 4)
    return fail(AQ_ERR_INVALID_CONFIG, "grid sizes must be >= 4 per axis");
  if ((double)(c->size_x + 1) * (c->size_y + 1) * (c->size_z + 1) > 1.5e9)
    return fail(AQ_ERR_INVALID_CONFIG, "grid too large");
  if (c->phase_count > AQ_MAX_PHASES) return fail(AQ_ERR_INVALID_CONFIG, "Only supports up to 4 phases");
  if (c->volume_count < 0 || c->volume_count > AQ_MAX_VOLUMES)
    return fail(AQ_ERR_INVALID_CONFIG, "volume_count out of range");
  for (int i = 0; i < c->volume_count; ++i) {
    const aq_volume& v = c->volumes[i];
    if (v.shape != AQ_SHAPE_SPHERE && v.shape != AQ_SHAPE_SQUARE)
      return fail(AQ_ERR_INVALID_CONFIG, "unknown volume shape");
    if (v.phase < 0 || v.phase >= AQ_MAX_PHASES)
      return fail(AQ_ERR_INVALID_CONFIG, "volume phase must be in [0,4)");
  }
  if (!(c->domain_size > 0.f) || !std::isfinite(c->domain_size))
    return fail(AQ_ERR_INVALID_CONFIG, "domain_size must be positive");
  if (!std::isfinite(c->timestep) || c->timestep < 0.f) return fail(AQ_ERR_INVALID_CONFIG, "timestep must be >= 0");
  if (c->pressure_iterations < 0 || c->diffusion_iterations < 0)
    return fail(AQ_ERR_INVALID_CONFIG, "iteration counts must be >= 0");
  if (c->pressure_init != AQ_PRESSURE_CARRY && c->pressure_init != AQ_PRESSURE_ZERO &&
      c->pressure_init != AQ_PRESSURE_LEARNED)
    return fail(AQ_ERR_INVALID_CONFIG, "unknown pressure_init");
  if (c->pressure_init == AQ_PRESSURE_LEARNED) {
    if (c->size_x % 4 || c->size_y % 4 || c->size_z % 4)
      return fail(AQ_ERR_INVALID_CONFIG, "the learned warm start needs grid sizes divisible by 4");
    if (c->solve_mode == AQ_SOLVE_FIXED && c->pressure_iterations < kWarmSweeps)
      return fail(AQ_ERR_INVALID_CONFIG, "the learned warm start needs pressure_iterations >= 20");
  }
  if (c->solve_mode != AQ_SOLVE_FIXED && c->solve_mode != AQ_SOLVE_RESIDUAL)
    return fail(AQ_ERR_INVALID_CONFIG, "unknown solve_mode");
  if (c->solve_mode == AQ_SOLVE_RESIDUAL) {
    if (!(c->rel_residual > 0.f)) return fail(AQ_ERR_INVALID_CONFIG, "rel_residual must be > 0");
    if (c->check_interval < 1 || c->max_iterations < c->check_interval)
      return fail(AQ_ERR_INVALID_CONFIG, "need 1 <= check_interval <= max_iterations");
  }
  for (int k = 0; k < 3; ++k)
    if (!std::isfinite(c->gravity[k])) return fail(AQ_ERR_INVALID_CONFIG, "gravity must be finite");
  return AQ_OK;
}

}  // namespace

extern "C" {

int32_t aq_abi_version(void) { return AQ_ABI_VERSION; }

const char* aq_last_error(void) { return g_last_error.c_str(); }

aq_status aq_config_default(aq_config* c) {
  if (!c) return fail(AQ_ERR_INVALID_ARGUMENT, "config is NULL");
  memset(c, 0, sizeof(*c));
  c->volume_count = 2;
  c->volumes[0].shape = AQ_SHAPE_SQUARE;
  c->volumes[1].shape = AQ_SHAPE_SPHERE;
  for (int i = 0; i < 2; ++i) {
    aq_volume& v = c->volumes[i];
    v.box_min[0] = 0; v.box_min[1] = 0; v.box_min[2] = 0;
    v.box_max[0] = 1; v.box_max[1] = 0.1875f; v.box_max[2] = 1;
    v.ball_center[0] = 0.5f; v.ball_center[1] = 0.75f; v.ball_center[2] = 0.5f;
    v.ball_radius = 0.125f;
    v.phase = 0;
  }
  c->gravity[1] = -9.8f;
  c->phase_count = 2;
  for (int i = 0; i < 4; ++i) c->phase_densities[i] = 1.f;
  c->diffusion_coeff = 0.001f;
  c->size_x = c->size_y = c->size_z = 50;
  c->pressure_iterations = 100;
  c->diffusion_iterations = 100;
  c->timestep = 0.033f;
  c->flip_coeff = 0.95f;
  c->particle_jitter = 0.05f;
  c->domain_size = 10.f;
  c->seed = 1;
  c->pressure_init = AQ_PRESSURE_CARRY;
  c->solve_mode = AQ_SOLVE_FIXED;
  c->rel_residual = 1e-4f;
  c->max_iterations = 2000;
  c->check_interval = 40;
  c->device = 0;
  c->stream = nullptr;
  g_last_error.clear();
  return AQ_OK;
}

aq_status aq_config_validate(const aq_config* cfg) {
  aq_status st = validate(cfg);
  if (st == AQ_OK) g_last_error.clear();
  return st;
}

aq_status aq_fluid_create(const aq_config* cfg, aq_fluid** out) {
  if (!out) return fail(AQ_ERR_INVALID_ARGUMENT, "out is NULL");
  *out = nullptr;
  AQ_TRY(validate(cfg));
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return fail(AQ_ERR_NO_DEVICE, "no CUDA device");
  }
  if (cfg->device < 0 || cfg->device >= ndev) return fail(AQ_ERR_INVALID_CONFIG, "device ordinal out of range");
  aq_fluid* f = new aq_fluid();
  f->cfg = *cfg;
  f->device = cfg->device;
  cudaError_t e = cudaSetDevice(f->device);
  if (e != cudaSuccess) { delete f; return fail(AQ_ERR_CUDA, cudaGetErrorString(e)); }
  if (cfg->stream) {
    f->stream = (cudaStream_t)cfg->stream;
  } else {
    e = cudaStreamCreateWithFlags(&f->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) { delete f; return fail(AQ_ERR_CUDA, cudaGetErrorString(e)); }
    f->own_stream = true;
  }
  e = cudaStreamCreateWithFlags(&f->side, cudaStreamNonBlocking);
  if (e != cudaSuccess) { delete f; return fail(AQ_ERR_CUDA, cudaGetErrorString(e)); }
  Dims& d = f->d;
  d.sx = cfg->size_x; d.sy = cfg->size_y; d.sz = cfg->size_z;
  d.C = d.sx * d.sy * d.sz;
  d.F = (d.sx + 1) * (d.sy + 1) * (d.sz + 1);
  d.nz = d.sz + 1;
  d.nyz = (d.sy + 1) * (d.sz + 1);
  d.h = cfg->domain_size / (float)d.sy;  // cellPhysicalSize (Fluid/Fluid_3D_FLIP.cu:444)
  d.inv_h = 1.0f / d.h;
  d.bx = (d.sx + kBrick - 1) / kBrick; d.by = (d.sy + kBrick - 1) / kBrick; d.bz = (d.sz + kBrick - 1) / kBrick;
  d.cov_x = covered_faces(d.sy, d.sz);
  d.cov_y = covered_faces(d.sx, d.sz);
  d.cov_z = covered_faces(d.sx, d.sy);
  StepParams& sp = f->sp;
  sp.dt = cfg->timestep;
  sp.flip = cfg->flip_coeff;
  sp.gdx = cfg->gravity[0] * cfg->timestep;
  sp.gdy = cfg->gravity[1] * cfg->timestep;
  sp.gdz = cfg->gravity[2] * cfg->timestep;
  sp.gx_nz = cfg->gravity[0] != 0.f; sp.gy_nz = cfg->gravity[1] != 0.f; sp.gz_nz = cfg->gravity[2] != 0.f;
  for (int k = 0; k < 4; ++k) sp.rho[k] = cfg->phase_densities[k];
  e = jacobi_prepare();
  if (e != cudaSuccess) { delete f; return fail(AQ_ERR_CUDA, std::string("jacobi_prepare: ") + cudaGetErrorString(e)); }
  aq_status st = f->seed_and_init();
  if (st != AQ_OK) { delete f; return st; }
  *out = f;
  g_last_error.clear();
  return AQ_OK;
}

void aq_fluid_destroy(aq_fluid* f) { delete f; }

aq_status aq_fluid_step(aq_fluid* f, int32_t n_steps) {
  if (!f || n_steps < 0) return fail(AQ_ERR_INVALID_ARGUMENT, "bad argument");
  cudaSetDevice(f->device);
  return f->step(n_steps);
}

aq_status aq_fluid_step_host(aq_fluid* f, int32_t n_steps, const float* pin, const float* vin, float* pout,
                             float* vout) {
  if (!f || n_steps < 0) return fail(AQ_ERR_INVALID_ARGUMENT, "bad argument");
  cudaSetDevice(f->device);
  const size_t N = (size_t)f->n;
  cudaStream_t s = f->stream;
  if (N) {
    if (pin) {
      AQ_CUDA(cudaMemcpyAsync(f->cur.px, pin, 4 * N, cudaMemcpyHostToDevice, s));
      AQ_CUDA(cudaMemcpyAsync(f->cur.py, pin + N, 4 * N, cudaMemcpyHostToDevice, s));
      AQ_CUDA(cudaMemcpyAsync(f->cur.pz, pin + 2 * N, 4 * N, cudaMemcpyHostToDevice, s));
    }
    if (vin) {
      AQ_CUDA(cudaMemcpyAsync(f->cur.vx, vin, 4 * N, cudaMemcpyHostToDevice, s));
      AQ_CUDA(cudaMemcpyAsync(f->cur.vy, vin + N, 4 * N, cudaMemcpyHostToDevice, s));
      AQ_CUDA(cudaMemcpyAsync(f->cur.vz, vin + 2 * N, 4 * N, cudaMemcpyHostToDevice, s));
    }
  }
  AQ_TRY(f->step(n_steps));
  if (N) {
    if (pout) {
      AQ_CUDA(cudaMemcpyAsync(pout, f->cur.px, 4 * N, cudaMemcpyDeviceToHost, s));
      AQ_CUDA(cudaMemcpyAsync(pout + N, f->cur.py, 4 * N, cudaMemcpyDeviceToHost, s));
      AQ_CUDA(cudaMemcpyAsync(pout + 2 * N, f->cur.pz, 4 * N, cudaMemcpyDeviceToHost, s));
    }
    if (vout) {
      AQ_CUDA(cudaMemcpyAsync(vout, f->cur.vx, 4 * N, cudaMemcpyDeviceToHost, s));
      AQ_CUDA(cudaMemcpyAsync(vout + N, f->cur.vy, 4 * N, cudaMemcpyDeviceToHost, s));
      AQ_CUDA(cudaMemcpyAsync(vout + 2 * N, f->cur.vz, 4 * N, cudaMemcpyDeviceToHost, s));
    }
  }
  return f->health();
}

aq_status aq_fluid_set_graph_mode(aq_fluid* f, int32_t use_graph) {
  if (!f) return fail(AQ_ERR_INVALID_ARGUMENT, "fluid is NULL");
  f->use_graph = use_graph != 0;
  return AQ_OK;
}

aq_status aq_fluid_run_stage(aq_fluid* f, int32_t stage) {
  if (!f) return fail(AQ_ERR_INVALID_ARGUMENT, "fluid is NULL");
  cudaSetDevice(f->device);
  return f->run_stage(stage);
}

aq_status aq_fluid_synchronize(aq_fluid* f) {
  if (!f) return fail(AQ_ERR_INVALID_ARGUMENT, "fluid is NULL");
  cudaSetDevice(f->device);
  return f->health();
}

// Waits for the fluid's work, then reports what the device recorded: a
// bounded wait that gave up (AQ_ERR_TIMEOUT), or a non-finite divergence
// norm or pressure residual in any step since creation or the last upload
// (AQ_ERR_NONFINITE).  The reference has no such check: a NaN there simply
// propagates (Common/GpuCommons.h:118-142 only catches CUDA errors).
aq_status aq_fluid::health() {
  AQ_CUDA(cudaMemcpyAsync(ss_host, ss, sizeof(SolveState), cudaMemcpyDeviceToHost, stream));
  AQ_CUDA(cudaStreamSynchronize(stream));
  const SolveState& s = *ss_host;
  if (s.sync_timeout) return fail(AQ_ERR_TIMEOUT, "a persistent pressure solve gave up waiting at a grid barrier");
  if (s.nonfinite_seen) return fail(AQ_ERR_NONFINITE, "a step produced a non-finite divergence norm or pressure residual");
  return AQ_OK;
}

aq_status aq_p2g_set_variant(int32_t variant) {
  if (variant < 0 || variant > 3) return fail(AQ_ERR_INVALID_ARGUMENT, "P2G variant must be 0-3");
  set_p2g_variant(variant);
  return AQ_OK;
}

aq_status aq_selfcheck_division(int32_t device, uint64_t* mismatches) {
  if (!mismatches) return fail(AQ_ERR_INVALID_ARGUMENT, "bad argument");
  AQ_CUDA(cudaSetDevice(device));
  unsigned long long* bad = nullptr;
  AQ_CUDA(cudaMalloc(&bad, sizeof(unsigned long long)));
  cudaError_t e = cudaMemset(bad, 0, sizeof(unsigned long long));
  if (e == cudaSuccess) e = launch_div6_check(nullptr, bad);
  unsigned long long h = 0;
  if (e == cudaSuccess) e = cudaMemcpy(&h, bad, sizeof(h), cudaMemcpyDeviceToHost);
  cudaFree(bad);
  if (e != cudaSuccess) return fail(AQ_ERR_CUDA, cudaGetErrorString(e));
  *mismatches = h;
  return AQ_OK;
}

aq_status aq_fluid_test_barrier_timeout(aq_fluid* f, int32_t withhold_cta, uint32_t spin_limit) {
  if (!f) return fail(AQ_ERR_INVALID_ARGUMENT, "fluid is NULL");
  f->barrier_test.withhold_cta = withhold_cta;
  f->barrier_test.spin_limit = spin_limit;
  f->invalidate_graph();  // the step graph holds the solve's launch parameters
  return AQ_OK;
}

aq_status aq_fluid_time(const aq_fluid* f, double* t) {
  if (!f || !t) return fail(AQ_ERR_INVALID_ARGUMENT, "bad argument");
  *t = f->time;
  return AQ_OK;
}

aq_status aq_fluid_particle_count(const aq_fluid* f, int32_t* n) {
  if (!f || !n) return fail(AQ_ERR_INVALID_ARGUMENT, "bad argument");
  *n = f->n;
  return AQ_OK;
}

aq_status aq_fluid_container(const aq_fluid* f, float center[3], float* size) {
  if (!f) return fail(AQ_ERR_INVALID_ARGUMENT, "fluid is NULL");
  // Fluid::getCenter / getContainerSize (Fluid/Fluid_3D_FLIP.cu:728-733)
  const float g = f->cfg.domain_size;
  if (center) center[0] = center[1] = center[2] = g / 2;
  if (size) *size = g;
  return AQ_OK;
}

aq_status aq_fluid_stream(const aq_fluid* f, void** stream) {
  if (!f || !stream) return fail(AQ_ERR_INVALID_ARGUMENT, "bad argument");
  *stream = (void*)f->stream;
  return AQ_OK;
}

aq_status aq_fluid_download_state(aq_fluid* f, aq_host_state* s) {
  if (!f || !s) return fail(AQ_ERR_INVALID_ARGUMENT, "bad argument");
  cudaSetDevice(f->device);
  return f->download(s);
}

aq_status aq_fluid_upload_state(aq_fluid* f, const aq_host_state* s) {
  if (!f || !s) return fail(AQ_ERR_INVALID_ARGUMENT, "bad argument");
  cudaSetDevice(f->device);
  return f->upload(s);
}

aq_status aq_fluid_solve_stats(const aq_fluid* f, aq_solve_stats* st) {
  if (!f || !st) return fail(AQ_ERR_INVALID_ARGUMENT, "bad argument");
  cudaSetDevice(f->device);
  SolveState s;
  AQ_CUDA(cudaMemcpyAsync(f->ss_host, f->ss, sizeof(SolveState), cudaMemcpyDeviceToHost, f->stream));
  AQ_CUDA(cudaStreamSynchronize(f->stream));
  s = *f->ss_host;
  st->iterations = s.iterations;
  st->rel_residual = s.rel_residual;
  st->b_norm = s.b2 >= 0 ? sqrt(s.b2) : -1.0;
  st->fluid_cells = s.fluid_cells;
  st->converged = s.converged;
  st->blocks = s.bodies;
  st->total_sweeps = s.total_sweeps;
  st->total_blocks = s.total_bodies;
  st->warm_start = s.warm;
  st->warm_rel_residual = s.warm_rel;
  st->zero_rel_residual = s.zero_rel;
  if (s.sync_timeout) return fail(AQ_ERR_TIMEOUT, "persistent pressure solve timed out at a grid barrier");
  if (s.nonfinite) return fail(AQ_ERR_NONFINITE, "the last pressure solve's residual is not finite");
  if (f->cfg.solve_mode == AQ_SOLVE_RESIDUAL && !s.converged && s.rel_residual >= 0.0)
    return fail(AQ_ERR_NOT_CONVERGED, "the last pressure solve stopped at max_iterations above rel_residual");
  return AQ_OK;
}

aq_status aq_fluid_phase_mass(aq_fluid* f, double mass[4]) {
  if (!f || !mass) return fail(AQ_ERR_INVALID_ARGUMENT, "bad argument");
  cudaSetDevice(f->device);
  for (int k = 0; k < 4; ++k) mass[k] = 0.0;
  if (!f->multiphase) {
    mass[f->phase] = (double)f->n;
    return AQ_OK;
  }
  const int np = frac_sum_parts();
  double* part = nullptr;
  AQ_CUDA(cudaMallocAsync((void**)&part, sizeof(double) * 4 * np, f->stream));
  cudaError_t e = launch_frac_sum(f->stream, f->cur.frac, f->n, part);
  std::vector<double> h((size_t)4 * np);
  if (e == cudaSuccess) e = cudaMemcpyAsync(h.data(), part, sizeof(double) * 4 * np, cudaMemcpyDeviceToHost, f->stream);
  cudaFreeAsync(part, f->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(f->stream);
  AQ_CUDA(e);
  for (int b = 0; b < np; ++b)
    for (int k = 0; k < 4; ++k) mass[k] += h[(size_t)b * 4 + k];
  return AQ_OK;
}

aq_status aq_fluid_enable_ink(aq_fluid* f, int32_t* count) {
  if (!f) return fail(AQ_ERR_INVALID_ARGUMENT, "fluid is NULL");
  cudaSetDevice(f->device);
  AQ_CUDA(cudaStreamSynchronize(f->stream));
  AQ_TRY(f->enable_ink());
  if (count) *count = f->n_ink;
  return AQ_OK;
}

aq_status aq_fluid_ink_count(const aq_fluid* f, int32_t* count) {
  if (!f || !count) return fail(AQ_ERR_INVALID_ARGUMENT, "bad argument");
  *count = f->ink_on ? f->n_ink : 0;
  return AQ_OK;
}

aq_status aq_fluid_download_ink(aq_fluid* f, float* position, float* velocity) {
  if (!f) return fail(AQ_ERR_INVALID_ARGUMENT, "fluid is NULL");
  if (!f->ink_on) return fail(AQ_ERR_INVALID_ARGUMENT, "ink is not enabled");
  cudaSetDevice(f->device);
  AQ_CUDA(cudaStreamSynchronize(f->stream));
  const size_t N = (size_t)f->n_ink;
  const float* src[6] = {f->ink.px, f->ink.py, f->ink.pz, f->ink.vx, f->ink.vy, f->ink.vz};
  for (int k = 0; k < 6 && N; ++k) {
    float* dst = k < 3 ? position : velocity;
    if (!dst) continue;
    AQ_CUDA(cudaMemcpy(dst + (size_t)(k % 3) * N, src[k], sizeof(float) * N, cudaMemcpyDeviceToHost));
  }
  return AQ_OK;
}

aq_status aq_fluid_upload_ink(aq_fluid* f, const float* position, const float* velocity) {
  if (!f) return fail(AQ_ERR_INVALID_ARGUMENT, "fluid is NULL");
  if (!f->ink_on) return fail(AQ_ERR_INVALID_ARGUMENT, "ink is not enabled");
  cudaSetDevice(f->device);
  AQ_CUDA(cudaStreamSynchronize(f->stream));
  const size_t N = (size_t)f->n_ink;
  float* dst[6] = {f->ink.px, f->ink.py, f->ink.pz, f->ink.vx, f->ink.vy, f->ink.vz};
  for (int k = 0; k < 6 && N; ++k) {
    const float* src = k < 3 ? position : velocity;
    if (!src) continue;
    AQ_CUDA(cudaMemcpy(dst[k], src + (size_t)(k % 3) * N, sizeof(float) * N, cudaMemcpyHostToDevice));
  }
  return AQ_OK;
}

aq_status aq_fluid_ink_advance(aq_fluid* f) {
  if (!f) return fail(AQ_ERR_INVALID_ARGUMENT, "fluid is NULL");
  if (!f->ink_on) return fail(AQ_ERR_INVALID_ARGUMENT, "ink is not enabled");
  cudaSetDevice(f->device);
  AQ_TRY(f->enq_ink());
  AQ_CUDA(cudaStreamSynchronize(f->stream));
  return AQ_OK;
}

aq_status aq_fluid_set_warm_start(aq_fluid* f, aq_unet* net) {
  if (!f) return fail(AQ_ERR_INVALID_ARGUMENT, "fluid is NULL");
  cudaSetDevice(f->device);
  AQ_CUDA(cudaStreamSynchronize(f->stream));
  f->invalidate_graph();
  if (!net) {
    f->net = nullptr;
    f->net_acts = nullptr;
    return AQ_OK;
  }
  if (net->device != f->device) return fail(AQ_ERR_INVALID_ARGUMENT, "network and fluid are on different devices");
  aqb::UActs* acts = nullptr;
  AQ_TRY(unet_acts(net, f->d.sx, f->d.sy, f->d.sz, false, &acts));
  if (!f->za) {
    AQ_TRY(f->alloc(&f->za, (size_t)f->d.C));
    AQ_TRY(f->alloc(&f->zb, (size_t)f->d.C));
    AQ_TRY(f->alloc(&f->jpart2, (size_t)f->jpart_cap));
    AQ_TRY(f->alloc(&f->pick, 1));
  }
  if (f->plan.by == 1) f->plan = f->d.sz % 4 == 0 ? JacobiPlan{1, 0, 1} : JacobiPlan{2, 16, 16};
  AQ_CUDA(cudaStreamSynchronize(net->stream));
  f->net = net;
  f->net_acts = acts;
  return AQ_OK;
}

aq_status aq_fluid_launches_per_step(const aq_fluid* f, int32_t* launches) {
  if (!f || !launches) return fail(AQ_ERR_INVALID_ARGUMENT, "bad argument");
  int32_t bodies = 0;
  if (f->body_launches > 0) {
    cudaSetDevice(f->device);
    AQ_CUDA(cudaMemcpyAsync(f->ss_host, f->ss, sizeof(SolveState), cudaMemcpyDeviceToHost, f->stream));
    AQ_CUDA(cudaStreamSynchronize(f->stream));
    bodies = f->ss_host->bodies;
  }
  *launches = f->graph_launches + bodies * f->body_launches;
  return AQ_OK;
}

aq_status aq_fluid_set_jacobi_plan(aq_fluid* f, int32_t levels, int32_t rows, int32_t x_planes) {
  if (!f) return fail(AQ_ERR_INVALID_ARGUMENT, "fluid is NULL");
  if (rows == 1 && f->cfg.pressure_init == AQ_PRESSURE_LEARNED)
    return fail(AQ_ERR_INVALID_ARGUMENT, "the persistent solve does not take the learned warm start");
  if (rows == 1) {  // persistent cooperative solve
    if (levels != 1 || f->d.sz % 4 != 0 || f->ctas <= 0)
      return fail(AQ_ERR_INVALID_ARGUMENT, "persistent solve needs sz % 4 == 0");
    cudaSetDevice(f->device);
    AQ_CUDA(cudaStreamSynchronize(f->stream));
    f->plan = JacobiPlan{1, 1, 1};
    f->invalidate_graph();
    return AQ_OK;
  }
  if (rows == 4) {  // resident tiles: levels = sweeps per halo exchange, x_planes = tile shape
    cudaSetDevice(f->device);
    const int c = f->d.sz % 4 == 0 ? resident_ctas(f->device, x_planes, levels) : 0;
    if (c <= 0) return fail(AQ_ERR_INVALID_ARGUMENT, "unsupported resident plan (levels 4, shape 0-6, sz % 4 == 0)");
    if (f->cfg.pressure_init == AQ_PRESSURE_LEARNED && f->d.sz % 4 != 0)
      return fail(AQ_ERR_INVALID_ARGUMENT, "the learned warm start needs sz % 4 == 0");
    AQ_CUDA(cudaStreamSynchronize(f->stream));
    f->res_ctas = c;
    f->plan = JacobiPlan{levels, 4, x_planes};
    AQ_TRY(f->enq_row_items());  // the learned start's rows, if any
    AQ_CUDA(cudaStreamSynchronize(f->stream));
    f->invalidate_graph();
    return AQ_OK;
  }
  if (rows == 3) {  // list of active warp rows, one sweep per launch
    if (f->d.sz % 4 != 0 || levels != 1 || x_planes != 1)
      return fail(AQ_ERR_INVALID_ARGUMENT, "the list plan is (1, 3, 1) and needs sz % 4 == 0");
    cudaSetDevice(f->device);
    AQ_CUDA(cudaStreamSynchronize(f->stream));
    f->plan = JacobiPlan{1, 3, 1};
    AQ_TRY(f->enq_row_items());  // the current system's rows
    AQ_CUDA(cudaStreamSynchronize(f->stream));
    f->invalidate_graph();
    return AQ_OK;
  }
  if (rows == 2) {  // cube tiles: `levels` sweeps per launch on x_planes-edge tiles
    if (f->d.sz % 4 != 0 || !cube_plan_ok(levels, x_planes))
      return fail(AQ_ERR_INVALID_ARGUMENT, "unsupported cube plan (sz % 4 == 0; edge 8 with 1-4 levels or 16 with 2/4)");
    cudaSetDevice(f->device);
    AQ_CUDA(cudaStreamSynchronize(f->stream));
    f->plan = JacobiPlan{levels, 2, x_planes};
    f->invalidate_graph();
    return AQ_OK;
  }
  const bool flat = rows == 0;
  if (flat ? (levels != 1 || f->d.sz % 4 != 0 || !(x_planes == 1 || x_planes == 2 || x_planes == 4 || x_planes == 8))
           : (!(levels == 1 || levels == 2 || levels == 4 || levels == 8) || !(rows == 8 || rows == 16 || rows == 32) ||
              x_planes < 1))
    return fail(AQ_ERR_INVALID_ARGUMENT, "unsupported Jacobi plan");
  JacobiPlan p{levels, rows, x_planes};
  if (!flat) {
    // every level count the sweeps split into must fit the tile with its
    // halo, including the residual variant (one more level)
    for (int l = levels; l >= 1; l >>= 1) {
      JacobiPlan q = p;
      q.levels = l;
      if (jacobi_parts(f->d, q, true) <= 0 || jacobi_parts(f->d, q, false) <= 0)
        return fail(AQ_ERR_INVALID_ARGUMENT, "tile too small for the plan's halo");
    }
  }
  cudaSetDevice(f->device);
  AQ_CUDA(cudaStreamSynchronize(f->stream));
  int need = 0;
  if (flat) {
    need = resid_flat_parts(f->d);
  } else {
    for (int l = levels; l >= 1; l >>= 1) {
      JacobiPlan q = p;
      q.levels = l;
      need = std::max(need, jacobi_parts(f->d, q, true));
    }
  }
  if (need > f->jpart_cap) {
    double* np_ = nullptr;
    AQ_TRY(f->alloc(&np_, (size_t)need));
    f->jpart = np_;
    f->jpart_cap = need;
  }
  f->plan = p;
  f->invalidate_graph();
  return AQ_OK;
}

aq_status aq_fluid_get_jacobi_plan(const aq_fluid* f, int32_t* levels, int32_t* rows, int32_t* x_planes) {
  if (!f) return fail(AQ_ERR_INVALID_ARGUMENT, "fluid is NULL");
  if (levels) *levels = f->plan.levels;
  if (rows) *rows = f->plan.by;
  if (x_planes) *x_planes = f->plan.xc;
  return AQ_OK;
}

aq_status aq_fluid_launch_counts(const aq_fluid* f, int32_t* per_step, int32_t* per_block) {
  if (!f) return fail(AQ_ERR_INVALID_ARGUMENT, "fluid is NULL");
  if (per_step) *per_step = f->graph_launches;
  if (per_block) *per_block = f->body_launches;
  return AQ_OK;
}

aq_status aq_fluid_benchmark_pressure(aq_fluid* f, int32_t sweeps, float* ms, int32_t* launches,
                                      int64_t* cells_per_sweep) {
  if (!f || sweeps < 1) return fail(AQ_ERR_INVALID_ARGUMENT, "bad argument");
  cudaSetDevice(f->device);
  // The sweeps are captured into a graph and replayed, as inside a step.
  cudaGraph_t g = nullptr;
  AQ_CUDA(cudaStreamBeginCapture(f->stream, cudaStreamCaptureModeThreadLocal));
  aq_status st = f->plan.by == 1   ? enqueue_persistent(f, sweeps)
                 : f->plan.by == 4 ? enqueue_resident(f, sweeps)
                                   : enqueue_sweeps(f, sweeps, false);
  cudaGraph_t got = nullptr;
  cudaError_t ce = cudaStreamEndCapture(f->stream, &got);
  if (st != AQ_OK) { if (got) cudaGraphDestroy(got); return st; }
  if (ce != cudaSuccess) return fail(AQ_ERR_CUDA, cudaGetErrorString(ce));
  g = got;
  cudaGraphExec_t ex = nullptr;
  ce = cudaGraphInstantiate(&ex, g, 0);
  cudaGraphDestroy(g);
  if (ce != cudaSuccess) return fail(AQ_ERR_CUDA, cudaGetErrorString(ce));
  cudaEvent_t a, b;
  AQ_CUDA(cudaEventCreate(&a));
  AQ_CUDA(cudaEventCreate(&b));
  AQ_CUDA(cudaGraphLaunch(ex, f->stream));  // warm
  AQ_CUDA(cudaEventRecord(a, f->stream));
  AQ_CUDA(cudaGraphLaunch(ex, f->stream));
  AQ_CUDA(cudaEventRecord(b, f->stream));
  AQ_CUDA(cudaEventSynchronize(b));
  cudaGraphExecDestroy(ex);
  float t = 0.f;
  AQ_CUDA(cudaEventElapsedTime(&t, a, b));
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  const std::vector<int> parts = split_sweeps(sweeps, f->plan.levels);
  if (ms) *ms = t;
  if (launches)
    *launches = f->plan.by == 1 || f->plan.by == 4 ? 2 : (int32_t)(parts.size() + parts.size() % 2);
  if (cells_per_sweep) {
    std::vector<uint8_t> act((size_t)f->nbricks);
    AQ_CUDA(cudaMemcpy(act.data(), f->bact, act.size(), cudaMemcpyDeviceToHost));
    *cells_per_sweep =
        f->plan.by == 4 ? resident_cells_updated(f->d, f->plan.xc, act.data())
                        : jacobi_cells_updated(f->d, f->plan.by == 1 || f->plan.by == 3 ? JacobiPlan{1, 0, 1} : f->plan,
                                               act.data());
  }
  return AQ_OK;
}

namespace {

std::string tune_key(int device, const Dims& d) {
  cudaDeviceProp prop;
  std::string name = "unknown";
  if (cudaGetDeviceProperties(&prop, device) == cudaSuccess) name = prop.name;
  for (char& c : name)
    if (c == '"' || c == '\\') c = '_';
  return name + "|" + std::to_string(d.sx) + "x" + std::to_string(d.sy) + "x" + std::to_string(d.sz);
}

// The cache is a JSON object of "key": [levels, rows, x_planes, sweep_us];
// written and read by this function only (one entry per line).
bool tune_cache_lookup(const char* path, const std::string& key, int plan[3], float* us) {
  std::ifstream in(path);
  if (!in) return false;
  std::string line;
  const std::string pat = "\"" + key + "\": [";
  while (std::getline(in, line)) {
    const size_t p = line.find(pat);
    if (p == std::string::npos) continue;
    std::istringstream ss(line.substr(p + pat.size()));
    char comma;
    if (ss >> plan[0] >> comma >> plan[1] >> comma >> plan[2] >> comma >> *us) return true;
  }
  return false;
}

void tune_cache_store(const char* path, const std::string& key, const int plan[3], float us) {
  std::vector<std::string> lines;
  {
    std::ifstream in(path);
    std::string line;
    while (in && std::getline(in, line)) {
      if (line.find("\": [") != std::string::npos && line.find("\"" + key + "\"") == std::string::npos) {
        while (!line.empty() && (line.back() == ',' || line.back() == ' ')) line.pop_back();
        lines.push_back(line);
      }
    }
  }
  char buf[512];
  snprintf(buf, sizeof(buf), "  \"%s\": [%d, %d, %d, %.4f]", key.c_str(), plan[0], plan[1], plan[2], us);
  lines.push_back(buf);
  std::ofstream out(path, std::ios::trunc);
  out << "{\n";
  for (size_t i = 0; i < lines.size(); ++i) out << lines[i] << (i + 1 < lines.size() ? ",\n" : "\n");
  out << "}\n";
}

}  // namespace

aq_status aq_fluid_autotune(aq_fluid* f, int32_t sweeps_per_trial, const char* cache_path, aq_tune_result* out) {
  if (!f || sweeps_per_trial < 8) return fail(AQ_ERR_INVALID_ARGUMENT, "bad argument");
  cudaSetDevice(f->device);
  const std::string key = tune_key(f->device, f->d);
  aq_tune_result r;
  memset(&r, 0, sizeof(r));
  int plan[3];
  float us = 0.f;
  if (cache_path && tune_cache_lookup(cache_path, key, plan, &us) &&
      aq_fluid_set_jacobi_plan(f, plan[0], plan[1], plan[2]) == AQ_OK) {
    r.levels = plan[0]; r.rows = plan[1]; r.x_planes = plan[2];
    r.sweep_us = us;
    r.from_cache = 1;
    if (out) *out = r;
    return AQ_OK;
  }
  const int cands[][3] = {{1, 0, 1}, {1, 0, 2}, {1, 1, 1},  {1, 16, 8}, {2, 16, 16}, {2, 32, 16}, {4, 32, 16},
                          {2, 2, 8},  {3, 2, 8},  {4, 2, 8},  {2, 2, 16}, {4, 2, 16},  {1, 3, 1},   {4, 4, 0},
                          {4, 4, 1},  {4, 4, 2},  {4, 4, 3},  {4, 4, 4},  {4, 4, 5},   {4, 4, 6}};
  float best = 1e30f;
  int bestp[3] = {f->plan.levels, f->plan.by, f->plan.xc};
  for (const auto& c : cands) {
    if (aq_fluid_set_jacobi_plan(f, c[0], c[1], c[2]) != AQ_OK) continue;
    float ms = 0.f, ms2 = 0.f;
    if (aq_fluid_benchmark_pressure(f, sweeps_per_trial, &ms, nullptr, nullptr) != AQ_OK) continue;
    if (aq_fluid_benchmark_pressure(f, sweeps_per_trial, &ms2, nullptr, nullptr) != AQ_OK) continue;
    const float t = std::min(ms, ms2) * 1000.f / (float)sweeps_per_trial;
    r.candidates++;
    if (t < best) {
      best = t;
      bestp[0] = c[0]; bestp[1] = c[1]; bestp[2] = c[2];
    }
  }
  AQ_TRY(aq_fluid_set_jacobi_plan(f, bestp[0], bestp[1], bestp[2]));
  r.levels = bestp[0]; r.rows = bestp[1]; r.x_planes = bestp[2];
  r.sweep_us = best;
  if (cache_path && r.candidates > 0) tune_cache_store(cache_path, key, bestp, best);
  if (out) *out = r;
  g_last_error.clear();
  return AQ_OK;
}

}  // extern "C"

// FP64 diagonal-PCG on the fluid's current pressure system; the solution is
// left in f->pcg_x (device, FP64).
aq_status aqb::fluid_pcg_solve(aq_fluid* f, double rel_tol, int max_iter, int* iterations, double* achieved) {
  cudaSetDevice(f->device);
  const Dims& d = f->d;
  const size_t C = (size_t)d.C;
  const int nparts = 1024;
  if (!f->pcg_b) {
    AQ_TRY(f->alloc(&f->pcg_b, C)); AQ_TRY(f->alloc(&f->pcg_x, C)); AQ_TRY(f->alloc(&f->pcg_r, C));
    AQ_TRY(f->alloc(&f->pcg_z, C)); AQ_TRY(f->alloc(&f->pcg_p, C)); AQ_TRY(f->alloc(&f->pcg_q, C));
    AQ_TRY(f->alloc(&f->pcg_part, (size_t)nparts));
  }
  cudaStream_t s = f->stream;
  std::vector<double> hp(nparts);
  auto dot = [&](const double* a, const double* b, double* out) -> aq_status {
    AQ_CUDA(launch_pcg_dot(s, d.C, a, b, f->pcg_part, nparts));
    AQ_CUDA(cudaMemcpyAsync(hp.data(), f->pcg_part, sizeof(double) * nparts, cudaMemcpyDeviceToHost, s));
    AQ_CUDA(cudaStreamSynchronize(s));
    double t = 0.0;
    for (int i = 0; i < nparts; ++i) t += hp[i];
    *out = t;
    return AQ_OK;
  };
  AQ_CUDA(launch_pcg_init(s, d, f->type, f->rhs, f->pcg_b, f->pcg_x));
  AQ_CUDA(cudaMemcpyAsync(f->pcg_r, f->pcg_b, sizeof(double) * C, cudaMemcpyDeviceToDevice, s));
  double bb = 0.0;
  AQ_TRY(dot(f->pcg_b, f->pcg_b, &bb));
  const double bn = sqrt(bb);
  AQ_CUDA(launch_pcg_precond(s, d, f->type, f->pcg_r, f->pcg_z));
  AQ_CUDA(cudaMemcpyAsync(f->pcg_p, f->pcg_z, sizeof(double) * C, cudaMemcpyDeviceToDevice, s));
  double rz = 0.0;
  AQ_TRY(dot(f->pcg_r, f->pcg_z, &rz));
  int it = 0;
  double rn = bn;
  if (bn > 0) {
    for (it = 0; it < max_iter; ++it) {
      AQ_CUDA(launch_pcg_apply(s, d, f->type, f->pcg_p, f->pcg_q));
      double pq = 0.0;
      AQ_TRY(dot(f->pcg_p, f->pcg_q, &pq));
      if (!(pq > 0)) break;
      const double alpha = rz / pq;
      AQ_CUDA(launch_pcg_axpy(s, d.C, alpha, f->pcg_p, f->pcg_x));
      AQ_CUDA(launch_pcg_axpy(s, d.C, -alpha, f->pcg_q, f->pcg_r));
      double rr = 0.0;
      AQ_TRY(dot(f->pcg_r, f->pcg_r, &rr));
      rn = sqrt(rr);
      if (rn <= rel_tol * bn) { ++it; break; }
      AQ_CUDA(launch_pcg_precond(s, d, f->type, f->pcg_r, f->pcg_z));
      double rz2 = 0.0;
      AQ_TRY(dot(f->pcg_r, f->pcg_z, &rz2));
      const double beta = rz2 / rz;
      rz = rz2;
      AQ_CUDA(launch_pcg_xpby(s, d.C, f->pcg_z, beta, f->pcg_p));
    }
  }
  if (iterations) *iterations = it;
  if (achieved) *achieved = bn > 0 ? rn / bn : 0.0;
  return AQ_OK;
}

extern "C" {

aq_status aq_fluid_pcg_reference(aq_fluid* f, double rel_tol, int32_t max_iter, float* pressure_out,
                                 double* rel_error, int32_t* iterations, double* achieved) {
  if (!f) return fail(AQ_ERR_INVALID_ARGUMENT, "fluid is NULL");
  int it_ = 0;
  AQ_TRY(fluid_pcg_solve(f, rel_tol, max_iter, &it_, achieved));
  if (iterations) *iterations = it_;
  const size_t C = (size_t)f->d.C;
  cudaStream_t s = f->stream;
  std::vector<double> x(C);
  std::vector<float> p(C);
  std::vector<int8_t> ty(C);
  AQ_CUDA(cudaMemcpyAsync(x.data(), f->pcg_x, sizeof(double) * C, cudaMemcpyDeviceToHost, s));
  AQ_CUDA(cudaMemcpyAsync(p.data(), f->pa, sizeof(float) * C, cudaMemcpyDeviceToHost, s));
  AQ_CUDA(cudaMemcpyAsync(ty.data(), f->type, C, cudaMemcpyDeviceToHost, s));
  AQ_CUDA(cudaStreamSynchronize(s));
  double num = 0.0, den = 0.0;
  for (size_t c = 0; c < C; ++c) {
    if (ty[c] != kFluid) continue;
    const double e = (double)p[c] - x[c];
    num += e * e;
    den += x[c] * x[c];
  }
  if (rel_error) *rel_error = den > 0 ? sqrt(num / den) : 0.0;
  if (pressure_out)
    for (size_t c = 0; c < C; ++c) pressure_out[c] = (float)x[c];
  return AQ_OK;
}

aq_status aq_fluid_profile_step(aq_fluid* f, float stage_ms[8]) {
  if (!f || !stage_ms) return fail(AQ_ERR_INVALID_ARGUMENT, "bad argument");
  cudaSetDevice(f->device);
  cudaEvent_t ev[9];
  for (int i = 0; i < 9; ++i) AQ_CUDA(cudaEventCreate(&ev[i]));
  AQ_CUDA(cudaEventRecord(ev[0], f->stream));
  f->nv_cur = 2;
  // stages 1+2 are one fused pass here: stage_ms[0] gets it, stage_ms[1] = 0
  AQ_TRY(f->enq_particles(true));
  AQ_CUDA(cudaEventRecord(ev[1], f->stream));
  AQ_CUDA(cudaEventRecord(ev[2], f->stream));
  AQ_TRY(f->enq_p2g(true));
  AQ_CUDA(cudaEventRecord(ev[3], f->stream));
  AQ_TRY(f->enq_divergence());
  AQ_CUDA(cudaEventRecord(ev[4], f->stream));
  if (f->cfg.solve_mode == AQ_SOLVE_RESIDUAL) AQ_TRY(f->enq_solve_residual_eager());
  else AQ_TRY(f->enq_solve_fixed(f->cfg.pressure_iterations));
  AQ_CUDA(cudaEventRecord(ev[5], f->stream));
  AQ_TRY(f->enq_project());
  AQ_CUDA(cudaEventRecord(ev[6], f->stream));
  AQ_TRY(f->enq_extrapolate());
  AQ_CUDA(cudaEventRecord(ev[7], f->stream));
  AQ_TRY(f->enq_diffuse());
  AQ_TRY(f->enq_ink());
  AQ_CUDA(cudaEventRecord(ev[8], f->stream));
  AQ_CUDA(cudaEventSynchronize(ev[8]));
  f->time += (double)f->cfg.timestep;
  for (int i = 0; i < 8; ++i) AQ_CUDA(cudaEventElapsedTime(&stage_ms[i], ev[i], ev[i + 1]));
  for (int i = 0; i < 9; ++i) cudaEventDestroy(ev[i]);
  return AQ_OK;
}

}  // extern "C"
