// Host side of scene batches (aq_batch_* in include/aquarius_b200.h): many
// independent single-phase scenes of uneven grid sizes stepped together, one
// launch per stage over all scenes, the whole step captured in one CUDA graph.
//
// Layout in HBM: every per-particle, per-cell, per-node and per-brick array of
// the single-scene fluid becomes one concatenation over the scenes (scene s at
// offsets p_off / c_off / f_off / br_off / rp_off).  The particle counting
// sort runs once over the concatenated cell keys (key = c_off + cell): the
// exclusive scan then places scene s's particles at [p_off, p_off + n), so
// the sorted order inside a scene is exactly the single-scene order.
//
// Scenes are created by the single-scene path (aq_fluid_create: seeding,
// initial sort and transfer), copied into the concatenated arrays and
// released, so a scene's initial state is the single-scene one bit for bit.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "fluid_impl.cuh"

using namespace aqb;

#define AQB_CUDA(call)                                                                           \
  do {                                                                                           \
    cudaError_t e_ = (call);                                                                     \
    if (e_ != cudaSuccess)                                                                       \
      return fail(e_ == cudaErrorMemoryAllocation ? AQ_ERR_OUT_OF_MEMORY : AQ_ERR_CUDA,          \
                  std::string(#call) + ": " + cudaGetErrorString(e_));                           \
  } while (0)

#define AQB_TRY(expr)             \
  do {                            \
    aq_status s_ = (expr);        \
    if (s_ != AQ_OK) return s_;   \
  } while (0)

namespace {

__global__ void kb_add_const(int* __restrict__ dst, const int* __restrict__ src, int n, int add) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[i] = src[i] + add;
}

__global__ void kb_copy_f(const float* __restrict__ a, float* __restrict__ b, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) b[i] = a[i];
}

inline int cdiv(int a, int b) { return (a + b - 1) / b; }

}  // namespace

struct aq_batch {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  aq_config solver{};  // the shared solver settings
  int ns = 0;
  std::vector<SceneDesc> scenes;
  std::vector<aq_config> cfgs;
  std::vector<double> time;
  std::vector<int> phase;
  // prefix sums of virtual blocks per family, ns + 1 each
  std::vector<int> pre_p, pre_n, pre_b, pre_s, pre_f, pre_r;
  SceneDesc* scenes_d = nullptr;
  int* pre_d = nullptr;
  BatchIndex bi{};
  int N = 0, C = 0, F = 0, NB = 0, NRP = 0;
  int sms = 148;
  int multiple = 64;  // cap on CTAs per SM of a batched launch (occupancy decides below it)
  int xs = 1;         // x planes per packed-row Jacobi item
  bool pipe = false;  // pipelined plane loads (xs > 1)
  int2* row_list = nullptr;  // active (scene, item) pairs of the current systems
  int* n_row_list = nullptr;
  int row_list_cap = 0;

  Particles cur{}, tmp{};
  int *key = nullptr, *slot = nullptr, *perm_u = nullptr, *sort_index = nullptr;
  int *count = nullptr, *off = nullptr, *tile_sums = nullptr;
  float *u0 = nullptr, *v0 = nullptr, *w0 = nullptr;
  float *un1 = nullptr, *vn1 = nullptr, *wn1 = nullptr;
  float *un2 = nullptr, *vn2 = nullptr, *wn2 = nullptr;
  uint8_t *h1 = nullptr, *h2 = nullptr;
  int8_t* type = nullptr;
  float *density = nullptr, *div = nullptr, *rhs = nullptr, *pa = nullptr, *pb = nullptr;
  int* pcount = nullptr;
  uint8_t* bact = nullptr;
  double *part_b2 = nullptr, *rpart = nullptr;
  int* part_nf = nullptr;
  SolveState* ss = nullptr;
  int* live = nullptr;

  cudaGraphExec_t exec = nullptr;
  int graph_launches = 0, body_launches = 0;
  std::vector<void*> allocs;

  ~aq_batch() {
    cudaSetDevice(device);
    if (stream) cudaStreamSynchronize(stream);
    if (exec) cudaGraphExecDestroy(exec);
    for (void* p : allocs) cudaFree(p);
    if (own_stream && stream) cudaStreamDestroy(stream);
  }

  template <typename T>
  aq_status alloc(T** p, size_t n) {
    void* q = nullptr;
    const size_t bytes = std::max<size_t>(n * sizeof(T), 16);
    cudaError_t e = cudaMalloc(&q, bytes);
    if (e != cudaSuccess)
      return fail(e == cudaErrorMemoryAllocation ? AQ_ERR_OUT_OF_MEMORY : AQ_ERR_CUDA,
                  std::string("cudaMalloc: ") + cudaGetErrorString(e));
    allocs.push_back(q);
    *p = (T*)q;
    e = cudaMemsetAsync(q, 0, bytes, stream);
    if (e != cudaSuccess) return fail(AQ_ERR_CUDA, cudaGetErrorString(e));
    return AQ_OK;
  }

  int grid() const { return std::max(1, sms * multiple); }
  int grid512() const { return std::max(1, sms * std::max(1, multiple / 2)); }
  aq_status set_sweep_plan(int planes, bool pipelined);
  aq_status enq_row_list() {
    if (cudaError_t e = launch_batch_row_list(stream, bi, pre_r[ns], xs, bact, row_list, n_row_list))
      return fail(AQ_ERR_CUDA, std::string("row list: ") + cudaGetErrorString(e));
    return AQ_OK;
  }

  aq_status allocate();
  aq_status add_scene(int s, aq_fluid* f);
  aq_status enq_pre_solve();
  aq_status enq_sweeps(int sweeps);
  aq_status enq_solve_fixed();
  aq_status enq_solve_body(unsigned long long handle);
  aq_status enq_post_solve();
  aq_status build_graph();
  void invalidate_graph() {
    if (exec) {
      cudaGraphExecDestroy(exec);
      exec = nullptr;
    }
  }
};

aq_status aq_batch::allocate() {
  const size_t n = (size_t)N, c = (size_t)C, fz = (size_t)F;
  AQB_TRY(alloc(&cur.px, n)); AQB_TRY(alloc(&cur.py, n)); AQB_TRY(alloc(&cur.pz, n));
  AQB_TRY(alloc(&cur.vx, n)); AQB_TRY(alloc(&cur.vy, n)); AQB_TRY(alloc(&cur.vz, n));
  AQB_TRY(alloc(&tmp.px, n)); AQB_TRY(alloc(&tmp.py, n)); AQB_TRY(alloc(&tmp.pz, n));
  AQB_TRY(alloc(&tmp.vx, n)); AQB_TRY(alloc(&tmp.vy, n)); AQB_TRY(alloc(&tmp.vz, n));
  AQB_TRY(alloc(&key, n)); AQB_TRY(alloc(&slot, n)); AQB_TRY(alloc(&perm_u, n)); AQB_TRY(alloc(&sort_index, n));
  AQB_TRY(alloc(&count, c + 1)); AQB_TRY(alloc(&off, c + 1));
  AQB_TRY(alloc(&tile_sums, cell_scan_tiles(C)));
  AQB_TRY(alloc(&u0, fz)); AQB_TRY(alloc(&v0, fz)); AQB_TRY(alloc(&w0, fz));
  AQB_TRY(alloc(&un1, fz)); AQB_TRY(alloc(&vn1, fz)); AQB_TRY(alloc(&wn1, fz));
  AQB_TRY(alloc(&un2, fz)); AQB_TRY(alloc(&vn2, fz)); AQB_TRY(alloc(&wn2, fz));
  AQB_TRY(alloc(&h1, fz)); AQB_TRY(alloc(&h2, fz));
  AQB_TRY(alloc(&type, c)); AQB_TRY(alloc(&density, c)); AQB_TRY(alloc(&div, c)); AQB_TRY(alloc(&rhs, c));
  AQB_TRY(alloc(&pa, c)); AQB_TRY(alloc(&pb, c)); AQB_TRY(alloc(&pcount, c));
  AQB_TRY(alloc(&bact, (size_t)NB)); AQB_TRY(alloc(&part_b2, (size_t)NB)); AQB_TRY(alloc(&part_nf, (size_t)NB));
  AQB_TRY(alloc(&rpart, (size_t)NRP));
  AQB_TRY(alloc(&ss, (size_t)ns)); AQB_TRY(alloc(&live, (size_t)ns));
  AQB_TRY(alloc(&scenes_d, (size_t)ns));
  AQB_TRY(alloc(&pre_d, 6 * (size_t)(ns + 1)));
  row_list_cap = 0;
  for (const SceneDesc& S : scenes) row_list_cap += batch_row_items(S.d, 1);  // one plane per item: the most items
  AQB_TRY(alloc(&row_list, (size_t)row_list_cap));
  AQB_TRY(alloc(&n_row_list, 1));
  AQB_CUDA(cudaMemcpyAsync(scenes_d, scenes.data(), sizeof(SceneDesc) * ns, cudaMemcpyHostToDevice, stream));
  std::vector<int> pre;
  for (const auto* v : {&pre_p, &pre_n, &pre_b, &pre_s, &pre_f}) pre.insert(pre.end(), v->begin(), v->end());
  pre.resize(6 * (size_t)(ns + 1), 0);
  AQB_CUDA(cudaMemcpyAsync(pre_d, pre.data(), sizeof(int) * pre.size(), cudaMemcpyHostToDevice, stream));
  AQB_CUDA(cudaStreamSynchronize(stream));
  bi.scenes = scenes_d;
  bi.n_scenes = ns;
  bi.particles = pre_d;
  bi.nodes = pre_d + (ns + 1);
  bi.bricks = pre_d + 2 * (ns + 1);
  bi.slayer = pre_d + 3 * (ns + 1);
  bi.flat = pre_d + 4 * (ns + 1);
  bi.rows = pre_d + 5 * (ns + 1);
  return set_sweep_plan(xs, pipe);
}

// Packed-row Jacobi items depend on the x planes per item: rebuild their
// prefix sums (and the step graph).
aq_status aq_batch::set_sweep_plan(int planes, bool pipelined) {
  if (planes != 1 && planes != 2 && planes != 4 && planes != 8)
    return fail(AQ_ERR_INVALID_ARGUMENT, "x planes per sweep item must be 1, 2, 4 or 8");
  if (pipelined && planes == 1) return fail(AQ_ERR_INVALID_ARGUMENT, "pipelined sweeps need x planes > 1");
  xs = planes;
  pipe = pipelined;
  pre_r.assign(1, 0);
  for (const SceneDesc& S : scenes) pre_r.push_back(pre_r.back() + batch_row_items(S.d, xs));
  AQB_CUDA(cudaMemcpyAsync(pre_d + 5 * (ns + 1), pre_r.data(), sizeof(int) * (ns + 1), cudaMemcpyHostToDevice,
                           stream));
  AQB_TRY(enq_row_list());  // items depend on the plane count
  AQB_CUDA(cudaStreamSynchronize(stream));
  invalidate_graph();
  return AQ_OK;
}

// Copies the state a step carries over from a freshly initialised scene.
aq_status aq_batch::add_scene(int s, aq_fluid* f) {
  const SceneDesc& S = scenes[s];
  const size_t n = (size_t)S.n, c = (size_t)S.d.C, fz = (size_t)S.d.F;
  auto cp = [&](void* dst, const void* src, size_t bytes) -> aq_status {
    if (bytes) AQB_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, stream));
    return AQ_OK;
  };
  const int p = S.p_off;
  AQB_TRY(cp(cur.px + p, f->cur.px, 4 * n)); AQB_TRY(cp(cur.py + p, f->cur.py, 4 * n));
  AQB_TRY(cp(cur.pz + p, f->cur.pz, 4 * n)); AQB_TRY(cp(cur.vx + p, f->cur.vx, 4 * n));
  AQB_TRY(cp(cur.vy + p, f->cur.vy, 4 * n)); AQB_TRY(cp(cur.vz + p, f->cur.vz, 4 * n));
  if (n) {
    kb_add_const<<<cdiv((int)n, 256), 256, 0, stream>>>(sort_index + p, f->sort_index, (int)n, p);
    AQB_CUDA(cudaGetLastError());
  }
  kb_add_const<<<cdiv((int)c + 1, 256), 256, 0, stream>>>(off + S.c_off, f->off, (int)c + 1, p);
  AQB_CUDA(cudaGetLastError());
  const int o = S.f_off;
  AQB_TRY(cp(u0 + o, f->u0, 4 * fz)); AQB_TRY(cp(v0 + o, f->v0, 4 * fz)); AQB_TRY(cp(w0 + o, f->w0, 4 * fz));
  AQB_TRY(cp(un1 + o, f->un1, 4 * fz)); AQB_TRY(cp(vn1 + o, f->vn1, 4 * fz)); AQB_TRY(cp(wn1 + o, f->wn1, 4 * fz));
  AQB_TRY(cp(un2 + o, f->un2, 4 * fz)); AQB_TRY(cp(vn2 + o, f->vn2, 4 * fz)); AQB_TRY(cp(wn2 + o, f->wn2, 4 * fz));
  AQB_TRY(cp(h1 + o, f->h1, fz)); AQB_TRY(cp(h2 + o, f->h2, fz));
  const int q = S.c_off;
  AQB_TRY(cp(type + q, f->type, c)); AQB_TRY(cp(density + q, f->density, 4 * c)); AQB_TRY(cp(div + q, f->div, 4 * c));
  AQB_TRY(cp(rhs + q, f->rhs, 4 * c)); AQB_TRY(cp(pa + q, f->pa, 4 * c)); AQB_TRY(cp(pb + q, f->pb, 4 * c));
  AQB_TRY(cp(pcount + q, f->pcount, 4 * c));
  AQB_TRY(cp(bact + S.br_off, f->bact, (size_t)f->nbricks));
  AQB_TRY(cp(ss + s, f->ss, sizeof(SolveState)));
  return AQ_OK;
}

// ------------------------------------------------------------------ stages
aq_status aq_batch::enq_pre_solve() {
  const int tp = pre_p[ns], tn = pre_n[ns], tb = pre_b[ns], tsl = pre_s[ns];
  if (N > 0) {
    AQB_CUDA(launch_batch_particles_advance(stream, bi, tp, grid(), true, cur, tmp, u0, v0, w0, un2, vn2, wn2, key,
                                            slot, count));
    AQB_CUDA(launch_cell_scan(stream, C, count, off, tile_sums));
    AQB_CUDA(launch_scatter(stream, key, slot, off, perm_u, N));
    AQB_CUDA(launch_rank_gather(stream, false, key, off, perm_u, tmp, cur, sort_index, N));
  } else {
    AQB_CUDA(launch_cell_scan(stream, C, count, off, tile_sums));
  }
  AQB_CUDA(launch_batch_p2g(stream, bi, tn, grid(), true, cur, off, u0, v0, w0, un1, vn1, wn1, type, density));
  AQB_CUDA(launch_batch_slayer(stream, bi, tsl, grid(), type, un2, vn2, wn2, un1, vn1, wn1, un2, vn2, wn2));
  AQB_CUDA(launch_batch_divergence(stream, bi, tb, grid512(), off, type, density, un1, vn1, wn1, pcount, div, rhs,
                                   pa, pb, solver.pressure_init == AQ_PRESSURE_ZERO, bact, part_b2, part_nf));
  AQB_CUDA(launch_batch_b2_finalize(stream, bi, part_b2, part_nf, ss, live));
  AQB_TRY(enq_row_list());
  return AQ_OK;
}

// `sweeps` sweeps of every live scene from pa; the result of an even count
// ends in pa, of an odd count in pb.
aq_status aq_batch::enq_sweeps(int sweeps) {
  float* bufs[2] = {pa, pb};
  for (int k = 0; k < sweeps; ++k)
    AQB_CUDA(launch_batch_jacobi_rows(stream, bi, pre_r[ns], xs, pipe, grid(), live, bufs[k % 2], bufs[(k + 1) % 2],
                                      rhs, type, bact, row_list, n_row_list));
  return AQ_OK;
}

aq_status aq_batch::enq_solve_fixed() {
  const int K = solver.pressure_iterations;
  if (K <= 0) return AQ_OK;
  AQB_TRY(enq_sweeps(K));
  AQB_CUDA(launch_batch_resid_flat(stream, bi, pre_f[ns], grid(), live, K % 2 ? pb : pa, rhs, type, bact, rpart));
  if (K % 2) {
    kb_copy_f<<<cdiv(C, 256), 256, 0, stream>>>(pb, pa, C);
    AQB_CUDA(cudaGetLastError());
  }
  AQB_CUDA(launch_batch_resid_finalize(stream, bi, rpart, ss, live, K, 0.0, 0));
  return AQ_OK;
}

aq_status aq_batch::enq_solve_body(unsigned long long handle) {
  const int m = solver.check_interval;  // even: the iterate ends in pa
  AQB_TRY(enq_sweeps(m));
  AQB_CUDA(launch_batch_resid_flat(stream, bi, pre_f[ns], grid(), live, pa, rhs, type, bact, rpart));
  AQB_CUDA(launch_batch_resid_finalize(stream, bi, rpart, ss, live, m, (double)solver.rel_residual,
                                       solver.max_iterations));
  AQB_CUDA(launch_batch_solve_condition(stream, live, ns, handle));
  return AQ_OK;
}

aq_status aq_batch::enq_post_solve() {
  const int tn = pre_n[ns];
  AQB_CUDA(launch_batch_project(stream, bi, tn, grid(), type, pa, density, un1, vn1, wn1, h1));
  // extrapolateVelocity: three ping-pong passes, 1 -> 2 -> 1 -> 2
  AQB_CUDA(launch_batch_extrapolate(stream, bi, tn, grid(), un1, vn1, wn1, h1, un2, vn2, wn2, h2));
  AQB_CUDA(launch_batch_extrapolate(stream, bi, tn, grid(), un2, vn2, wn2, h2, un1, vn1, wn1, h1));
  AQB_CUDA(launch_batch_extrapolate(stream, bi, tn, grid(), un1, vn1, wn1, h1, un2, vn2, wn2, h2));
  return AQ_OK;
}

aq_status aq_batch::build_graph() {
  invalidate_graph();
  cudaGraph_t g = nullptr;
  AQB_CUDA(cudaGraphCreate(&g, 0));
  auto capture = [&](cudaGraph_t into, const cudaGraphNode_t* deps, size_t nd, auto&& body) -> aq_status {
    AQB_CUDA(cudaStreamBeginCaptureToGraph(stream, into, deps, nullptr, nd, cudaStreamCaptureModeThreadLocal));
    aq_status st = body();
    cudaGraph_t got = nullptr;
    cudaError_t e = cudaStreamEndCapture(stream, &got);
    if (st != AQ_OK) return st;
    if (e != cudaSuccess) return fail(AQ_ERR_CUDA, std::string("capture: ") + cudaGetErrorString(e));
    return AQ_OK;
  };
  const int pre_launches = (N > 0 ? 6 : 3) + 5;  // sort; p2g, s-layer, divergence, b2, row list
  const int post_launches = 4;
  aq_status st;
  if (solver.solve_mode == AQ_SOLVE_RESIDUAL) {
    st = capture(g, nullptr, 0, [&]() { return enq_pre_solve(); });
    if (st != AQ_OK) { cudaGraphDestroy(g); return st; }
    size_t nn = 0;
    cudaGraphGetNodes(g, nullptr, &nn);
    std::vector<cudaGraphNode_t> nodes(nn), leaves;
    cudaGraphGetNodes(g, nodes.data(), &nn);
    for (cudaGraphNode_t nd : nodes) {
      size_t k = 0;
      cudaGraphNodeGetDependentNodes(nd, nullptr, &k);
      if (k == 0) leaves.push_back(nd);
    }
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
    st = capture(cp.conditional.phGraph_out[0], nullptr, 0,
                 [&]() { return enq_solve_body((unsigned long long)handle); });
    if (st != AQ_OK) { cudaGraphDestroy(g); return st; }
    st = capture(g, &cnode, 1, [&]() { return enq_post_solve(); });
    body_launches = solver.check_interval + 3;
    graph_launches = pre_launches + post_launches;
  } else {
    st = capture(g, nullptr, 0, [&]() {
      aq_status s2 = enq_pre_solve();
      if (s2 != AQ_OK) return s2;
      s2 = enq_solve_fixed();
      if (s2 != AQ_OK) return s2;
      return enq_post_solve();
    });
    const int K = solver.pressure_iterations;
    body_launches = 0;
    graph_launches = pre_launches + post_launches + (K > 0 ? K + 2 + (K % 2) : 0);
  }
  if (st != AQ_OK) { cudaGraphDestroy(g); return st; }
  cudaError_t e = cudaGraphInstantiate(&exec, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) { exec = nullptr; return fail(AQ_ERR_CUDA, std::string("instantiate: ") + cudaGetErrorString(e)); }
  return AQ_OK;
}

// ====================================================================== ABI
namespace {

bool same_solver(const aq_config& a, const aq_config& b) {
  return a.pressure_iterations == b.pressure_iterations && a.pressure_init == b.pressure_init &&
         a.solve_mode == b.solve_mode && a.rel_residual == b.rel_residual &&
         a.max_iterations == b.max_iterations && a.check_interval == b.check_interval && a.device == b.device &&
         a.stream == b.stream;
}

}  // namespace

extern "C" {

aq_status aq_batch_create(const aq_config* configs, int32_t n_scenes, aq_batch** out) {
  if (!out) return fail(AQ_ERR_INVALID_ARGUMENT, "out is NULL");
  *out = nullptr;
  if (!configs || n_scenes < 1) return fail(AQ_ERR_INVALID_ARGUMENT, "need at least one scene config");
  const aq_config& c0 = configs[0];
  long long C = 0, F = 0, NB = 0, NRP = 0;
  for (int s = 0; s < n_scenes; ++s) {
    const aq_config& c = configs[s];
    AQB_TRY(aq_config_validate(&c));
    if (c.size_z % 4 != 0) return fail(AQ_ERR_INVALID_CONFIG, "batched scenes need size_z % 4 == 0");
    if (!same_solver(c, c0))
      return fail(AQ_ERR_INVALID_CONFIG, "batched scenes must share the pressure solver settings, device and stream");
    for (int v = 1; v < c.volume_count; ++v)
      if (c.volumes[v].phase != c.volumes[0].phase)
        return fail(AQ_ERR_INVALID_CONFIG, "batched scenes must be single-phase");
    C += (long long)c.size_x * c.size_y * c.size_z;
    F += (long long)(c.size_x + 1) * (c.size_y + 1) * (c.size_z + 1);
    NB += (long long)cdiv(c.size_x, kBrick) * cdiv(c.size_y, kBrick) * cdiv(c.size_z, kBrick);
    NRP += (long long)((c.size_z / 4 + 31) / 32) * ((c.size_y + 7) / 8) * c.size_x;
  }
  if (c0.pressure_init == AQ_PRESSURE_LEARNED)
    return fail(AQ_ERR_INVALID_CONFIG, "batched scenes do not take the learned warm start");
  if (c0.solve_mode == AQ_SOLVE_RESIDUAL && c0.check_interval % 2 != 0)
    return fail(AQ_ERR_INVALID_CONFIG, "batched residual solves need an even check_interval");
  if (C + 1 >= (1LL << 31) || F >= (1LL << 31)) return fail(AQ_ERR_INVALID_CONFIG, "batch too large for 32-bit indices");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return fail(AQ_ERR_NO_DEVICE, "no CUDA device");
  }
  if (c0.device < 0 || c0.device >= ndev) return fail(AQ_ERR_INVALID_CONFIG, "device ordinal out of range");

  aq_batch* b = new aq_batch();
  b->device = c0.device;
  b->solver = c0;
  b->ns = n_scenes;
  auto bail = [&](aq_status st) {
    delete b;
    return st;
  };
  if (cudaSetDevice(b->device) != cudaSuccess) return bail(fail(AQ_ERR_CUDA, "cudaSetDevice"));
  if (c0.stream) {
    b->stream = (cudaStream_t)c0.stream;
  } else {
    if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess)
      return bail(fail(AQ_ERR_CUDA, "cudaStreamCreate"));
    b->own_stream = true;
  }
  cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, b->device);
  b->C = (int)C;
  b->F = (int)F;
  b->NB = (int)NB;
  b->NRP = (int)NRP;

  // Each scene is created alone (seeding, initial sort and transfer), then
  // copied into the concatenated arrays; the scene fluids are released after.
  std::vector<aq_fluid*> fl((size_t)n_scenes, nullptr);
  auto release = [&]() {
    for (aq_fluid*& f : fl) {
      if (f) aq_fluid_destroy(f);
      f = nullptr;
    }
  };
  b->scenes.resize(n_scenes);
  b->cfgs.assign(configs, configs + n_scenes);
  b->time.assign(n_scenes, 0.0);
  b->phase.assign(n_scenes, 0);
  long long P = 0;
  int c_off = 0, f_off = 0, br_off = 0, rp_off = 0;
  b->pre_p.assign(1, 0); b->pre_n.assign(1, 0); b->pre_b.assign(1, 0); b->pre_s.assign(1, 0); b->pre_f.assign(1, 0);
  for (int s = 0; s < n_scenes; ++s) {
    aq_config c = configs[s];
    c.stream = b->stream;
    aq_status st = aq_fluid_create(&c, &fl[s]);
    if (st != AQ_OK) { release(); return bail(st); }
    const aq_fluid* f = fl[s];
    if (f->multiphase) {
      release();
      return bail(fail(AQ_ERR_INVALID_CONFIG, "batched scenes must be single-phase"));
    }
    SceneDesc& S = b->scenes[s];
    S.d = f->d;
    S.sp = f->sp;
    S.n = f->n;
    S.p_off = (int)P;
    S.c_off = c_off;
    S.f_off = f_off;
    S.br_off = br_off;
    S.rp_off = rp_off;
    b->phase[s] = f->phase;
    P += S.n;
    if (P >= (1LL << 31)) {
      release();
      return bail(fail(AQ_ERR_INVALID_CONFIG, "batch too large for 32-bit particle indices"));
    }
    const Dims& d = S.d;
    c_off += d.C;
    f_off += d.F;
    br_off += d.bx * d.by * d.bz;
    rp_off += resid_flat_parts(d);
    b->pre_p.push_back(b->pre_p.back() + cdiv(S.n, 256));
    b->pre_n.push_back(b->pre_n.back() + cdiv(d.sz, 32) * cdiv(d.sy, 8) * d.sx);
    b->pre_b.push_back(b->pre_b.back() + d.bx * d.by * d.bz);
    b->pre_s.push_back(b->pre_s.back() + cdiv(d.F - d.C, 256));
    b->pre_f.push_back(b->pre_f.back() + resid_flat_parts(d));
  }
  b->N = (int)P;
  aq_status st = b->allocate();
  for (int s = 0; s < n_scenes && st == AQ_OK; ++s) st = b->add_scene(s, fl[s]);
  if (st == AQ_OK) st = b->enq_row_list();  // the scenes' initial activity bricks
  if (st == AQ_OK && cudaStreamSynchronize(b->stream) != cudaSuccess)
    st = fail(AQ_ERR_CUDA, "batch initialisation failed");
  release();
  if (st != AQ_OK) return bail(st);

  *out = b;
  return AQ_OK;
}

aq_status aq_batch_step(aq_batch* b, int32_t n_steps) {
  if (!b || n_steps < 0) return fail(AQ_ERR_INVALID_ARGUMENT, "bad argument");
  cudaSetDevice(b->device);
  if (!b->exec) AQB_TRY(b->build_graph());
  for (int i = 0; i < n_steps; ++i) {
    AQB_CUDA(cudaGraphLaunch(b->exec, b->stream));
    for (int s = 0; s < b->ns; ++s) b->time[s] += (double)b->cfgs[s].timestep;
  }
  return AQ_OK;
}

aq_status aq_batch_step_host(aq_batch* b, int32_t n_steps, const float* pin, const float* vin, float* pout,
                             float* vout) {
  if (!b || n_steps < 0) return fail(AQ_ERR_INVALID_ARGUMENT, "bad argument");
  cudaSetDevice(b->device);
  const size_t N = (size_t)b->N;
  cudaStream_t s = b->stream;
  float* dp[3] = {b->cur.px, b->cur.py, b->cur.pz};
  float* dv[3] = {b->cur.vx, b->cur.vy, b->cur.vz};
  if (N) {
    for (int k = 0; k < 3; ++k) {
      if (pin) AQB_CUDA(cudaMemcpyAsync(dp[k], pin + k * N, 4 * N, cudaMemcpyHostToDevice, s));
      if (vin) AQB_CUDA(cudaMemcpyAsync(dv[k], vin + k * N, 4 * N, cudaMemcpyHostToDevice, s));
    }
  }
  AQB_TRY(aq_batch_step(b, n_steps));
  if (N) {
    for (int k = 0; k < 3; ++k) {
      if (pout) AQB_CUDA(cudaMemcpyAsync(pout + k * N, dp[k], 4 * N, cudaMemcpyDeviceToHost, s));
      if (vout) AQB_CUDA(cudaMemcpyAsync(vout + k * N, dv[k], 4 * N, cudaMemcpyDeviceToHost, s));
    }
  }
  AQB_CUDA(cudaStreamSynchronize(s));
  return AQ_OK;
}

aq_status aq_batch_stream(const aq_batch* b, void** stream) {
  if (!b || !stream) return fail(AQ_ERR_INVALID_ARGUMENT, "bad argument");
  *stream = (void*)b->stream;
  return AQ_OK;
}

aq_status aq_batch_synchronize(aq_batch* b) {
  if (!b) return fail(AQ_ERR_INVALID_ARGUMENT, "batch is NULL");
  cudaSetDevice(b->device);
  AQB_CUDA(cudaStreamSynchronize(b->stream));
  return AQ_OK;
}

int32_t aq_batch_scene_count(const aq_batch* b) { return b ? b->ns : 0; }

aq_status aq_batch_scene_info(const aq_batch* b, int32_t scene, int32_t size_xyz[3], int64_t* particle_count) {
  if (!b || scene < 0 || scene >= b->ns) return fail(AQ_ERR_INVALID_ARGUMENT, "bad scene index");
  const SceneDesc& S = b->scenes[scene];
  if (size_xyz) { size_xyz[0] = S.d.sx; size_xyz[1] = S.d.sy; size_xyz[2] = S.d.sz; }
  if (particle_count) *particle_count = S.n;
  return AQ_OK;
}

aq_status aq_batch_totals(const aq_batch* b, int64_t* cells, int64_t* nodes, int64_t* particles) {
  if (!b) return fail(AQ_ERR_INVALID_ARGUMENT, "batch is NULL");
  if (cells) *cells = b->C;
  if (nodes) *nodes = b->F;
  if (particles) *particles = b->N;
  return AQ_OK;
}

aq_status aq_batch_download_scene(aq_batch* b, int32_t scene, aq_host_state* s) {
  if (!b || !s || scene < 0 || scene >= b->ns) return fail(AQ_ERR_INVALID_ARGUMENT, "bad argument");
  cudaSetDevice(b->device);
  const SceneDesc& S = b->scenes[scene];
  // A non-owning single-scene view of the scene's slices.
  aq_fluid v;
  v.cfg = b->cfgs[scene];
  v.device = b->device;
  v.stream = b->stream;
  v.d = S.d;
  v.sp = S.sp;
  v.n = S.n;
  v.multiphase = false;
  v.phase = b->phase[scene];
  v.time = b->time[scene];
  v.index_base = S.p_off;
  const int p = S.p_off, c = S.c_off, o = S.f_off;
  v.cur.px = b->cur.px + p; v.cur.py = b->cur.py + p; v.cur.pz = b->cur.pz + p;
  v.cur.vx = b->cur.vx + p; v.cur.vy = b->cur.vy + p; v.cur.vz = b->cur.vz + p;
  v.sort_index = b->sort_index + p;
  v.off = b->off + c;
  v.u0 = b->u0 + o; v.v0 = b->v0 + o; v.w0 = b->w0 + o;
  v.un1 = b->un1 + o; v.vn1 = b->vn1 + o; v.wn1 = b->wn1 + o;
  v.un2 = b->un2 + o; v.vn2 = b->vn2 + o; v.wn2 = b->wn2 + o;
  v.h1 = b->h1 + o; v.h2 = b->h2 + o;
  v.nv_cur = v.has_cur = 2;
  v.type = b->type + c; v.density = b->density + c; v.div = b->div + c; v.rhs = b->rhs + c;
  v.pa = b->pa + c; v.pb = b->pb + c; v.pcount = b->pcount + c;
  aq_status st = v.download(s);
  v.stream = nullptr;  // the view owns nothing
  v.device = -1;
  return st;
}

aq_status aq_batch_solve_stats(aq_batch* b, int32_t scene, aq_solve_stats* out) {
  if (!b || !out || scene < 0 || scene >= b->ns) return fail(AQ_ERR_INVALID_ARGUMENT, "bad argument");
  cudaSetDevice(b->device);
  SolveState s;
  AQB_CUDA(cudaStreamSynchronize(b->stream));
  AQB_CUDA(cudaMemcpy(&s, b->ss + scene, sizeof(SolveState), cudaMemcpyDeviceToHost));
  out->iterations = s.iterations;
  out->rel_residual = s.rel_residual;
  out->b_norm = s.b2 >= 0 ? sqrt(s.b2) : -1.0;
  out->fluid_cells = s.fluid_cells;
  out->converged = s.converged;
  out->blocks = s.bodies;
  out->total_sweeps = s.total_sweeps;
  out->total_blocks = s.total_bodies;
  out->warm_start = s.warm;
  out->warm_rel_residual = s.warm_rel;
  out->zero_rel_residual = s.zero_rel;
  return AQ_OK;
}

aq_status aq_batch_launch_counts(const aq_batch* b, int32_t* per_step, int32_t* per_block) {
  if (!b) return fail(AQ_ERR_INVALID_ARGUMENT, "batch is NULL");
  if (!b->exec) AQB_TRY(const_cast<aq_batch*>(b)->build_graph());
  if (per_step) *per_step = b->graph_launches;
  if (per_block) *per_block = b->body_launches;
  return AQ_OK;
}

aq_status aq_batch_set_grid_multiple(aq_batch* b, int32_t multiple) {
  if (!b || multiple < 1 || multiple > 64) return fail(AQ_ERR_INVALID_ARGUMENT, "multiple must be in [1, 64]");
  b->multiple = multiple;
  b->invalidate_graph();
  return AQ_OK;
}

aq_status aq_batch_set_sweep_plan(aq_batch* b, int32_t x_planes, int32_t pipelined) {
  if (!b) return fail(AQ_ERR_INVALID_ARGUMENT, "batch is NULL");
  cudaSetDevice(b->device);
  return b->set_sweep_plan(x_planes, pipelined != 0);
}

aq_status aq_batch_get_sweep_plan(const aq_batch* b, int32_t* x_planes, int32_t* pipelined) {
  if (!b) return fail(AQ_ERR_INVALID_ARGUMENT, "batch is NULL");
  if (x_planes) *x_planes = b->xs;
  if (pipelined) *pipelined = b->pipe ? 1 : 0;
  return AQ_OK;
}

aq_status aq_batch_autotune(aq_batch* b, int32_t sweeps_per_trial, int32_t* x_planes, int32_t* pipelined,
                            float* sweep_us) {
  if (!b || sweeps_per_trial < 2) return fail(AQ_ERR_INVALID_ARGUMENT, "bad argument");
  cudaSetDevice(b->device);
  int best = b->xs;
  bool best_pipe = b->pipe;
  float best_ms = -1.f;
  const int cand[][2] = {{1, 0}, {2, 0}, {4, 0}, {8, 0}, {2, 1}, {4, 1}, {8, 1}};
  for (const auto& c : cand) {
    AQB_TRY(b->set_sweep_plan(c[0], c[1] != 0));
    float ms = 0.f;
    AQB_TRY(aq_batch_benchmark_pressure(b, sweeps_per_trial, &ms, nullptr));
    if (best_ms < 0.f || ms < best_ms) {
      best_ms = ms;
      best = c[0];
      best_pipe = c[1] != 0;
    }
  }
  AQB_TRY(b->set_sweep_plan(best, best_pipe));
  if (x_planes) *x_planes = best;
  if (pipelined) *pipelined = best_pipe ? 1 : 0;
  if (sweep_us) *sweep_us = 1000.f * best_ms / (float)sweeps_per_trial;
  return AQ_OK;
}

aq_status aq_batch_benchmark_pressure(aq_batch* b, int32_t sweeps, float* ms, int64_t* cells_per_sweep) {
  if (!b || sweeps < 1) return fail(AQ_ERR_INVALID_ARGUMENT, "bad argument");
  cudaSetDevice(b->device);
  // every scene takes part
  std::vector<int> ones((size_t)b->ns, 1);
  AQB_CUDA(cudaMemcpyAsync(b->live, ones.data(), sizeof(int) * ones.size(), cudaMemcpyHostToDevice, b->stream));
  AQB_CUDA(cudaStreamSynchronize(b->stream));
  const int k = sweeps + (sweeps % 2);  // even: the iterate stays in pa
  AQB_CUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
  aq_status st = b->enq_sweeps(k);
  cudaGraph_t g = nullptr;
  cudaError_t ce = cudaStreamEndCapture(b->stream, &g);
  if (st != AQ_OK) { if (g) cudaGraphDestroy(g); return st; }
  if (ce != cudaSuccess) return fail(AQ_ERR_CUDA, cudaGetErrorString(ce));
  cudaGraphExec_t ex = nullptr;
  ce = cudaGraphInstantiate(&ex, g, 0);
  cudaGraphDestroy(g);
  if (ce != cudaSuccess) return fail(AQ_ERR_CUDA, cudaGetErrorString(ce));
  cudaEvent_t e0, e1;
  AQB_CUDA(cudaEventCreate(&e0));
  AQB_CUDA(cudaEventCreate(&e1));
  AQB_CUDA(cudaGraphLaunch(ex, b->stream));
  AQB_CUDA(cudaEventRecord(e0, b->stream));
  AQB_CUDA(cudaGraphLaunch(ex, b->stream));
  AQB_CUDA(cudaEventRecord(e1, b->stream));
  AQB_CUDA(cudaEventSynchronize(e1));
  cudaGraphExecDestroy(ex);
  float t = 0.f;
  AQB_CUDA(cudaEventElapsedTime(&t, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (ms) *ms = t * (float)sweeps / (float)k;
  if (cells_per_sweep) {
    std::vector<uint8_t> act((size_t)b->NB);
    AQB_CUDA(cudaMemcpy(act.data(), b->bact, act.size(), cudaMemcpyDeviceToHost));
    long long cells = 0;
    for (int s = 0; s < b->ns; ++s)
      cells += batch_row_cells_updated(b->scenes[s].d, b->xs, act.data() + b->scenes[s].br_off);
    *cells_per_sweep = cells;
  }
  return AQ_OK;
}

void aq_batch_destroy(aq_batch* b) { delete b; }

}  // extern "C"
