// Host side of the learned pressure warm start (aq_unet_*, aq_dataset_* and
// the convolution building blocks in include/aquarius_b200.h).  No
// counterpart in the reference.
//
// Network: a 3-level 3D U-Net, 16/32/64 channels, 3x3x3 convolutions + ReLU,
// 2x2x2 average pooling down, nearest-neighbour upsampling + concatenation
// up, a 1x1x1 output head.  BF16 weights and activations, FP32 accumulation
// and FP32 master weights (Adam).  Input (16 channels, 2 used): rhs scaled by
// its max-abs, and 1 on fluid cells / 0 on air (no solid cells exist inside
// the grid); output: pressure / (max|rhs| * out_scale).
//
//   e1a = conv(in,16) e1 = conv(e1a,16) | p1 = pool(e1)
//   e2a = conv(p1,32) e2 = conv(e2a,32) | p2 = pool(e2)
//   b1 = conv(p2,64)  b2 = conv(b1,64)
//   u2 = [up(b2), e2] d2a = conv(u2,32) d2 = conv(d2a,32)
//   u1 = [up(d2), e1] d1a = conv(u1,16) d1 = conv(d1a,16) | out = head(d1)
#include <cuda_bf16.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "fluid_impl.cuh"
#include "unet_impl.cuh"

using namespace aqb;
using bf16 = __nv_bfloat16;

#define UN_CUDA(call)                                                                            \
  do {                                                                                           \
    cudaError_t e_ = (call);                                                                     \
    if (e_ != cudaSuccess)                                                                       \
      return fail(e_ == cudaErrorMemoryAllocation ? AQ_ERR_OUT_OF_MEMORY : AQ_ERR_CUDA,          \
                  std::string(#call) + ": " + cudaGetErrorString(e_));                           \
  } while (0)

#define UN_TRY(expr)              \
  do {                            \
    aq_status s_ = (expr);        \
    if (s_ != AQ_OK) return s_;   \
  } while (0)

namespace {

constexpr int kLayerIO[10][2] = {{16, 16}, {16, 16}, {16, 32}, {32, 32}, {32, 64},
                                 {64, 64}, {96, 32}, {32, 32}, {48, 16}, {16, 16}};
constexpr uint32_t kMagic = 0x54454e55u;  // "UNET"
constexpr uint32_t kVersion = 1;

template <typename T>
aq_status dalloc(std::vector<void*>& allocs, T** p, size_t n, cudaStream_t st) {
  void* q = nullptr;
  const size_t bytes = std::max<size_t>(n * sizeof(T), 16);
  cudaError_t e = cudaMalloc(&q, bytes);
  if (e != cudaSuccess)
    return fail(e == cudaErrorMemoryAllocation ? AQ_ERR_OUT_OF_MEMORY : AQ_ERR_CUDA,
                std::string("cudaMalloc: ") + cudaGetErrorString(e));
  allocs.push_back(q);
  *p = (T*)q;
  e = cudaMemsetAsync(q, 0, bytes, st);
  if (e != cudaSuccess) return fail(AQ_ERR_CUDA, cudaGetErrorString(e));
  return AQ_OK;
}

aq_status refresh_bf16(aq_unet* net) {
  for (UConv& c : net->L) {
    UN_CUDA(launch_f32_to_bf16(net->stream, c.w, c.wb, c.nw()));
    UN_CUDA(launch_flip_transpose(net->stream, c.wb, c.wt, c.cin, c.cout));
  }
  return AQ_OK;
}

}  // namespace

aq_unet::~aq_unet() {
  cudaSetDevice(device);
  if (stream) cudaStreamSynchronize(stream);
  for (UActs* a : acts) {
    for (void* p : a->allocs) cudaFree(p);
    delete a;
  }
  for (void* p : allocs) cudaFree(p);
  if (own_stream && stream) cudaStreamDestroy(stream);
}

aq_status aqb::unet_acts(aq_unet* net, int sx, int sy, int sz, bool grads, UActs** out) {
  if (sx % 4 || sy % 4 || sz % 4 || sx < 4 || sy < 4 || sz < 4)
    return fail(AQ_ERR_INVALID_ARGUMENT, "the U-Net needs grid sizes divisible by 4");
  for (UActs* a : net->acts)
    if (a->sx == sx && a->sy == sy && a->sz == sz && (a->grads || !grads)) {
      *out = a;
      return AQ_OK;
    }
  UActs* a = new UActs();
  a->sx = sx; a->sy = sy; a->sz = sz;
  net->acts.push_back(a);
  const size_t V = (size_t)sx * sy * sz, V2 = V / 8, V4 = V / 64;
  cudaStream_t st = net->stream;
  auto& al = a->allocs;
  UN_TRY(dalloc(al, &a->in0, V * 16, st));
  UN_TRY(dalloc(al, &a->e1a, V * 16, st)); UN_TRY(dalloc(al, &a->e1, V * 16, st));
  UN_TRY(dalloc(al, &a->p1, V2 * 16, st));
  UN_TRY(dalloc(al, &a->e2a, V2 * 32, st)); UN_TRY(dalloc(al, &a->e2, V2 * 32, st));
  UN_TRY(dalloc(al, &a->p2, V4 * 32, st));
  UN_TRY(dalloc(al, &a->b1, V4 * 64, st)); UN_TRY(dalloc(al, &a->b2, V4 * 64, st));
  UN_TRY(dalloc(al, &a->u2, V2 * 96, st));
  UN_TRY(dalloc(al, &a->d2a, V2 * 32, st)); UN_TRY(dalloc(al, &a->d2, V2 * 32, st));
  UN_TRY(dalloc(al, &a->u1, V * 48, st));
  UN_TRY(dalloc(al, &a->d1a, V * 16, st)); UN_TRY(dalloc(al, &a->d1, V * 16, st));
  UN_TRY(dalloc(al, &a->out, V, st));
  if (grads) {
    a->grads = true;
    UN_TRY(dalloc(al, &a->g_e1a, V * 16, st)); UN_TRY(dalloc(al, &a->g_e1, V * 16, st));
    UN_TRY(dalloc(al, &a->g_p1, V2 * 16, st));
    UN_TRY(dalloc(al, &a->g_e2a, V2 * 32, st)); UN_TRY(dalloc(al, &a->g_e2, V2 * 32, st));
    UN_TRY(dalloc(al, &a->g_p2, V4 * 32, st));
    UN_TRY(dalloc(al, &a->g_b1, V4 * 64, st)); UN_TRY(dalloc(al, &a->g_b2, V4 * 64, st));
    UN_TRY(dalloc(al, &a->g_u2, V2 * 96, st));
    UN_TRY(dalloc(al, &a->g_d2a, V2 * 32, st)); UN_TRY(dalloc(al, &a->g_d2, V2 * 32, st));
    UN_TRY(dalloc(al, &a->g_u1, V * 48, st));
    UN_TRY(dalloc(al, &a->g_d1a, V * 16, st)); UN_TRY(dalloc(al, &a->g_d1, V * 16, st));
    size_t wp = 0;
    const size_t vox[10] = {V, V, V2, V2, V4, V4, V2, V2, V, V};
    for (int l = 0; l < 10; ++l)
      wp = std::max(wp, conv3_wgrad_part_floats(kLayerIO[l][0], kLayerIO[l][1], (int)vox[l]));
    UN_TRY(dalloc(al, &a->wpart, wp, st));
    UN_TRY(dalloc(al, &a->cpart, (size_t)chan_sum_parts((int)V) * 96, st));
    UN_TRY(dalloc(al, &a->le, V, st)); UN_TRY(dalloc(al, &a->l0, V, st)); UN_TRY(dalloc(al, &a->l1, V, st));
    UN_TRY(dalloc(al, &a->l2, V, st)); UN_TRY(dalloc(al, &a->l3, V, st)); UN_TRY(dalloc(al, &a->lg, V, st));
    UN_TRY(dalloc(al, &a->lpart, (size_t)loss_parts() * 8, st));
    UN_TRY(dalloc(al, &a->lsums, 8, st));
    UN_TRY(dalloc(al, &a->hpart, (size_t)loss_parts() * 17, st));
  }
  *out = a;
  return AQ_OK;
}

namespace {

aq_status conv(aq_unet* net, cudaStream_t st, int l, const bf16* in, bf16* out, int sx, int sy, int sz) {
  const UConv& c = net->L[l];
  UN_CUDA(launch_conv3_fwd(st, c.cin, c.cout, true, in, c.wb, c.b, out, sx, sy, sz));
  return AQ_OK;
}

aq_status forward(aq_unet* net, cudaStream_t st, UActs* a) {
  const int sx = a->sx, sy = a->sy, sz = a->sz;
  const int hx = sx / 2, hy = sy / 2, hz = sz / 2, qx = sx / 4, qy = sy / 4, qz = sz / 4;
  UN_TRY(conv(net, st, 0, a->in0, a->e1a, sx, sy, sz));
  UN_TRY(conv(net, st, 1, a->e1a, a->e1, sx, sy, sz));
  UN_CUDA(launch_pool2(st, a->e1, a->p1, sx, sy, sz, 16));
  UN_TRY(conv(net, st, 2, a->p1, a->e2a, hx, hy, hz));
  UN_TRY(conv(net, st, 3, a->e2a, a->e2, hx, hy, hz));
  UN_CUDA(launch_pool2(st, a->e2, a->p2, hx, hy, hz, 32));
  UN_TRY(conv(net, st, 4, a->p2, a->b1, qx, qy, qz));
  UN_TRY(conv(net, st, 5, a->b1, a->b2, qx, qy, qz));
  UN_CUDA(launch_upcat(st, a->b2, a->e2, a->u2, hx, hy, hz, 64, 32));
  UN_TRY(conv(net, st, 6, a->u2, a->d2a, hx, hy, hz));
  UN_TRY(conv(net, st, 7, a->d2a, a->d2, hx, hy, hz));
  UN_CUDA(launch_upcat(st, a->d2, a->e1, a->u1, sx, sy, sz, 32, 16));
  UN_TRY(conv(net, st, 8, a->u1, a->d1a, sx, sy, sz));
  UN_TRY(conv(net, st, 9, a->d1a, a->d1, sx, sy, sz));
  UN_CUDA(launch_head_fwd(st, a->d1, net->hp, net->hp + 16, a->out, sx * sy * sz));
  return AQ_OK;
}

// Gradients of layer l from dy (ReLU already applied to dy): weights, bias
// and, if dx, the data gradient.
aq_status conv_bwd(aq_unet* net, cudaStream_t st, UActs* a, int l, const bf16* x, bf16* dy, bf16* dx, int sx, int sy,
                   int sz) {
  const UConv& c = net->L[l];
  UN_CUDA(launch_conv3_wgrad(st, c.cin, c.cout, x, dy, a->wpart, c.g, sx, sy, sz));
  UN_CUDA(launch_chan_sum(st, dy, sx * sy * sz, c.cout, a->cpart, c.gb));
  if (dx) UN_CUDA(launch_conv3_fwd(st, c.cout, c.cin, false, dy, c.wt, nullptr, dx, sx, sy, sz));
  return AQ_OK;
}

aq_status backward(aq_unet* net, cudaStream_t st, UActs* a, const float* target, const int8_t* type, float alpha,
                   int k) {
  const int sx = a->sx, sy = a->sy, sz = a->sz;
  const int hx = sx / 2, hy = sy / 2, hz = sz / 2, qx = sx / 4, qy = sy / 4, qz = sz / 4;
  const int V = sx * sy * sz, V2 = V / 8, V4 = V / 64;
  UN_CUDA(launch_unet_loss_bwd(st, a->out, target, type, a->d1, net->hp, alpha, k, a->g_d1, sx, sy, sz, a->le, a->l0,
                               a->l1, a->l2, a->l3, a->lg, a->lpart, a->lsums, a->hpart, net->hg));
  UN_CUDA(launch_relu_bwd(st, a->g_d1, a->d1, V * 16));
  UN_TRY(conv_bwd(net, st, a, 9, a->d1a, a->g_d1, a->g_d1a, sx, sy, sz));
  UN_CUDA(launch_relu_bwd(st, a->g_d1a, a->d1a, V * 16));
  UN_TRY(conv_bwd(net, st, a, 8, a->u1, a->g_d1a, a->g_u1, sx, sy, sz));
  UN_CUDA(launch_upcat_bwd(st, a->g_u1, a->g_d2, a->g_e1, sx, sy, sz, 32, 16));
  UN_CUDA(launch_relu_bwd(st, a->g_d2, a->d2, V2 * 32));
  UN_TRY(conv_bwd(net, st, a, 7, a->d2a, a->g_d2, a->g_d2a, hx, hy, hz));
  UN_CUDA(launch_relu_bwd(st, a->g_d2a, a->d2a, V2 * 32));
  UN_TRY(conv_bwd(net, st, a, 6, a->u2, a->g_d2a, a->g_u2, hx, hy, hz));
  UN_CUDA(launch_upcat_bwd(st, a->g_u2, a->g_b2, a->g_e2, hx, hy, hz, 64, 32));
  UN_CUDA(launch_relu_bwd(st, a->g_b2, a->b2, V4 * 64));
  UN_TRY(conv_bwd(net, st, a, 5, a->b1, a->g_b2, a->g_b1, qx, qy, qz));
  UN_CUDA(launch_relu_bwd(st, a->g_b1, a->b1, V4 * 64));
  UN_TRY(conv_bwd(net, st, a, 4, a->p2, a->g_b1, a->g_p2, qx, qy, qz));
  UN_CUDA(launch_pool2_bwd(st, a->g_p2, a->g_e2, hx, hy, hz, 32, true));
  UN_CUDA(launch_relu_bwd(st, a->g_e2, a->e2, V2 * 32));
  UN_TRY(conv_bwd(net, st, a, 3, a->e2a, a->g_e2, a->g_e2a, hx, hy, hz));
  UN_CUDA(launch_relu_bwd(st, a->g_e2a, a->e2a, V2 * 32));
  UN_TRY(conv_bwd(net, st, a, 2, a->p1, a->g_e2a, a->g_p1, hx, hy, hz));
  UN_CUDA(launch_pool2_bwd(st, a->g_p1, a->g_e1, sx, sy, sz, 16, true));
  UN_CUDA(launch_relu_bwd(st, a->g_e1, a->e1, V * 16));
  UN_TRY(conv_bwd(net, st, a, 1, a->e1a, a->g_e1, a->g_e1a, sx, sy, sz));
  UN_CUDA(launch_relu_bwd(st, a->g_e1a, a->e1a, V * 16));
  UN_TRY(conv_bwd(net, st, a, 0, a->in0, a->g_e1a, nullptr, sx, sy, sz));
  return AQ_OK;
}

aq_status adam_step(aq_unet* net, cudaStream_t st, float lr) {
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  const int t = ++net->adam_t;
  for (UConv& c : net->L) {
    UN_CUDA(launch_adam(st, c.w, c.g, c.m, c.v, c.nw(), lr, b1, b2, eps, t, c.wb));
    UN_CUDA(launch_adam(st, c.b, c.gb, c.mb, c.vb, c.cout, lr, b1, b2, eps, t, nullptr));
    UN_CUDA(launch_flip_transpose(st, c.wb, c.wt, c.cin, c.cout));
  }
  // head: hg holds [dw 16, db, loss]; the first 17 are the gradient
  UN_CUDA(launch_adam(st, net->hp, net->hg, net->hm, net->hv, 17, lr, b1, b2, eps, t, nullptr));
  return AQ_OK;
}

}  // namespace

aq_status aqb::unet_predict(aq_unet* net, cudaStream_t st, UActs* a, const float* rhs, const int8_t* type, float* p) {
  const int V = a->sx * a->sy * a->sz;
  UN_CUDA(launch_absmax(st, rhs, V, net->absmax_part, net->scale));
  UN_CUDA(launch_unet_input(st, rhs, type, net->scale, a->in0, V));
  UN_TRY(forward(net, st, a));
  UN_CUDA(launch_unet_to_pressure(st, a->out, net->scale, net->out_scale, type, p, V));
  return AQ_OK;
}

// ================================================================= dataset
struct aq_dataset {
  int device = 0;
  int sx = 0, sy = 0, sz = 0, cap = 0, n = 0;
  float* rhs = nullptr;     // [cap][V] rhs / max|rhs|
  int8_t* type = nullptr;   // [cap][V]
  float* target = nullptr;  // [cap][V] FP64-PCG pressure / max|rhs| (f32)
  float* scratch = nullptr;  // absmax parts + scale
  std::vector<void*> allocs;
  ~aq_dataset() {
    cudaSetDevice(device);
    cudaDeviceSynchronize();
    for (void* p : allocs) cudaFree(p);
  }
};

extern "C" {

// ----------------------------------------------------------- building blocks
aq_status aq_conv3_forward(int32_t cin, int32_t cout, int32_t relu, const void* in, const void* w, const float* bias,
                           void* out, int32_t sx, int32_t sy, int32_t sz, void* stream) {
  if (!in || !w || !out || sx < 1 || sy < 1 || sz < 1) return fail(AQ_ERR_INVALID_ARGUMENT, "bad argument");
  UN_CUDA(launch_conv3_fwd((cudaStream_t)stream, cin, cout, relu != 0, in, w, bias, out, sx, sy, sz));
  return AQ_OK;
}

aq_status aq_conv3_weight_grad(int32_t cin, int32_t cout, const void* x, const void* dy, float* dw, int32_t sx,
                               int32_t sy, int32_t sz, void* stream) {
  if (!x || !dy || !dw || sx < 1 || sy < 1 || sz < 1) return fail(AQ_ERR_INVALID_ARGUMENT, "bad argument");
  float* part = nullptr;
  const size_t n = conv3_wgrad_part_floats(cin, cout, sx * sy * sz);
  UN_CUDA(cudaMallocAsync((void**)&part, n * sizeof(float), (cudaStream_t)stream));
  const cudaError_t e = launch_conv3_wgrad((cudaStream_t)stream, cin, cout, x, dy, part, dw, sx, sy, sz);
  cudaFreeAsync(part, (cudaStream_t)stream);
  UN_CUDA(e);
  return AQ_OK;
}

aq_status aq_conv3_set_tiled(int32_t tiled) {
  if (tiled < 0 || tiled > 2) return fail(AQ_ERR_INVALID_ARGUMENT, "conv variant must be 0, 1 or 2");
  set_conv_impl(tiled);
  return AQ_OK;
}

aq_status aq_conv3_umma_status(int32_t* timeouts) {
  if (!timeouts) return fail(AQ_ERR_INVALID_ARGUMENT, "NULL");
  *timeouts = conv_umma_timeouts();
  return AQ_OK;
}

aq_status aq_conv3_test_wait_timeout(int32_t skip_mma, uint64_t wait_ns) {
  if (skip_mma != 0 && skip_mma != 1) return fail(AQ_ERR_INVALID_ARGUMENT, "skip_mma must be 0 or 1");
  UN_CUDA(cudaDeviceSynchronize());
  UN_CUDA(conv_umma_test_hook(skip_mma, (unsigned long long)wait_ns));
  return AQ_OK;
}

aq_status aq_conv3_flip_transpose(int32_t cin, int32_t cout, const void* w, void* wt, void* stream) {
  if (!w || !wt) return fail(AQ_ERR_INVALID_ARGUMENT, "bad argument");
  UN_CUDA(launch_flip_transpose((cudaStream_t)stream, w, wt, cin, cout));
  return AQ_OK;
}

// ------------------------------------------------------------------ network
aq_status aq_unet_create(int32_t device, uint32_t seed, aq_unet** out) {
  if (!out) return fail(AQ_ERR_INVALID_ARGUMENT, "out is NULL");
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return fail(AQ_ERR_NO_DEVICE, "no CUDA device");
  }
  if (device < 0 || device >= ndev) return fail(AQ_ERR_INVALID_ARGUMENT, "device ordinal out of range");
  aq_unet* net = new aq_unet();
  net->device = device;
  auto bail = [&](aq_status st) {
    delete net;
    return st;
  };
  if (cudaSetDevice(device) != cudaSuccess) return bail(fail(AQ_ERR_CUDA, "cudaSetDevice"));
  if (cudaStreamCreateWithFlags(&net->stream, cudaStreamNonBlocking) != cudaSuccess)
    return bail(fail(AQ_ERR_CUDA, "cudaStreamCreate"));
  net->own_stream = true;
  // He-normal weights from a seeded host generator (input layer: 2 live channels)
  std::mt19937 rng(seed);
  std::normal_distribution<float> nd(0.f, 1.f);
  cudaStream_t st = net->stream;
  for (int l = 0; l < 10; ++l) {
    UConv& c = net->L[l];
    c.cin = kLayerIO[l][0];
    c.cout = kLayerIO[l][1];
    const int n = c.nw();
    aq_status s;
    if ((s = dalloc(net->allocs, &c.w, n, st)) != AQ_OK || (s = dalloc(net->allocs, &c.g, n, st)) != AQ_OK ||
        (s = dalloc(net->allocs, &c.m, n, st)) != AQ_OK || (s = dalloc(net->allocs, &c.v, n, st)) != AQ_OK ||
        (s = dalloc(net->allocs, &c.b, c.cout, st)) != AQ_OK || (s = dalloc(net->allocs, &c.gb, c.cout, st)) != AQ_OK ||
        (s = dalloc(net->allocs, &c.mb, c.cout, st)) != AQ_OK || (s = dalloc(net->allocs, &c.vb, c.cout, st)) != AQ_OK ||
        (s = dalloc(net->allocs, &c.wb, n, st)) != AQ_OK || (s = dalloc(net->allocs, &c.wt, n, st)) != AQ_OK)
      return bail(s);
    const int fan_in = 27 * (l == 0 ? 2 : c.cin);
    const float sd = sqrtf(2.f / (float)fan_in);
    std::vector<float> h(n);
    for (int i = 0; i < n; ++i) h[i] = nd(rng) * sd;
    if (l == 0)  // padding input channels carry nothing
      for (int i = 0; i < n; ++i)
        if (i % c.cin >= 2) h[i] = 0.f;
    if (cudaMemcpy(c.w, h.data(), sizeof(float) * n, cudaMemcpyHostToDevice) != cudaSuccess)
      return bail(fail(AQ_ERR_CUDA, "weight upload"));
  }
  aq_status s;
  if ((s = dalloc(net->allocs, &net->hp, 17, st)) != AQ_OK || (s = dalloc(net->allocs, &net->hg, 18, st)) != AQ_OK ||
      (s = dalloc(net->allocs, &net->hm, 17, st)) != AQ_OK || (s = dalloc(net->allocs, &net->hv, 17, st)) != AQ_OK ||
      (s = dalloc(net->allocs, &net->absmax_part, 1024, st)) != AQ_OK ||
      (s = dalloc(net->allocs, &net->scale, 1, st)) != AQ_OK)
    return bail(s);
  std::vector<float> hh(17, 0.f);
  for (int i = 0; i < 16; ++i) hh[i] = nd(rng) * 0.25f;
  if (cudaMemcpy(net->hp, hh.data(), sizeof(float) * 17, cudaMemcpyHostToDevice) != cudaSuccess)
    return bail(fail(AQ_ERR_CUDA, "head upload"));
  if ((s = refresh_bf16(net)) != AQ_OK) return bail(s);
  if (cudaStreamSynchronize(st) != cudaSuccess) return bail(fail(AQ_ERR_CUDA, "network initialisation"));
  *out = net;
  return AQ_OK;
}

void aq_unet_destroy(aq_unet* net) { delete net; }

aq_status aq_unet_parameter_count(const aq_unet* net, int64_t* count) {
  if (!net || !count) return fail(AQ_ERR_INVALID_ARGUMENT, "bad argument");
  int64_t n = 17;
  for (const UConv& c : net->L) n += c.nw() + c.cout;
  *count = n;
  return AQ_OK;
}

aq_status aq_unet_save(aq_unet* net, const char* path) {
  if (!net || !path) return fail(AQ_ERR_INVALID_ARGUMENT, "bad argument");
  cudaSetDevice(net->device);
  UN_CUDA(cudaStreamSynchronize(net->stream));
  FILE* fp = fopen(path, "wb");
  if (!fp) return fail(AQ_ERR_INVALID_ARGUMENT, std::string("cannot write ") + path);
  bool ok = fwrite(&kMagic, 4, 1, fp) == 1 && fwrite(&kVersion, 4, 1, fp) == 1 &&
            fwrite(&net->out_scale, 4, 1, fp) == 1;
  for (const UConv& c : net->L) {
    std::vector<float> h((size_t)c.nw() + c.cout);
    ok = ok && cudaMemcpy(h.data(), c.w, sizeof(float) * c.nw(), cudaMemcpyDeviceToHost) == cudaSuccess &&
         cudaMemcpy(h.data() + c.nw(), c.b, sizeof(float) * c.cout, cudaMemcpyDeviceToHost) == cudaSuccess;
    const int32_t io[2] = {c.cin, c.cout};
    ok = ok && fwrite(io, 4, 2, fp) == 2 && fwrite(h.data(), 4, h.size(), fp) == h.size();
  }
  std::vector<float> hh(17);
  ok = ok && cudaMemcpy(hh.data(), net->hp, sizeof(float) * 17, cudaMemcpyDeviceToHost) == cudaSuccess &&
       fwrite(hh.data(), 4, 17, fp) == 17;
  ok = fclose(fp) == 0 && ok;
  if (!ok) return fail(AQ_ERR_CUDA, std::string("writing ") + path + " failed");
  return AQ_OK;
}

aq_status aq_unet_load(aq_unet* net, const char* path) {
  if (!net || !path) return fail(AQ_ERR_INVALID_ARGUMENT, "bad argument");
  cudaSetDevice(net->device);
  FILE* fp = fopen(path, "rb");
  if (!fp) return fail(AQ_ERR_INVALID_ARGUMENT, std::string("cannot read ") + path);
  uint32_t magic = 0, version = 0;
  float scale = 1.f;
  bool ok = fread(&magic, 4, 1, fp) == 1 && fread(&version, 4, 1, fp) == 1 && fread(&scale, 4, 1, fp) == 1 &&
            magic == kMagic && version == kVersion;
  std::vector<std::vector<float>> ws(10);
  for (int l = 0; l < 10 && ok; ++l) {
    int32_t io[2];
    ok = fread(io, 4, 2, fp) == 2 && io[0] == net->L[l].cin && io[1] == net->L[l].cout;
    ws[l].resize((size_t)net->L[l].nw() + net->L[l].cout);
    ok = ok && fread(ws[l].data(), 4, ws[l].size(), fp) == ws[l].size();
  }
  std::vector<float> hh(17);
  ok = ok && fread(hh.data(), 4, 17, fp) == 17;
  fclose(fp);
  if (!ok) return fail(AQ_ERR_INVALID_ARGUMENT, std::string(path) + " is not a weights file of this network");
  UN_CUDA(cudaStreamSynchronize(net->stream));
  for (int l = 0; l < 10; ++l) {
    UConv& c = net->L[l];
    UN_CUDA(cudaMemcpy(c.w, ws[l].data(), sizeof(float) * c.nw(), cudaMemcpyHostToDevice));
    UN_CUDA(cudaMemcpy(c.b, ws[l].data() + c.nw(), sizeof(float) * c.cout, cudaMemcpyHostToDevice));
    UN_CUDA(cudaMemset(c.m, 0, sizeof(float) * c.nw()));
    UN_CUDA(cudaMemset(c.v, 0, sizeof(float) * c.nw()));
  }
  UN_CUDA(cudaMemcpy(net->hp, hh.data(), sizeof(float) * 17, cudaMemcpyHostToDevice));
  net->out_scale = scale;
  net->adam_t = 0;
  UN_TRY(refresh_bf16(net));
  UN_CUDA(cudaStreamSynchronize(net->stream));
  return AQ_OK;
}

aq_status aq_unet_get_output_scale(const aq_unet* net, float* scale) {
  if (!net || !scale) return fail(AQ_ERR_INVALID_ARGUMENT, "bad argument");
  *scale = net->out_scale;
  return AQ_OK;
}

// ------------------------------------------------------------------ dataset
aq_status aq_dataset_create(int32_t sx, int32_t sy, int32_t sz, int32_t capacity, int32_t device, aq_dataset** out) {
  if (!out || capacity < 1 || sx % 4 || sy % 4 || sz % 4 || sx < 4 || sy < 4 || sz < 4)
    return fail(AQ_ERR_INVALID_ARGUMENT, "bad argument (sizes must be divisible by 4)");
  *out = nullptr;
  aq_dataset* ds = new aq_dataset();
  ds->device = device;
  ds->sx = sx; ds->sy = sy; ds->sz = sz; ds->cap = capacity;
  if (cudaSetDevice(device) != cudaSuccess) {
    delete ds;
    return fail(AQ_ERR_NO_DEVICE, "cudaSetDevice");
  }
  const size_t V = (size_t)sx * sy * sz, n = V * capacity;
  aq_status s;
  if ((s = dalloc(ds->allocs, &ds->rhs, n, nullptr)) != AQ_OK || (s = dalloc(ds->allocs, &ds->type, n, nullptr)) != AQ_OK ||
      (s = dalloc(ds->allocs, &ds->target, n, nullptr)) != AQ_OK ||
      (s = dalloc(ds->allocs, &ds->scratch, 1025, nullptr)) != AQ_OK) {
    delete ds;
    return s;
  }
  cudaDeviceSynchronize();
  *out = ds;
  return AQ_OK;
}

void aq_dataset_destroy(aq_dataset* ds) { delete ds; }

int32_t aq_dataset_count(const aq_dataset* ds) { return ds ? ds->n : 0; }

aq_status aq_dataset_add_fluid(aq_dataset* ds, aq_fluid* f, double pcg_rel_tol, int32_t pcg_max_iter,
                               int32_t* pcg_iterations) {
  if (!ds || !f) return fail(AQ_ERR_INVALID_ARGUMENT, "bad argument");
  if (f->d.sx != ds->sx || f->d.sy != ds->sy || f->d.sz != ds->sz)
    return fail(AQ_ERR_INVALID_ARGUMENT, "fluid grid size differs from the dataset's");
  if (ds->n >= ds->cap) return fail(AQ_ERR_INVALID_ARGUMENT, "dataset is full");
  cudaSetDevice(f->device);
  int it = 0;
  double ach = 0.0;
  UN_TRY(fluid_pcg_solve(f, pcg_rel_tol, pcg_max_iter, &it, &ach));
  if (pcg_iterations) *pcg_iterations = it;
  const int V = f->d.C;
  const size_t o = (size_t)ds->n * V;
  UN_CUDA(launch_absmax(f->stream, f->rhs, V, ds->scratch, ds->scratch + 1024));
  UN_CUDA(launch_unet_sample(f->stream, f->rhs, f->type, f->pcg_x, ds->scratch + 1024, ds->rhs + o, ds->type + o,
                             ds->target + o, V));
  UN_CUDA(cudaStreamSynchronize(f->stream));
  ds->n += 1;
  return AQ_OK;
}

aq_status aq_dataset_get(aq_dataset* ds, int32_t i, float* rhs, int8_t* type, float* target) {
  if (!ds || i < 0 || i >= ds->n) return fail(AQ_ERR_INVALID_ARGUMENT, "bad sample index");
  cudaSetDevice(ds->device);
  const size_t V = (size_t)ds->sx * ds->sy * ds->sz, o = (size_t)i * V;
  if (rhs) UN_CUDA(cudaMemcpy(rhs, ds->rhs + o, 4 * V, cudaMemcpyDeviceToHost));
  if (type) UN_CUDA(cudaMemcpy(type, ds->type + o, V, cudaMemcpyDeviceToHost));
  if (target) UN_CUDA(cudaMemcpy(target, ds->target + o, 4 * V, cudaMemcpyDeviceToHost));
  return AQ_OK;
}

// RMS of the targets over fluid cells of samples [first, first+count).
aq_status aq_dataset_target_rms(aq_dataset* ds, int32_t first, int32_t count, double* rms) {
  if (!ds || !rms || first < 0 || count < 1 || first + count > ds->n) return fail(AQ_ERR_INVALID_ARGUMENT, "bad range");
  cudaSetDevice(ds->device);
  const size_t V = (size_t)ds->sx * ds->sy * ds->sz;
  std::vector<float> t(V);
  std::vector<int8_t> ty(V);
  double ss = 0.0, nn = 0.0;
  for (int i = first; i < first + count; ++i) {
    UN_CUDA(cudaMemcpy(t.data(), ds->target + i * V, 4 * V, cudaMemcpyDeviceToHost));
    UN_CUDA(cudaMemcpy(ty.data(), ds->type + i * V, V, cudaMemcpyDeviceToHost));
    for (size_t v = 0; v < V; ++v)
      if (ty[v] == kFluid) {
        ss += (double)t[v] * t[v];
        nn += 1.0;
      }
  }
  *rms = nn > 0 ? sqrt(ss / nn) : 0.0;
  return AQ_OK;
}

// ----------------------------------------------------------------- training
// `steps` Adam steps on samples drawn (seeded) from [first, first+count);
// targets are divided by out_scale (set here if out_scale <= 0: the targets'
// RMS).  mean_loss: mean loss over the last tenth of the steps.
aq_status aq_unet_train(aq_unet* net, aq_dataset* ds, int32_t first, int32_t count, int32_t steps, float lr,
                        uint32_t seed, float out_scale, float residual_weight, int32_t residual_sweeps,
                        float* mean_loss) {
  if (!net || !ds || first < 0 || count < 1 || first + count > ds->n || steps < 1 || residual_sweeps < 0 ||
      residual_sweeps > 1000)
    return fail(AQ_ERR_INVALID_ARGUMENT, "bad argument");
  cudaSetDevice(net->device);
  if (out_scale <= 0.f) {
    double rms = 0.0;
    UN_TRY(aq_dataset_target_rms(ds, first, count, &rms));
    out_scale = rms > 0 ? (float)rms : 1.f;
  }
  net->out_scale = out_scale;
  UActs* a = nullptr;
  UN_TRY(unet_acts(net, ds->sx, ds->sy, ds->sz, true, &a));
  const int V = ds->sx * ds->sy * ds->sz;
  cudaStream_t st = net->stream;
  float* tgt = nullptr;  // scaled target of the current sample
  UN_CUDA(cudaMallocAsync((void**)&tgt, sizeof(float) * V, st));
  float* losses = nullptr;
  UN_CUDA(cudaMallocAsync((void**)&losses, sizeof(float) * steps, st));
  float* one = nullptr;
  UN_CUDA(cudaMallocAsync((void**)&one, sizeof(float), st));
  const float h_one = 1.f;
  UN_CUDA(cudaMemcpyAsync(one, &h_one, sizeof(float), cudaMemcpyHostToDevice, st));
  std::mt19937 rng(seed);
  aq_status status = AQ_OK;
  for (int s = 0; s < steps && status == AQ_OK; ++s) {
    const int i = first + (int)(rng() % (uint32_t)count);
    const size_t o = (size_t)i * V;
    // input from the stored scaled rhs (scale 1), target / out_scale
    if (launch_unet_input(st, ds->rhs + o, ds->type + o, one, a->in0, V) != cudaSuccess ||
        launch_unet_scale_copy(st, ds->target + o, 1.f / out_scale, tgt, V) != cudaSuccess) {
      status = fail(AQ_ERR_CUDA, "training step setup");
      break;
    }
    // cosine learning-rate decay to 5% of lr
    const float lr_s = lr * (0.05f + 0.95f * 0.5f * (1.f + cosf(3.14159265f * (float)s / (float)steps)));
    if ((status = forward(net, st, a)) != AQ_OK) break;
    if ((status = backward(net, st, a, tgt, ds->type + o, residual_weight, residual_sweeps)) != AQ_OK) break;
    if ((status = adam_step(net, st, lr_s)) != AQ_OK) break;
    if (cudaMemcpyAsync(losses + s, net->hg + 17, sizeof(float), cudaMemcpyDeviceToDevice, st) != cudaSuccess)
      status = fail(AQ_ERR_CUDA, "loss copy");
    if (s % 64 == 63) cudaStreamSynchronize(st);  // bound the host-side queue
  }
  std::vector<float> h((size_t)steps);
  if (status == AQ_OK) {
    UN_CUDA(cudaMemcpyAsync(h.data(), losses, sizeof(float) * steps, cudaMemcpyDeviceToHost, st));
  }
  cudaFreeAsync(tgt, st);
  cudaFreeAsync(losses, st);
  cudaFreeAsync(one, st);
  UN_CUDA(cudaStreamSynchronize(st));
  if (status != AQ_OK) return status;
  if (mean_loss) {
    const int k0 = steps - std::max(1, steps / 10);
    double acc = 0.0;
    for (int s = k0; s < steps; ++s) acc += h[s];
    *mean_loss = (float)(acc / (steps - k0));
  }
  return AQ_OK;
}

// Mean over samples of the relative L2 error of the predicted pressure
// against the FP64-PCG target, over fluid cells.
aq_status aq_unet_evaluate(aq_unet* net, aq_dataset* ds, int32_t first, int32_t count, double* mean_rel_error) {
  if (!net || !ds || !mean_rel_error || first < 0 || count < 1 || first + count > ds->n)
    return fail(AQ_ERR_INVALID_ARGUMENT, "bad argument");
  cudaSetDevice(net->device);
  UActs* a = nullptr;
  UN_TRY(unet_acts(net, ds->sx, ds->sy, ds->sz, false, &a));
  const size_t V = (size_t)ds->sx * ds->sy * ds->sz;
  cudaStream_t st = net->stream;
  float* p = nullptr;
  UN_CUDA(cudaMallocAsync((void**)&p, sizeof(float) * V, st));
  std::vector<float> hp(V), ht(V);
  std::vector<int8_t> ty(V);
  double acc = 0.0;
  aq_status status = AQ_OK;
  for (int i = first; i < first + count && status == AQ_OK; ++i) {
    const size_t o = (size_t)i * V;
    // rhs is stored scaled (max-abs 1): the prediction is the scaled pressure
    if ((status = unet_predict(net, st, a, ds->rhs + o, ds->type + o, p)) != AQ_OK) break;
    if (cudaMemcpyAsync(hp.data(), p, 4 * V, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaMemcpyAsync(ht.data(), ds->target + o, 4 * V, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaMemcpyAsync(ty.data(), ds->type + o, V, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess) {
      status = fail(AQ_ERR_CUDA, "evaluation copy");
      break;
    }
    double num = 0.0, den = 0.0;
    for (size_t v = 0; v < V; ++v)
      if (ty[v] == kFluid) {
        const double e = (double)hp[v] - ht[v];
        num += e * e;
        den += (double)ht[v] * ht[v];
      }
    acc += den > 0 ? sqrt(num / den) : 0.0;
  }
  cudaFreeAsync(p, st);
  UN_CUDA(cudaStreamSynchronize(st));
  if (status != AQ_OK) return status;
  *mean_rel_error = acc / count;
  return AQ_OK;
}

// Mean over samples of (residual after `sweeps` Jacobi sweeps from the
// prediction) / (the same from zero), the ratio the warm start's fallback
// rule compares: below 1 the prediction is kept.
aq_status aq_unet_evaluate_warm(aq_unet* net, aq_dataset* ds, int32_t first, int32_t count, int32_t sweeps,
                                double* mean_ratio) {
  if (!net || !ds || !mean_ratio || first < 0 || count < 1 || first + count > ds->n || sweeps < 0 || sweeps > 1000)
    return fail(AQ_ERR_INVALID_ARGUMENT, "bad argument");
  cudaSetDevice(net->device);
  UActs* a = nullptr;
  UN_TRY(unet_acts(net, ds->sx, ds->sy, ds->sz, true, &a));
  const int sx = ds->sx, sy = ds->sy, sz = ds->sz;
  const size_t V = (size_t)sx * sy * sz;
  cudaStream_t st = net->stream;
  float* p = nullptr;
  UN_CUDA(cudaMallocAsync((void**)&p, sizeof(float) * V, st));
  double acc = 0.0;
  aq_status status = AQ_OK;
  for (int i = first; i < first + count && status == AQ_OK; ++i) {
    const size_t o = (size_t)i * V;
    // rhs is stored scaled (max-abs 1): p is in the targets' units
    if ((status = unet_predict(net, st, a, ds->rhs + o, ds->type + o, p)) != AQ_OK) break;
    float sums[6];
    if (launch_unet_loss_bwd(st, p, ds->target + o, ds->type + o, a->d1, net->hp, 1.f, sweeps, a->g_d1, sx, sy, sz,
                             a->le, a->l0, a->l1, a->l2, a->l3, a->lg, a->lpart, a->lsums, a->hpart,
                             net->hg) != cudaSuccess ||
        cudaMemcpyAsync(sums, a->lsums, sizeof(sums), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess) {
      status = fail(AQ_ERR_CUDA, "warm-start evaluation");
      break;
    }
    acc += sums[3] > 0.f ? sqrt((double)sums[2] / (double)sums[3]) : 0.0;
  }
  cudaFreeAsync(p, st);
  UN_CUDA(cudaStreamSynchronize(st));
  if (status != AQ_OK) return status;
  *mean_ratio = acc / count;
  return AQ_OK;
}

aq_status aq_unet_set_output_scale(aq_unet* net, float scale) {
  if (!net || !(scale > 0.f)) return fail(AQ_ERR_INVALID_ARGUMENT, "scale must be > 0");
  net->out_scale = scale;
  return AQ_OK;
}

aq_status aq_unet_gradients(aq_unet* net, float* out, int64_t n) {
  int64_t total = 0;
  UN_TRY(aq_unet_parameter_count(net, &total));
  if (!out || n != total) return fail(AQ_ERR_INVALID_ARGUMENT, "output must hold parameter_count floats");
  cudaSetDevice(net->device);
  UN_CUDA(cudaStreamSynchronize(net->stream));
  size_t o = 0;
  for (const UConv& c : net->L) {
    UN_CUDA(cudaMemcpy(out + o, c.g, sizeof(float) * c.nw(), cudaMemcpyDeviceToHost));
    o += c.nw();
    UN_CUDA(cudaMemcpy(out + o, c.gb, sizeof(float) * c.cout, cudaMemcpyDeviceToHost));
    o += c.cout;
  }
  UN_CUDA(cudaMemcpy(out + o, net->hg, sizeof(float) * 17, cudaMemcpyDeviceToHost));
  return AQ_OK;
}

// Forward pass on caller buffers: p = warm-start pressure for (rhs, type).
aq_status aq_unet_predict(aq_unet* net, int32_t sx, int32_t sy, int32_t sz, const float* rhs, const int8_t* type,
                          float* pressure, void* stream) {
  if (!net || !rhs || !type || !pressure) return fail(AQ_ERR_INVALID_ARGUMENT, "bad argument");
  cudaSetDevice(net->device);
  UActs* a = nullptr;
  UN_TRY(unet_acts(net, sx, sy, sz, false, &a));
  cudaStream_t st = stream ? (cudaStream_t)stream : net->stream;
  UN_CUDA(cudaStreamSynchronize(net->stream));
  UN_TRY(unet_predict(net, st, a, rhs, type, pressure));
  return AQ_OK;
}

}  // extern "C"
