// The learned warm start's network object (aq_unet), shared by its host code
// (unet.cu) and the fluid step that runs it (fluid.cu).
#pragma once

#include <cuda_bf16.h>

#include <vector>

#include "../../include/aquarius_b200.h"
#include "aq_kernels.cuh"

namespace aqb {

// One 3x3x3 convolution: f32 master weights [27][cout][cin] and bias, their
// gradients and Adam moments, the bf16 copy the forward kernel reads and the
// flipped transpose the data gradient reads.
struct UConv {
  int cin = 0, cout = 0;
  float *w = nullptr, *g = nullptr, *m = nullptr, *v = nullptr;
  float *b = nullptr, *gb = nullptr, *mb = nullptr, *vb = nullptr;
  __nv_bfloat16 *wb = nullptr, *wt = nullptr;
  int nw() const { return 27 * cin * cout; }
};

// Activations and their gradients for one grid size (all sizes % 4 == 0).
struct UActs {
  int sx = 0, sy = 0, sz = 0;
  __nv_bfloat16 *in0 = nullptr, *e1a = nullptr, *e1 = nullptr, *p1 = nullptr, *e2a = nullptr, *e2 = nullptr,
                *p2 = nullptr, *b1 = nullptr, *b2 = nullptr, *u2 = nullptr, *d2a = nullptr, *d2 = nullptr,
                *u1 = nullptr, *d1a = nullptr, *d1 = nullptr;
  __nv_bfloat16 *g_e1a = nullptr, *g_e1 = nullptr, *g_p1 = nullptr, *g_e2a = nullptr, *g_e2 = nullptr,
                *g_p2 = nullptr, *g_b1 = nullptr, *g_b2 = nullptr, *g_u2 = nullptr, *g_d2a = nullptr,
                *g_d2 = nullptr, *g_u1 = nullptr, *g_d1a = nullptr, *g_d1 = nullptr;
  float* out = nullptr;
  float* wpart = nullptr;  // weight-gradient partial sums (largest layer)
  float* cpart = nullptr;  // channel-sum partials
  // training loss scratch: error, four work buffers, output gradient (V each)
  float *le = nullptr, *l0 = nullptr, *l1 = nullptr, *l2 = nullptr, *l3 = nullptr, *lg = nullptr;
  float *lpart = nullptr, *lsums = nullptr, *hpart = nullptr;
  bool grads = false;
  std::vector<void*> allocs;
};

}  // namespace aqb

struct aq_unet {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  aqb::UConv L[10];
  // output head: 16 weights + 1 bias (one vector), gradient, moments
  float *hp = nullptr, *hg = nullptr, *hm = nullptr, *hv = nullptr;
  float out_scale = 1.f;  // network output x out_scale = pressure / max|rhs|
  int adam_t = 0;
  float *absmax_part = nullptr, *scale = nullptr;
  std::vector<aqb::UActs*> acts;
  std::vector<void*> allocs;
  ~aq_unet();
};

namespace aqb {
// Kernel launches of unet_predict: absmax 2, input 1, 10 convolutions, 2
// poolings, 2 upsample-concatenations, head 1, output 1.
constexpr int kUNetForwardLaunches = 19;
// Activations for a grid size (allocated once per size, before any capture).
aq_status unet_acts(aq_unet* net, int sx, int sy, int sz, bool grads, UActs** out);
// Enqueues the forward pass on `st`: p[v] = pressure warm start on fluid
// cells (0 elsewhere) for the system (rhs, type) of grid (sx,sy,sz).
aq_status unet_predict(aq_unet* net, cudaStream_t st, UActs* a, const float* rhs, const int8_t* type, float* p);
}  // namespace aqb
