// Host side of the learned pressure warm start (aq_unet_* in
// include/aquarius_b200.h).  No counterpart in the reference.
#include <cuda_bf16.h>

#include <string>
#include <vector>

#include "../../include/aquarius_b200.h"
#include "aq_kernels.cuh"

using namespace aqb;

namespace {

aq_status cuda_status(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return AQ_OK;
  return set_last_error(e == cudaErrorMemoryAllocation ? AQ_ERR_OUT_OF_MEMORY : AQ_ERR_CUDA,
                        std::string(what) + ": " + cudaGetErrorString(e));
}

}  // namespace

extern "C" {

aq_status aq_conv3_forward(int32_t cin, int32_t cout, int32_t relu, const void* in, const void* w, const float* bias,
                           void* out, int32_t sx, int32_t sy, int32_t sz, void* stream) {
  if (!in || !w || !out || sx < 1 || sy < 1 || sz < 1)
    return set_last_error(AQ_ERR_INVALID_ARGUMENT, "bad argument");
  return cuda_status(launch_conv3_fwd((cudaStream_t)stream, cin, cout, relu != 0, in, w, bias, out, sx, sy, sz),
                     "conv3 forward (unsupported channel pair?)");
}

aq_status aq_conv3_weight_grad(int32_t cin, int32_t cout, const void* x, const void* dy, float* dw, int32_t sx,
                               int32_t sy, int32_t sz, void* stream) {
  if (!x || !dy || !dw || sx < 1 || sy < 1 || sz < 1) return set_last_error(AQ_ERR_INVALID_ARGUMENT, "bad argument");
  float* part = nullptr;
  const size_t n = conv3_wgrad_part_floats(cin, cout, sx * sy * sz);
  aq_status st = cuda_status(cudaMallocAsync((void**)&part, n * sizeof(float), (cudaStream_t)stream), "alloc");
  if (st != AQ_OK) return st;
  st = cuda_status(launch_conv3_wgrad((cudaStream_t)stream, cin, cout, x, dy, part, dw, sx, sy, sz),
                   "conv3 weight grad (unsupported channel pair?)");
  cudaFreeAsync(part, (cudaStream_t)stream);
  return st;
}

aq_status aq_conv3_flip_transpose(int32_t cin, int32_t cout, const void* w, void* wt, void* stream) {
  if (!w || !wt) return set_last_error(AQ_ERR_INVALID_ARGUMENT, "bad argument");
  return cuda_status(launch_flip_transpose((cudaStream_t)stream, w, wt, cin, cout), "flip transpose");
}

}  // extern "C"
