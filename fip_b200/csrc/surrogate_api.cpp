// C ABI of the surrogate kernels (include/fip_surrogate.h).
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "fip.h"
#include "fip_surrogate.h"
#include "surrogate.h"

namespace fip {
void set_last_error(const std::string& msg);
}

namespace {

int sg_fail(int code, const std::string& m) {
  fip::set_last_error(m);
  return code;
}

int sg_cuda(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return FIP_OK;
  return sg_fail(FIP_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

std::mutex g_part_mu;
float* g_part[64] = {};

}  // namespace

extern "C" {

int fip_sg_conv3x3(const void* in, const void* w, const float* bias, const void* res, const void* mask, void* out,
                   int N, int H, int W, int epi, int* dev_err, void* stream) {
  if (!in || !w || !out || N <= 0 || H <= 0 || W <= 0) return sg_fail(FIP_ERR_ARG, "fip_sg_conv3x3: bad argument");
  if (epi < FIP_SG_EPI_BIAS_RELU || epi > FIP_SG_EPI_PLAIN) return sg_fail(FIP_ERR_ARG, "fip_sg_conv3x3: unknown epilogue");
  if ((epi == FIP_SG_EPI_BIAS_RES_RELU || epi == FIP_SG_EPI_RES_MASK) && !res)
    return sg_fail(FIP_ERR_ARG, "fip_sg_conv3x3: this epilogue needs res");
  if ((epi == FIP_SG_EPI_MASK || epi == FIP_SG_EPI_RES_MASK) && !mask)
    return sg_fail(FIP_ERR_ARG, "fip_sg_conv3x3: this epilogue needs mask");
  if ((reinterpret_cast<uintptr_t>(in) | reinterpret_cast<uintptr_t>(w) | reinterpret_cast<uintptr_t>(out)) & 15u)
    return sg_fail(FIP_ERR_ARG, "fip_sg_conv3x3: tensors must be 16-byte aligned");
  if ((long long)N * (H + 2) * (W + 2) >= (1LL << 31)) return sg_fail(FIP_ERR_ARG, "fip_sg_conv3x3: too many pixels");
  fip::sg::ConvShape s{N, H, W};
  return sg_cuda(fip::sg::conv3x3(s, static_cast<const __nv_bfloat16*>(in), static_cast<const __nv_bfloat16*>(w), bias,
                                  static_cast<const __nv_bfloat16*>(res), static_cast<const __nv_bfloat16*>(mask), out, epi,
                                  dev_err, static_cast<cudaStream_t>(stream)),
                 "fip_sg_conv3x3");
}

int fip_sg_conv3x3_wgrad(const void* x, const void* dy, float* dw, int N, int H, int W, int* dev_err, void* stream) {
  if (!x || !dy || !dw || N <= 0 || H <= 0 || W <= 0) return sg_fail(FIP_ERR_ARG, "fip_sg_conv3x3_wgrad: bad argument");
  if ((reinterpret_cast<uintptr_t>(x) | reinterpret_cast<uintptr_t>(dy)) & 15u)
    return sg_fail(FIP_ERR_ARG, "fip_sg_conv3x3_wgrad: tensors must be 16-byte aligned");
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64) return sg_fail(FIP_ERR_ARG, "device ordinal");
  float* part = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_part_mu);
    if (!g_part[dev]) {
      const int rc = sg_cuda(cudaMalloc((void**)&g_part[dev], fip::sg::wgrad_scratch_floats() * sizeof(float)),
                             "fip_sg_conv3x3_wgrad scratch");
      if (rc) return rc;
    }
    part = g_part[dev];
  }
  fip::sg::ConvShape s{N, H, W};
  return sg_cuda(fip::sg::conv3x3_wgrad(s, static_cast<const __nv_bfloat16*>(x), static_cast<const __nv_bfloat16*>(dy),
                                        part, dw, dev_err, static_cast<cudaStream_t>(stream)),
                 "fip_sg_conv3x3_wgrad");
}

}  // extern "C"
