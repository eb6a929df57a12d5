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
                   int N, int H, int W, int dilation, int epi, int* dev_err, void* stream) {
  if (!in || !w || !out || N <= 0 || H <= 0 || W <= 0) return sg_fail(FIP_ERR_ARG, "fip_sg_conv3x3: bad argument");
  if (epi < FIP_SG_EPI_BIAS_RELU || epi > FIP_SG_EPI_PLAIN) return sg_fail(FIP_ERR_ARG, "fip_sg_conv3x3: unknown epilogue");
  if ((epi == FIP_SG_EPI_BIAS_RES_RELU || epi == FIP_SG_EPI_RES_MASK) && !res)
    return sg_fail(FIP_ERR_ARG, "fip_sg_conv3x3: this epilogue needs res");
  if ((epi == FIP_SG_EPI_MASK || epi == FIP_SG_EPI_RES_MASK) && !mask)
    return sg_fail(FIP_ERR_ARG, "fip_sg_conv3x3: this epilogue needs mask");
  if ((reinterpret_cast<uintptr_t>(in) | reinterpret_cast<uintptr_t>(w) | reinterpret_cast<uintptr_t>(out) |
       reinterpret_cast<uintptr_t>(res) | reinterpret_cast<uintptr_t>(mask)) & 15u)
    return sg_fail(FIP_ERR_ARG, "fip_sg_conv3x3: tensors must be 16-byte aligned");
  if ((long long)N * (H + 2 * fip::sg::kPad) * (W + 2 * fip::sg::kPad) >= (1LL << 31))
    return sg_fail(FIP_ERR_ARG, "fip_sg_conv3x3: too many pixels");
  if (dilation < 1 || dilation > fip::sg::kMaxDil) return sg_fail(FIP_ERR_ARG, "fip_sg_conv3x3: dilation must be 1..8");
  fip::sg::ConvShape s{N, H, W, dilation};
  return sg_cuda(fip::sg::conv3x3(s, static_cast<const __nv_bfloat16*>(in), static_cast<const __nv_bfloat16*>(w), bias,
                                  static_cast<const __nv_bfloat16*>(res), static_cast<const __nv_bfloat16*>(mask), out, epi,
                                  dev_err, static_cast<cudaStream_t>(stream)),
                 "fip_sg_conv3x3");
}

int fip_sg_conv3x3_wgrad(const void* x, const void* dy, float* dw, int N, int H, int W, int dilation, int* dev_err,
                         void* stream) {
  if (!x || !dy || !dw || N <= 0 || H <= 0 || W <= 0) return sg_fail(FIP_ERR_ARG, "fip_sg_conv3x3_wgrad: bad argument");
  if ((reinterpret_cast<uintptr_t>(x) | reinterpret_cast<uintptr_t>(dy)) & 15u)
    return sg_fail(FIP_ERR_ARG, "fip_sg_conv3x3_wgrad: tensors must be 16-byte aligned");
  if ((long long)N * (H + 2 * fip::sg::kPad) * (W + 2 * fip::sg::kPad) >= (1LL << 31))
    return sg_fail(FIP_ERR_ARG, "fip_sg_conv3x3_wgrad: too many pixels");
  if (dilation < 1 || dilation > fip::sg::kMaxDil) return sg_fail(FIP_ERR_ARG, "fip_sg_conv3x3_wgrad: dilation must be 1..8");
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
  fip::sg::ConvShape s{N, H, W, dilation};
  return sg_cuda(fip::sg::conv3x3_wgrad(s, static_cast<const __nv_bfloat16*>(x), static_cast<const __nv_bfloat16*>(dy),
                                        part, dw, dev_err, static_cast<cudaStream_t>(stream)),
                 "fip_sg_conv3x3_wgrad");
}

#define SG_S static_cast<cudaStream_t>(stream)

int fip_sg_pack_input(const float* h, const float* qx, const float* qy, const float* terrain, const float* kst,
                      const float* zref, int N, int H, int W, float no_value, void* out, void* stream) {
  if (!h || !qx || !qy || !terrain || !kst || !zref || !out || N <= 0 || H <= 0 || W <= 0)
    return sg_fail(FIP_ERR_ARG, "fip_sg_pack_input: bad argument");
  if (reinterpret_cast<uintptr_t>(out) & 15u) return sg_fail(FIP_ERR_ARG, "fip_sg_pack_input: out must be 16-byte aligned");
  return sg_cuda(fip::sg::pack_input(h, qx, qy, terrain, kst, zref, N, H, W, no_value, static_cast<__nv_bfloat16*>(out),
                                     SG_S),
                 "fip_sg_pack_input");
}

int fip_sg_target(const float* h0, const float* qx0, const float* qy0, const float* h1, const float* qx1,
                  const float* qy1, const float* terrain, long long total, float no_value, float* tgt, void* stream) {
  if (!h0 || !qx0 || !qy0 || !h1 || !qx1 || !qy1 || !terrain || !tgt || total <= 0)
    return sg_fail(FIP_ERR_ARG, "fip_sg_target: bad argument");
  return sg_cuda(fip::sg::make_target(h0, qx0, qy0, h1, qx1, qy1, terrain, (size_t)total, no_value, tgt, SG_S),
                 "fip_sg_target");
}

int fip_sg_loss(const float* pred, const float* tgt, int N, int H, int W, float dx, float* scratch, void* grad,
                double* loss, void* stream) {
  if (!pred || !tgt || !grad || !loss || !scratch || N <= 0 || H <= 0 || W <= 0 || !(dx > 0.f))
    return sg_fail(FIP_ERR_ARG, "fip_sg_loss: bad argument");
  if (reinterpret_cast<uintptr_t>(grad) & 15u) return sg_fail(FIP_ERR_ARG, "fip_sg_loss: grad must be 16-byte aligned");
  return sg_cuda(fip::sg::loss_and_grad(pred, tgt, N, H, W, dx, scratch, static_cast<__nv_bfloat16*>(grad), loss, SG_S),
                 "fip_sg_loss");
}

int fip_sg_bias_grad(const void* g, long long n_pix, float* db, void* stream) {
  if (!g || !db || n_pix <= 0) return sg_fail(FIP_ERR_ARG, "fip_sg_bias_grad: bad argument");
  return sg_cuda(fip::sg::bias_grad(static_cast<const __nv_bfloat16*>(g), (size_t)n_pix, db, SG_S), "fip_sg_bias_grad");
}

int fip_sg_adamw(float* p, const float* g, float* m, float* v, long long n, float lr, float beta1, float beta2,
                 float eps, float weight_decay, int step, void* stream) {
  if (!p || !g || !m || !v || n <= 0 || step < 1) return sg_fail(FIP_ERR_ARG, "fip_sg_adamw: bad argument");
  return sg_cuda(fip::sg::adamw(p, g, m, v, (size_t)n, lr, beta1, beta2, eps, weight_decay, step, SG_S), "fip_sg_adamw");
}

int fip_sg_cast_weights(const float* p, int n_layers, void* wf, void* wd, void* stream) {
  if (!p || !wf || !wd || n_layers <= 0) return sg_fail(FIP_ERR_ARG, "fip_sg_cast_weights: bad argument");
  return sg_cuda(fip::sg::cast_weights(p, n_layers, static_cast<__nv_bfloat16*>(wf), static_cast<__nv_bfloat16*>(wd),
                                       SG_S),
                 "fip_sg_cast_weights");
}

int fip_sg_apply(const float* pred, int N, int H, int W, float dx, const float* terrain, float no_value, float* h,
                 float* qx, float* qy, double* dvol, float* hmax, void* stream) {
  if (!pred || !terrain || !h || !qx || !qy || !dvol || N <= 0 || (long long)H * W < 256 || !(dx > 0.f))
    return sg_fail(FIP_ERR_ARG, "fip_sg_apply: bad argument (images of at least 256 cells)");
  return sg_cuda(fip::sg::apply_update(pred, N, H, W, dx, terrain, no_value, h, qx, qy, dvol, hmax, SG_S), "fip_sg_apply");
}

int fip_sg_level_bound(float* h, float* qx, float* qy, const float* terrain, const float* zcap, int N, int H, int W,
                       float no_value, int clip, float umax, double* excess, float* hmax, void* stream) {
  if (!h || !qx || !qy || !terrain || !zcap || !excess || N <= 0 || (long long)H * W < 256 || !(umax >= 0.f))
    return sg_fail(FIP_ERR_ARG, "fip_sg_level_bound: bad argument (images of at least 256 cells)");
  return sg_cuda(fip::sg::level_bound(h, qx, qy, terrain, zcap, N, H, W, no_value, clip, umax, excess, hmax, SG_S),
                 "fip_sg_level_bound");
}

int fip_sg_consistency(const float* pred, int N, int H, int W, float dx, const float* terrain, float no_value,
                       const float* qx, const float* qy, double* res, void* stream) {
  if (!pred || !terrain || !qx || !qy || !res || N <= 0 || (long long)H * W < 256 || H < 3 || W < 4 || !(dx > 0.f))
    return sg_fail(FIP_ERR_ARG, "fip_sg_consistency: bad argument (images of at least 256 cells)");
  return sg_cuda(fip::sg::consistency(pred, N, H, W, dx, terrain, no_value, qx, qy, res, SG_S), "fip_sg_consistency");
}

int fip_sg_edge_flux(const float* qx, const float* qy, int N, int H, int W, double* flux, void* stream) {
  if (!qx || !qy || !flux || N <= 0 || H < 3 || W < 3) return sg_fail(FIP_ERR_ARG, "fip_sg_edge_flux: bad argument");
  return sg_cuda(fip::sg::edge_flux(qx, qy, N, H, W, flux, SG_S), "fip_sg_edge_flux");
}

int fip_sg_edges(float* h, const float* terrain, int N, int H, int W, int t_left, int t_right, int t_top, int t_bottom,
                 float no_value, void* stream) {
  if (!h || !terrain || N <= 0 || H < 3 || W < 3) return sg_fail(FIP_ERR_ARG, "fip_sg_edges: bad argument");
  const int types[4] = {t_left, t_right, t_top, t_bottom};
  for (int t : types)
    if (t < 0 || t > 2) return sg_fail(FIP_ERR_ARG, "fip_sg_edges: side type must be 0 (none), 1 (close) or 2 (open)");
  return sg_cuda(fip::sg::edge_cells(h, terrain, N, H, W, types, no_value, SG_S), "fip_sg_edges");
}

int fip_sg_pin(const unsigned char* mask, const float* h_val, const float* qx_val, const float* qy_val, long long total,
               float* h, float* qx, float* qy, void* stream) {
  if (!mask || !h_val || !qx_val || !qy_val || !h || !qx || !qy || total <= 0)
    return sg_fail(FIP_ERR_ARG, "fip_sg_pin: bad argument");
  return sg_cuda(fip::sg::pin_cells(mask, h_val, qx_val, qy_val, (size_t)total, h, qx, qy, SG_S), "fip_sg_pin");
}

}  // extern "C"
