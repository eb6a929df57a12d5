// Learned surrogate of the slim shallow-water step: BF16 tcgen05 convolution kernels
// (surrogate_conv.cu) and the element-wise training kernels (surrogate_ops.cu). Internal to
// libfip_b200; the C ABI is in include/fip_surrogate.h.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stddef.h>

#include <algorithm>
#include <string>

// fused epilogues of conv3x3 (out = f(acc)) at interior pixels; border pixels get 0
#define EPI_BIAS_RELU 0      // relu(acc + bias)                      bf16 [pix][64]
#define EPI_BIAS_RES_RELU 1  // relu(acc + bias + res)                bf16 [pix][64]
#define EPI_HEAD 2           // acc[0..3] + bias[0..3]                f32  [pix][4]
#define EPI_MASK 3           // acc * (mask > 0)                      bf16 [pix][64]
#define EPI_RES_MASK 4       // (acc + res) * (mask > 0)              bf16 [pix][64]
#define EPI_PLAIN 5          // acc                                   bf16 [pix][64]

namespace fip {
namespace sg {

// feature and output scales of the network
constexpr float kFeatZ = 0.1f;   // terrain / level relative to the image's mean terrain, per metre
constexpr float kFeatK = 0.025f; // Strickler coefficient
constexpr float kFeatQ = 0.2f;   // discharge per unit width, per m2/s
constexpr float kOutZ = 0.5f;    // depth change of one call, metres per target unit
constexpr float kOutQ = 1.0f;    // discharge change of one call, m2/s per output unit
constexpr float kOutF = 1.0f;    // mean face discharge over one call, m2/s per output unit
constexpr float kCallS = 60.0f;  // simulated seconds of one call
constexpr size_t kLayerParams = (size_t)9 * 64 * 64 + 64;  // weights then biases of one conv layer

// zero border around every image of a network tensor: taps of dilation up to kPad stay inside it
constexpr int kPad = 8;
constexpr int kMaxDil = 8;

struct ConvShape {
  int N, H, W;  // images and interior size; tensors hold N x (H + 2 kPad) x (W + 2 kPad) pixels x 64 channels
  int dil;      // dilation of the 3x3 kernel: tap (dy, dx) reads (y + dil * dy, x + dil * dx)
};

// 3x3 convolution, 64 -> 64 channels, weights bf16 [9 taps][64 out][64 in] (tap = (dy + 1) * 3 + dx + 1).
cudaError_t conv3x3(const ConvShape& s, const __nv_bfloat16* in, const __nv_bfloat16* w, const float* bias,
                    const __nv_bfloat16* res, const __nv_bfloat16* mask, void* out, int epi, int* err,
                    cudaStream_t stream);

// dw[tap][out][in] = sum over pixels of x[p + off(tap)][in] * dy[p][out]; `part` holds
// wgrad_scratch_floats() floats.
size_t wgrad_scratch_floats();
cudaError_t conv3x3_wgrad(const ConvShape& s, const __nv_bfloat16* x, const __nv_bfloat16* dy, float* part, float* dw,
                          int* err, cudaStream_t stream);

int conv_grid();

// element-wise kernels (surrogate_ops.cu)
cudaError_t pack_input(const float* h, const float* qx, const float* qy, const float* terr, const float* kst,
                       const float* zref, int N, int H, int W, float no_value, __nv_bfloat16* out, cudaStream_t s);
cudaError_t make_target(const float* h0, const float* qx0, const float* qy0, const float* h1, const float* qx1,
                        const float* qy1, const float* terr, size_t total, float no_value, float* tgt, cudaStream_t s);
cudaError_t loss_and_grad(const float* pred, const float* tgt, int N, int H, int W, float dx, float* scratch,
                          __nv_bfloat16* grad, double* loss, cudaStream_t s);
cudaError_t bias_grad(const __nv_bfloat16* g, size_t n_pix, float* db, cudaStream_t s);
cudaError_t adamw(float* p, const float* g, float* m, float* v, size_t n, float lr, float b1, float b2, float eps,
                  float wd, int step, cudaStream_t s);
cudaError_t cast_weights(const float* p, int n_layers, __nv_bfloat16* wf, __nv_bfloat16* wd, cudaStream_t s);
cudaError_t apply_update(const float* pred, int N, int H, int W, float dx, const float* terr, float no_value, float* h,
                         float* qx, float* qy, double* dvol, float* hmax, cudaStream_t s);
cudaError_t edge_flux(const float* qx, const float* qy, int N, int H, int W, double* flux, cudaStream_t s);
cudaError_t level_bound(float* h, float* qx, float* qy, const float* terr, const float* zcap, int N, int H, int W,
                        float no_value, int clip, float umax, double* excess, float* hmax, cudaStream_t s);
cudaError_t consistency(const float* pred, int N, int H, int W, float dx, const float* terr, float no_value,
                        const float* qx, const float* qy, double* res, cudaStream_t s);
cudaError_t edge_cells(float* h, const float* terr, int N, int H, int W, const int* types, float no_value,
                       cudaStream_t s);
cudaError_t pin_cells(const unsigned char* mask, const float* hv, const float* qxv, const float* qyv, size_t total,
                      float* h, float* qx, float* qy, cudaStream_t s);

}  // namespace sg
}  // namespace fip
