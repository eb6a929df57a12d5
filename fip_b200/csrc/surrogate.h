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

struct ConvShape {
  int N, H, W;  // images and interior size; tensors hold N x (H + 2) x (W + 2) pixels x 64 channels
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

}  // namespace sg
}  // namespace fip
