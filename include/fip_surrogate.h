/*
 * fip_b200 -- learned surrogate of the slim shallow-water step (no counterpart in the reference).
 *
 * BF16 3x3 convolutions on the sm_100a tensor cores (tcgen05, fp32 accumulation in tensor
 * memory) and the element-wise kernels of training and inference. Tensors are device pointers:
 * activations are NHWC bf16 with 64 channels and a one-pixel zero border around each image
 * ([N][H+2][W+2][64]); weights are bf16 [9 taps][64 out][64 in], tap = (dy+1)*3 + (dx+1).
 * `stream` is a cudaStream_t (NULL: the default stream). `dev_err` (may be NULL) is a device int
 * that a kernel sets to a nonzero code when one of its bounded waits runs out. Functions return
 * FIP_OK (0) or a negative FIP_ERR_* code (include/fip.h).
 */
#ifndef FIP_B200_FIP_SURROGATE_H
#define FIP_B200_FIP_SURROGATE_H

#ifdef __cplusplus
extern "C" {
#endif

#define FIP_SG_EPI_BIAS_RELU 0     /* out = relu(conv + bias) */
#define FIP_SG_EPI_BIAS_RES_RELU 1 /* out = relu(conv + bias + res) */
#define FIP_SG_EPI_HEAD 2          /* out (f32 [pixels][4]) = conv[0..3] + bias[0..3] */
#define FIP_SG_EPI_MASK 3          /* out = conv * (mask > 0)          (ReLU backward) */
#define FIP_SG_EPI_RES_MASK 4      /* out = (conv + res) * (mask > 0)  (residual + ReLU backward) */
#define FIP_SG_EPI_PLAIN 5         /* out = conv */

/* out = epilogue(conv3x3(in, w)); border pixels of out are written as zero. */
int fip_sg_conv3x3(const void* in, const void* w, const float* bias, const void* res, const void* mask, void* out,
                   int N, int H, int W, int epi, int* dev_err, void* stream);

/* dw (f32 [9][64 out][64 in]) = sum over pixels of x[p + tap offset][in] * dy[p][out]. */
int fip_sg_conv3x3_wgrad(const void* x, const void* dy, float* dw, int N, int H, int W, int* dev_err, void* stream);

#ifdef __cplusplus
}
#endif
#endif
