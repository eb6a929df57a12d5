/*
 * fip_b200 -- learned surrogate of the slim shallow-water step (no counterpart in the reference).
 *
 * BF16 3x3 convolutions on the sm_100a tensor cores (tcgen05, fp32 accumulation in tensor
 * memory) and the element-wise kernels of training and inference. Tensors are device pointers:
 * activations are NHWC bf16 with 64 channels and a zero border of FIP_SG_PAD pixels around each
 * image ([N][H+16][W+16][64]); weights are bf16 [9 taps][64 out][64 in], tap = (dy+1)*3 + (dx+1);
 * a convolution of dilation d (1..8) reads tap (dy, dx) at (y + d dy, x + d dx).
 * `stream` is a cudaStream_t (NULL: the default stream). `dev_err` (may be NULL) is a device int
 * that a kernel sets to a nonzero code when one of its bounded waits runs out. Functions return
 * FIP_OK (0) or a negative FIP_ERR_* code (include/fip.h).
 */
#ifndef FIP_B200_FIP_SURROGATE_H
#define FIP_B200_FIP_SURROGATE_H

#ifdef __cplusplus
extern "C" {
#endif

#define FIP_SG_PAD 8               /* zero border of every network tensor, pixels */
#define FIP_SG_EPI_BIAS_RELU 0     /* out = relu(conv + bias) */
#define FIP_SG_EPI_BIAS_RES_RELU 1 /* out = relu(conv + bias + res) */
#define FIP_SG_EPI_HEAD 2          /* out (f32 [pixels][4]) = conv[0..3] + bias[0..3] */
#define FIP_SG_EPI_MASK 3          /* out = conv * (mask > 0)          (ReLU backward) */
#define FIP_SG_EPI_RES_MASK 4      /* out = (conv + res) * (mask > 0)  (residual + ReLU backward) */
#define FIP_SG_EPI_PLAIN 5         /* out = conv */

/* out = epilogue(conv3x3(in, w)); border pixels of out are written as zero. */
int fip_sg_conv3x3(const void* in, const void* w, const float* bias, const void* res, const void* mask, void* out,
                   int N, int H, int W, int dilation, int epi, int* dev_err, void* stream);

/* dw (f32 [9][64 out][64 in]) = sum over pixels of x[p + tap offset][in] * dy[p][out].
 * The per-CTA partial sums go to one scratch buffer per device, allocated by the first call on
 * that device and shared by every later call: wgrad calls on one device must not overlap (another
 * stream or host thread), or they race on it. */
int fip_sg_conv3x3_wgrad(const void* x, const void* dy, float* dw, int N, int H, int W, int dilation, int* dev_err,
                         void* stream);

/* ---- element-wise kernels; grids are f32 [N][H][W] (row 0 = southern edge) ---- */

/* Network input [N][H+16][W+16][64] bf16: (terrain - zref[n]) * 0.1, kSt * 0.025,
 * (h + terrain - zref[n]) * 0.1, qx * 0.2, qy * 0.2, (h > 1 cm); zero on no-data cells and in
 * channels 6..63. */
int fip_sg_pack_input(const float* h, const float* qx, const float* qy, const float* terrain, const float* kst,
                      const float* zref, int N, int H, int W, float no_value, void* out, void* stream);
/* Training target f32 [N][H][W][3]: (h1 - h0) / 0.5, (qx1 - qx0) / 1, (qy1 - qy0) / 1. */
int fip_sg_target(const float* h0, const float* qx0, const float* qy0, const float* h1, const float* qx1,
                  const float* qy1, const float* terrain, long long total, float no_value, float* tgt, void* stream);
/* The network output pred (f32 [N][H+16][W+16][4]) holds per cell the mean discharges through
 * the east and north faces over the 60-s call (Fx, Fy, m2/s) and the changes of qx and qy; the
 * depth change is dh = -(60 / dx) (Fx - Fx_west + Fy - Fy_south) (mass conserving).
 * *loss += sum of squared errors of (dh / 0.5, dqx, dqy) against tgt (dh over the inner cells
 * [2, W-2] x [1, H-2], whose depth only continuity changes); grad (bf16
 * [N][H+16][W+16][64], channels 0..3) = d(mean squared error)/d(pred); scratch holds N*H*W
 * floats. grad must be zeroed first. */
int fip_sg_loss(const float* pred, const float* tgt, int N, int H, int W, float dx, float* scratch, void* grad,
                double* loss, void* stream);
/* db[c] += sum over pixels of g[p][c] (bf16 [n_pix][64]). */
int fip_sg_bias_grad(const void* g, long long n_pix, float* db, void* stream);
/* AdamW step (step >= 1) over n parameters laid out as layers of 9*64*64 weights + 64 biases;
 * decoupled weight decay on the weights only. */
int fip_sg_adamw(float* p, const float* g, float* m, float* v, long long n, float lr, float beta1, float beta2,
                 float eps, float weight_decay, int step, void* stream);
/* bf16 copies of n_layers layers of f32 parameters: wf [l][9][out][in] for the forward
 * convolution, wd [l][9][in][out] with reversed taps for the input gradient. */
int fip_sg_cast_weights(const float* p, int n_layers, void* wf, void* wd, void* stream);
/* One surrogate call: h = max(0, h + dh) on the inner cells [2, W-2] x [1, H-2] with dh from the
 * face discharges (edge cells: fip_sg_edges), qx += pred2, qy += pred3 (no-data cells kept);
 * dvol[n] += change of the depth sum over the inner cells [2, W-2] x [1, H-2] of image n
 * (H * W >= 256); hmax (may be NULL) = max(hmax, new h). */
int fip_sg_apply(const float* pred, int N, int H, int W, float dx, const float* terrain, float no_value, float* h,
                 float* qx, float* qy, double* dvol, float* hmax, void* stream);
/* Level bound of a surrogate state (after fip_sg_apply): where the water level h + terrain of
 * image n exceeds zcap[n] (the highest level its boundary conditions impose, plus a margin),
 * excess[n] += the depth above the bound (a depth sum, H * W >= 256); with clip != 0 the depth is
 * cut back to the bound and qx, qy to |q| <= umax * h; hmax (may be NULL) = max(hmax, depth).
 * No-data cells are skipped. */
int fip_sg_level_bound(float* h, float* qx, float* qy, const float* terrain, const float* zcap, int N, int H, int W,
                       float no_value, int clip, float umax, double* excess, float* hmax, void* stream);
/* Fallback indicator of one call, evaluated before fip_sg_apply: res[n] += sum over the inner
 * cells of image n (H * W >= 256) of |dh_F - dh_q|, the disagreement between the depth change
 * the face-discharge outputs imply (continuity) and the one the discharge-change outputs imply
 * (mean discharge over the call, q + dq / 2). A depth sum: times dx^2 it is a volume. */
int fip_sg_consistency(const float* pred, int N, int H, int W, float dx, const float* terrain, float no_value,
                       const float* qx, const float* qy, double* res, void* stream);
/* flux[n] = net discharge per unit width into the inner cells [2, W-2] x [1, H-2] of image n
 * (through qx[:, 1], qx[:, W-2], qy[0, :], qy[H-2, :]). */
int fip_sg_edge_flux(const float* qx, const float* qy, int N, int H, int W, double* flux, void* stream);

/* Edge cells after a surrogate call by the boundary type of each side: 0 none (kept), 1 close
 * (depth of the inner neighbour), 2 open (min(h_nb, max(0, z_nb - terrain))). */
int fip_sg_edges(float* h, const float* terrain, int N, int H, int W, int t_left, int t_right, int t_top, int t_bottom,
                 float no_value, void* stream);
/* Cells fixed by boundary conditions: mask bit 0 sets h, bit 1 qx, bit 2 qy to the given values. */
int fip_sg_pin(const unsigned char* mask, const float* h_val, const float* qx_val, const float* qy_val, long long total,
               float* h, float* qx, float* qy, void* stream);

#ifdef __cplusplus
}
#endif
#endif
