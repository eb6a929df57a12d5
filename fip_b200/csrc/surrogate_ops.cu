// Element-wise kernels of the learned surrogate: input features, training targets, loss and
// its gradient, bias gradients, AdamW with the bf16 weight layouts of the forward and backward
// convolutions, the surrogate's state update and its mass-balance residual.
//
// The network's four outputs per cell are the mean discharges through its east and north faces
// over the call (Fx, Fy, per unit width) and the changes of qx and qy. The depth changes by the
// discrete continuity equation, dh = -(T / dx) (Fx - Fx_west + Fy - Fy_south), so water only
// moves between neighbours or through the domain edge: the surrogate conserves mass by
// construction (up to the clamp of negative depths).
//
// Grids are fp32 [N][H][W] (one image per scenario, row 0 = southern edge); network tensors are
// NHWC bf16 [N][H + 2 kPad][W + 2 kPad][64] with a zero border (see surrogate_conv.cu), the
// network output is fp32 [N][H + 2 kPad][W + 2 kPad][4]. Feature and output scales are fixed constants (kFeat*, kOut*).
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "surrogate.h"

namespace fip {
namespace sg {

namespace {

__device__ __forceinline__ size_t ppix(int n, int y, int x, int H, int W) {  // padded pixel of interior (y, x)
  return ((size_t)n * (H + 2 * kPad) + (y + kPad)) * (size_t)(W + 2 * kPad) + (x + kPad);
}

// depth change of cell (y, x) from the face discharges (the border pixels of pred are zero, so
// faces outside the image carry nothing); c = T / dx * kOutF
__device__ __forceinline__ float dh_of(const float* __restrict__ pred, size_t p, int Wp, float c) {
  return -c * ((pred[p * 4 + 0] - pred[(p - 1) * 4 + 0]) + (pred[p * 4 + 1] - pred[(p - Wp) * 4 + 1]));
}

// features: 0 terrain - zref, 1 kSt, 2 level - zref, 3 qx, 4 qy, 5 wet (h > 1 cm); 6..63 zero
__global__ void pack_input_kernel(const float* __restrict__ h, const float* __restrict__ qx,
                                  const float* __restrict__ qy, const float* __restrict__ terr,
                                  const float* __restrict__ kst, const float* __restrict__ zref, int N, int H, int W,
                                  float no_value, __nv_bfloat16* __restrict__ out) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t total = (size_t)N * H * W;
  if (i >= total) return;
  const int n = (int)(i / ((size_t)H * W));
  const int y = (int)((i / W) % H), x = (int)(i % W);
  const float t = terr[i];
  const bool valid = t != no_value;
  const float zr = zref[n];
  const float hh = valid ? h[i] : 0.f;
  float f[8];
  f[0] = valid ? (t - zr) * kFeatZ : 0.f;
  f[1] = kst[i] * kFeatK;
  f[2] = valid ? (hh + t - zr) * kFeatZ : 0.f;
  f[3] = valid ? qx[i] * kFeatQ : 0.f;
  f[4] = valid ? qy[i] * kFeatQ : 0.f;
  f[5] = hh > 0.01f ? 1.f : 0.f;
  f[6] = 0.f;
  f[7] = 0.f;
  __nv_bfloat16* d = out + ppix(n, y, x, H, W) * 64;
  uint4 v;
  __nv_bfloat162* pv = reinterpret_cast<__nv_bfloat162*>(&v);
  for (int k = 0; k < 4; ++k) pv[k] = __floats2bfloat162_rn(f[2 * k], f[2 * k + 1]);
  reinterpret_cast<uint4*>(d)[0] = v;
  const uint4 z = make_uint4(0, 0, 0, 0);
  for (int k = 1; k < 8; ++k) reinterpret_cast<uint4*>(d)[k] = z;
}

// target[n][y][x][0..2] = (state1 - state0) / output scale (0 on no-data cells)
__global__ void target_kernel(const float* __restrict__ h0, const float* __restrict__ qx0, const float* __restrict__ qy0,
                              const float* __restrict__ h1, const float* __restrict__ qx1, const float* __restrict__ qy1,
                              const float* __restrict__ terr, size_t total, float no_value, float* __restrict__ tgt) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= total) return;
  const bool valid = terr[i] != no_value;
  tgt[3 * i + 0] = valid ? (h1[i] - h0[i]) * (1.f / kOutZ) : 0.f;
  tgt[3 * i + 1] = valid ? (qx1[i] - qx0[i]) * (1.f / kOutQ) : 0.f;
  tgt[3 * i + 2] = valid ? (qy1[i] - qy0[i]) * (1.f / kOutQ) : 0.f;
}

// loss = squared errors of (dh / kOutZ, dqx, dqy) against the target, summed over the cells (the
// depth term over the inner cells [2, W-2] x [1, H-2] only) and divided by 3 N H W.
// Pass 1: the loss and e[i] = d loss / d(dh / kOutZ) per cell.
__global__ void loss_pass1_kernel(const float* __restrict__ pred, const float* __restrict__ tgt, int N, int H, int W,
                                  float c, float inv_count, float* __restrict__ e, double* __restrict__ loss) {
  __shared__ double red[256];
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t total = (size_t)N * H * W;
  double acc = 0.0;
  if (i < total) {
    const int n = (int)(i / ((size_t)H * W));
    const int y = (int)((i / W) % H), x = (int)(i % W);
    const size_t p = ppix(n, y, x, H, W);
    // only cells the continuity equation updates carry a depth error: the edge cells (and the
    // second column, which a z condition on the left edge also sets) get their depths from the
    // boundary conditions, and fitting them would push the discharges through their faces to 0
    const bool inner = x >= 2 && x <= W - 2 && y >= 1 && y <= H - 2;
    const float d0 = inner ? dh_of(pred, p, W + 2 * kPad, c) * (1.f / kOutZ) - tgt[3 * i + 0] : 0.f;
    const float d1 = pred[p * 4 + 2] - tgt[3 * i + 1];
    const float d2 = pred[p * 4 + 3] - tgt[3 * i + 2];
    acc = (double)d0 * d0 + (double)d1 * d1 + (double)d2 * d2;
    e[i] = 2.f * d0 * inv_count;
  }
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int s = 128; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) atomicAdd(loss, red[0]);
}

// Pass 2: output gradient as bf16 [pix][64] (channels 0..3). Fx[y][x] enters dh of (y, x) with
// -c and of (y, x + 1) with +c; Fy[y][x] enters (y, x) and (y + 1, x) likewise.
__global__ void loss_pass2_kernel(const float* __restrict__ pred, const float* __restrict__ tgt, int N, int H, int W,
                                  float c, float inv_count, const float* __restrict__ e,
                                  __nv_bfloat16* __restrict__ grad) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t total = (size_t)N * H * W;
  if (i >= total) return;
  const int y = (int)((i / W) % H), x = (int)(i % W);
  const int n = (int)(i / ((size_t)H * W));
  const size_t p = ppix(n, y, x, H, W);
  const float cz = c * (1.f / kOutZ);
  const float e0 = e[i];
  const float ee = x + 1 < W ? e[i + 1] : 0.f;
  const float en = y + 1 < H ? e[i + W] : 0.f;
  float g[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  g[0] = cz * (ee - e0);
  g[1] = cz * (en - e0);
  g[2] = 2.f * (pred[p * 4 + 2] - tgt[3 * i + 1]) * inv_count;
  g[3] = 2.f * (pred[p * 4 + 3] - tgt[3 * i + 2]) * inv_count;
  uint4 v;
  __nv_bfloat162* pv = reinterpret_cast<__nv_bfloat162*>(&v);
  for (int k = 0; k < 4; ++k) pv[k] = __floats2bfloat162_rn(g[2 * k], g[2 * k + 1]);
  reinterpret_cast<uint4*>(grad + p * 64)[0] = v;
}

// db[c] += sum over pixels of g[p][c] (border pixels are zero); 64 channels x pixel slices
__global__ void bias_grad_kernel(const __nv_bfloat16* __restrict__ g, size_t n_pix, float* __restrict__ db) {
  __shared__ float red[4][64];
  const int c = threadIdx.x & 63, slot = threadIdx.x >> 6;  // 256 threads: 4 pixel lanes x 64 channels
  float acc = 0.f;
  for (size_t p = (size_t)blockIdx.x * 4 + slot; p < n_pix; p += (size_t)gridDim.x * 4) acc += __bfloat162float(g[p * 64 + c]);
  red[slot][c] = acc;
  __syncthreads();
  if (slot == 0) atomicAdd(&db[c], red[0][c] + red[1][c] + red[2][c] + red[3][c]);
}

// AdamW over all parameters (fp32 master copy); weights of layer l are [9][64][64] at
// l * kLayerParams, biases the 64 values after them. Weight decay applies to weights only.
__global__ void adamw_kernel(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                             float* __restrict__ v, size_t n, float lr, float b1, float b2, float eps, float wd,
                             float bc1, float bc2) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const bool is_w = (i % kLayerParams) < (size_t)9 * 64 * 64;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  float pi = p[i];
  if (is_w) pi -= lr * wd * pi;
  pi -= lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
  p[i] = pi;
}

// bf16 weights of every layer: forward [9][out][in], backward [9][in][out] with taps reversed
__global__ void cast_weights_kernel(const float* __restrict__ p, int n_layers, __nv_bfloat16* __restrict__ wf,
                                    __nv_bfloat16* __restrict__ wd) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t per = (size_t)9 * 64 * 64;
  if (i >= per * n_layers) return;
  const size_t l = i / per, r = i % per;
  const int t = (int)(r / 4096), o = (int)((r / 64) % 64), c = (int)(r % 64);
  const __nv_bfloat16 b = __float2bfloat16_rn(p[l * kLayerParams + r]);
  wf[i] = b;
  wd[l * per + ((size_t)(8 - t) * 64 + c) * 64 + o] = b;
}

// state update of one surrogate call: h += dh of the face discharges (clamped at 0), qx += dqx,
// qy += dqy; no-data cells keep their values. dvol[n] += volume change (depth sum) of image n's
// inner cells; hmax (optional) = max(hmax, new depth).
__global__ void apply_kernel(const float* __restrict__ pred, int N, int H, int W, float c,
                             const float* __restrict__ terr, float no_value, float* __restrict__ h,
                             float* __restrict__ qx, float* __restrict__ qy, double* __restrict__ dvol,
                             float* __restrict__ hmax) {
  __shared__ double red[2][256];
  __shared__ int s_n0;
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t total = (size_t)N * H * W;
  const size_t img = (size_t)H * W;
  double dv = 0.0;
  int n = 0;
  if (i < total) {
    n = (int)(i / img);
    const int y = (int)((i / W) % H), x = (int)(i % W);
    if (terr[i] != no_value) {
      const size_t p = ppix(n, y, x, H, W);
      const float h0 = h[i];
      // continuity moves the depth of the inner cells; the edge cells follow the boundary
      // conditions (fip_sg_edges, pins), as in the solver
      const bool inner = x >= 2 && x <= W - 2 && y >= 1 && y <= H - 2;
      const float h1 = inner ? fmaxf(0.f, h0 + dh_of(pred, p, W + 2 * kPad, c)) : h0;
      h[i] = h1;
      if (hmax) hmax[i] = fmaxf(hmax[i], h1);
      qx[i] += pred[p * 4 + 2] * kOutQ;
      qy[i] += pred[p * 4 + 3] * kOutQ;
      // volume of the cells only the continuity equation updates (a z condition on the left
      // edge also sets column 1): its change must match the discharge through the faces around
      if (inner) dv = (double)h1 - (double)h0;
    }
  }
  if (threadIdx.x == 0) s_n0 = (int)(((size_t)blockIdx.x * blockDim.x) / img);
  __syncthreads();
  const int slot = n - s_n0;  // 0 or 1: a block spans at most two images when H * W >= 256
  red[0][threadIdx.x] = (i < total && slot == 0) ? dv : 0.0;
  red[1][threadIdx.x] = (i < total && slot == 1) ? dv : 0.0;
  __syncthreads();
  for (int s = 128; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      red[0][threadIdx.x] += red[0][threadIdx.x + s];
      red[1][threadIdx.x] += red[1][threadIdx.x + s];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    atomicAdd(&dvol[s_n0], red[0][0]);
    if (s_n0 + 1 < N && red[1][0] != 0.0) atomicAdd(&dvol[s_n0 + 1], red[1][0]);
  }
}

// Consistency residual of one call, before the update: the network predicts the water moved
// through each face twice, as the mean face discharges (Fx, Fy: the depth change by continuity)
// and as the change of the discharges (dqx, dqy: the mean discharge over the call by the
// trapezoid rule, q + dq / 2). Per inner cell the depth changes they imply differ by
// |dh_F - dh_q|; res[n] += the sum over image n (a depth sum: times dx^2 a volume). A network that
// left the states it was trained on stops agreeing with itself.
__global__ void consistency_kernel(const float* __restrict__ pred, int N, int H, int W, float c,
                                   const float* __restrict__ terr, float no_value, const float* __restrict__ qx,
                                   const float* __restrict__ qy, double* __restrict__ res) {
  __shared__ double red[2][256];
  __shared__ int s_n0;
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t total = (size_t)N * H * W;
  const size_t img = (size_t)H * W;
  double r = 0.0;
  int n = 0;
  if (i < total) {
    n = (int)(i / img);
    const int y = (int)((i / W) % H), x = (int)(i % W);
    const bool inner = x >= 2 && x <= W - 2 && y >= 1 && y <= H - 2;
    if (inner && terr[i] != no_value) {
      const size_t p = ppix(n, y, x, H, W);
      const int Wp = W + 2 * kPad;
      const float dhf = dh_of(pred, p, Wp, c);
      // mean discharges of the faces east / west / north / south of the cell over the call
      const float fe = qx[i] + 0.5f * kOutQ * pred[p * 4 + 2];
      const float fw = qx[i - 1] + 0.5f * kOutQ * pred[(p - 1) * 4 + 2];
      const float fn = qy[i] + 0.5f * kOutQ * pred[p * 4 + 3];
      const float fs = qy[i - W] + 0.5f * kOutQ * pred[(p - Wp) * 4 + 3];
      const float dhq = -(c / kOutF) * ((fe - fw) + (fn - fs));
      r = fabs((double)dhf - (double)dhq);
    }
  }
  if (threadIdx.x == 0) s_n0 = (int)(((size_t)blockIdx.x * blockDim.x) / img);
  __syncthreads();
  const int slot = n - s_n0;
  red[0][threadIdx.x] = (i < total && slot == 0) ? r : 0.0;
  red[1][threadIdx.x] = (i < total && slot == 1) ? r : 0.0;
  __syncthreads();
  for (int s = 128; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      red[0][threadIdx.x] += red[0][threadIdx.x + s];
      red[1][threadIdx.x] += red[1][threadIdx.x + s];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    atomicAdd(&res[s_n0], red[0][0]);
    if (s_n0 + 1 < N && red[1][0] != 0.0) atomicAdd(&res[s_n0 + 1], red[1][0]);
  }
}

// Level bound of one call, after the update: in the surrogate's scenarios the water comes from
// a level condition, so no water surface may rise above that level (plus a margin): every cell
// whose level h + terrain exceeds zcap[n] holds water that the network made up. excess[n] +=
// the sum of those depths above the bound (a depth sum: times dx^2 a volume); with `clip` the
// depth is cut back to the bound and the discharges to |q| <= umax * h; hmax (optional) folds
// the resulting depth.
__global__ void level_bound_kernel(float* __restrict__ h, float* __restrict__ qx, float* __restrict__ qy,
                                   const float* __restrict__ terr, const float* __restrict__ zcap, int N, int H,
                                   int W, float no_value, int clip, float umax, double* __restrict__ excess,
                                   float* __restrict__ hmax) {
  __shared__ double red[2][256];
  __shared__ int s_n0;
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t total = (size_t)N * H * W;
  const size_t img = (size_t)H * W;
  double ex = 0.0;
  int n = 0;
  if (i < total) {
    n = (int)(i / img);
    if (terr[i] != no_value) {
      const float cap = fmaxf(0.f, zcap[n] - terr[i]);
      float d = h[i];
      if (d > cap) {
        ex = (double)d - (double)cap;
        if (clip) h[i] = d = cap;
      }
      if (clip) {
        const float qm = umax * fmaxf(d, 0.f);
        qx[i] = fminf(fmaxf(qx[i], -qm), qm);
        qy[i] = fminf(fmaxf(qy[i], -qm), qm);
      }
      if (hmax) hmax[i] = fmaxf(hmax[i], d);
    }
  }
  if (threadIdx.x == 0) s_n0 = (int)(((size_t)blockIdx.x * blockDim.x) / img);
  __syncthreads();
  const int slot = n - s_n0;
  red[0][threadIdx.x] = (i < total && slot == 0) ? ex : 0.0;
  red[1][threadIdx.x] = (i < total && slot == 1) ? ex : 0.0;
  __syncthreads();
  for (int s = 128; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      red[0][threadIdx.x] += red[0][threadIdx.x + s];
      red[1][threadIdx.x] += red[1][threadIdx.x + s];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    atomicAdd(&excess[s_n0], red[0][0]);
    if (s_n0 + 1 < N && red[1][0] != 0.0) atomicAdd(&excess[s_n0 + 1], red[1][0]);
  }
}

// Net discharge into the inner cells [2, W-2] x [1, H-2] per image (qx sits on east faces,
// qy on north faces): + qx[y][1] - qx[y][W-2] over rows 1..H-2, + qy[0][x] - qy[H-2][x] over
// columns 2..W-2 (a sum of discharges per unit width; times dx gives m3/s).
__global__ void edge_flux_kernel(const float* __restrict__ qx, const float* __restrict__ qy, int N, int H, int W,
                                 double* __restrict__ flux) {
  const int n = blockIdx.y;
  double acc = 0.0;
  const size_t base = (size_t)n * H * W;
  for (int k = threadIdx.x; k < (H - 2) + (W - 3); k += blockDim.x) {
    if (k < H - 2) {
      const size_t row = base + (size_t)(k + 1) * W;
      acc += (double)qx[row + 1] - (double)qx[row + (W - 2)];
    } else {
      const int x = 2 + (k - (H - 2));
      acc += (double)qy[base + x] - (double)qy[base + (size_t)(H - 2) * W + x];
    }
  }
  __shared__ double red[256];
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int s = 128; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) flux[n] = red[0];
}

// cells whose state a boundary condition fixes: mask bit 0 resets h, bit 1 qx, bit 2 qy
__global__ void pin_kernel(const unsigned char* __restrict__ mask, const float* __restrict__ hv,
                           const float* __restrict__ qxv, const float* __restrict__ qyv, size_t total,
                           float* __restrict__ h, float* __restrict__ qx, float* __restrict__ qy) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= total) return;
  const unsigned m = mask[i];
  if (m & 1u) h[i] = hv[i];
  if (m & 2u) qx[i] = qxv[i];
  if (m & 4u) qy[i] = qyv[i];
}

// Edge cells by boundary type after a surrogate call, per side (left, right, top, bottom):
// 0 none (the solver never writes the edge: keep), 1 close (depth of the inner neighbour,
// src/bc_kernel_gen.cpp:112-116), 2 open (min(h_nb, max(0, z_nb - terrain)), :128-136).
__global__ void edges_kernel(float* __restrict__ h, const float* __restrict__ terr, int N, int H, int W, int t_left,
                             int t_right, int t_top, int t_bottom, float no_value) {
  const int n = blockIdx.y;
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  float* hn = h + (size_t)n * H * W;
  const float* tn = terr + (size_t)n * H * W;
  auto set = [&](int type, size_t e, size_t nb) {
    if (type == 0 || tn[e] == no_value) return;
    const float hb = hn[nb];
    hn[e] = type == 1 ? hb : (hb > 0.f ? fminf(hb, fmaxf(0.f, hb + tn[nb] - tn[e])) : hn[e]);
  };
  if (k < H) {
    set(t_left, (size_t)k * W, (size_t)k * W + 1);
    set(t_right, (size_t)k * W + (W - 1), (size_t)k * W + (W - 2));
  }
  if (k < W) {
    set(t_bottom, (size_t)k, (size_t)W + k);
    set(t_top, (size_t)(H - 1) * W + k, (size_t)(H - 2) * W + k);
  }
}

}  // namespace

cudaError_t edge_cells(float* h, const float* terr, int N, int H, int W, const int* types, float no_value,
                       cudaStream_t s) {
  const int n = H > W ? H : W;
  edges_kernel<<<dim3((n + 255) / 256, N), 256, 0, s>>>(h, terr, N, H, W, types[0], types[1], types[2], types[3],
                                                       no_value);
  return cudaGetLastError();
}

cudaError_t pin_cells(const unsigned char* mask, const float* hv, const float* qxv, const float* qyv, size_t total,
                      float* h, float* qx, float* qy, cudaStream_t s) {
  pin_kernel<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(mask, hv, qxv, qyv, total, h, qx, qy);
  return cudaGetLastError();
}

cudaError_t pack_input(const float* h, const float* qx, const float* qy, const float* terr, const float* kst,
                       const float* zref, int N, int H, int W, float no_value, __nv_bfloat16* out, cudaStream_t s) {
  const size_t total = (size_t)N * H * W;
  pack_input_kernel<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(h, qx, qy, terr, kst, zref, N, H, W, no_value, out);
  return cudaGetLastError();
}

cudaError_t make_target(const float* h0, const float* qx0, const float* qy0, const float* h1, const float* qx1,
                        const float* qy1, const float* terr, size_t total, float no_value, float* tgt, cudaStream_t s) {
  target_kernel<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(h0, qx0, qy0, h1, qx1, qy1, terr, total, no_value, tgt);
  return cudaGetLastError();
}

cudaError_t loss_and_grad(const float* pred, const float* tgt, int N, int H, int W, float dx, float* scratch,
                          __nv_bfloat16* grad, double* loss, cudaStream_t s) {
  const size_t total = (size_t)N * H * W;
  const float c = kCallS / dx * kOutF, inv = 1.f / (3.f * (float)total);
  const unsigned blocks = (unsigned)((total + 255) / 256);
  loss_pass1_kernel<<<blocks, 256, 0, s>>>(pred, tgt, N, H, W, c, inv, scratch, loss);
  loss_pass2_kernel<<<blocks, 256, 0, s>>>(pred, tgt, N, H, W, c, inv, scratch, grad);
  return cudaGetLastError();
}

cudaError_t bias_grad(const __nv_bfloat16* g, size_t n_pix, float* db, cudaStream_t s) {
  bias_grad_kernel<<<1184, 256, 0, s>>>(g, n_pix, db);
  return cudaGetLastError();
}

cudaError_t adamw(float* p, const float* g, float* m, float* v, size_t n, float lr, float b1, float b2, float eps,
                  float wd, int step, cudaStream_t s) {
  const float bc1 = 1.f - powf(b1, (float)step), bc2 = 1.f - powf(b2, (float)step);
  adamw_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(p, g, m, v, n, lr, b1, b2, eps, wd, bc1, bc2);
  return cudaGetLastError();
}

cudaError_t cast_weights(const float* p, int n_layers, __nv_bfloat16* wf, __nv_bfloat16* wd, cudaStream_t s) {
  const size_t n = (size_t)n_layers * 9 * 64 * 64;
  cast_weights_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(p, n_layers, wf, wd);
  return cudaGetLastError();
}

cudaError_t apply_update(const float* pred, int N, int H, int W, float dx, const float* terr, float no_value, float* h,
                         float* qx, float* qy, double* dvol, float* hmax, cudaStream_t s) {
  const size_t total = (size_t)N * H * W;
  apply_kernel<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(pred, N, H, W, kCallS / dx * kOutF, terr, no_value, h,
                                                                qx, qy, dvol, hmax);
  return cudaGetLastError();
}

cudaError_t consistency(const float* pred, int N, int H, int W, float dx, const float* terr, float no_value,
                        const float* qx, const float* qy, double* res, cudaStream_t s) {
  const size_t total = (size_t)N * H * W;
  consistency_kernel<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(pred, N, H, W, kCallS / dx * kOutF, terr,
                                                                      no_value, qx, qy, res);
  return cudaGetLastError();
}

cudaError_t level_bound(float* h, float* qx, float* qy, const float* terr, const float* zcap, int N, int H, int W,
                        float no_value, int clip, float umax, double* excess, float* hmax, cudaStream_t s) {
  const size_t total = (size_t)N * H * W;
  level_bound_kernel<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(h, qx, qy, terr, zcap, N, H, W, no_value, clip,
                                                                      umax, excess, hmax);
  return cudaGetLastError();
}

cudaError_t edge_flux(const float* qx, const float* qy, int N, int H, int W, double* flux, cudaStream_t s) {
  edge_flux_kernel<<<dim3(1, N), 256, 0, s>>>(qx, qy, N, H, W, flux);
  return cudaGetLastError();
}

}  // namespace sg
}  // namespace fip
