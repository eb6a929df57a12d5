"""FP64 CPU oracle of the surrogate network's forward pass and gradients (test infrastructure
only: tests compare the GPU training kernels with it; the product never calls it).

Same network as fip_b200/surrogate.py, on unpadded NHWC arrays:
  a0 = relu(conv(x, W0) + b0)
  h_k = relu(conv_d(a_k, W_{2k+1}) + b_{2k+1}),  a_{k+1} = relu(conv_d(h_k, W_{2k+2}) + b_{2k+2} + a_k)
  pred = conv(a_8, W17)[..., :4] + b17[:4]      (Fx, Fy, dqx, dqy)
  dh = -(60 / dx) (Fx - Fx_west + Fy - Fy_south)  (faces outside the image carry nothing)
  loss = squared errors of (dh / 0.5, dqx, dqy) summed over the cells (dh over the inner cells
         [2, W-2] x [1, H-2] only: the edge cells follow the boundary conditions) / (3 N H W)
with the dilation d of layer l given by DIL (block k: 1, 2, 4, 8, 1, 2, 4, 8).
Gradients by reverse-mode differentiation of the same expressions (conv_oracle supplies the
convolution and its two adjoints).
"""
import numpy as np

import conv_oracle

C, TAP = 64, 9 * 64 * 64
LAYER = TAP + C
DIL = [1] + [d for d in (1, 2, 4, 8, 1, 2, 4, 8) for _ in range(2)] + [1]


def unpack(p, l):
    w = p[l * LAYER:l * LAYER + TAP].reshape(9, C, C).astype(np.float64)
    b = p[l * LAYER + TAP:(l + 1) * LAYER].astype(np.float64)
    return w, b


def forward(p, x):
    acts = {}
    w, b = unpack(p, 0)
    a = np.maximum(conv_oracle.conv3x3(x, w, DIL[0]) + b, 0)
    acts["a0"] = a
    for k in range(8):
        w1, b1 = unpack(p, 1 + 2 * k)
        w2, b2 = unpack(p, 2 + 2 * k)
        h = np.maximum(conv_oracle.conv3x3(a, w1, DIL[1 + 2 * k]) + b1, 0)
        a = np.maximum(conv_oracle.conv3x3(h, w2, DIL[2 + 2 * k]) + b2 + a, 0)
        acts[f"h{k}"] = h
        acts[f"a{k + 1}"] = a
    w, b = unpack(p, 17)
    pred = conv_oracle.conv3x3(a, w, DIL[17])[..., :4] + b[:4]
    return pred, acts


def depth_change(pred, dx=3.0):
    fx, fy = pred[..., 0], pred[..., 1]
    fxw = np.pad(fx, ((0, 0), (0, 0), (1, 0)))[:, :, :-1]
    fys = np.pad(fy, ((0, 0), (1, 0), (0, 0)))[:, :-1, :]
    return -(60.0 / dx) * (fx - fxw + fy - fys)


def loss_and_grads(p, x, target, dx=3.0):
    """target: [N, H, W, 3] (dh / 0.5, dqx, dqy); returns (loss, grads shaped like p, pred)."""
    pred, acts = forward(p, x)
    count = target.size
    c = 60.0 / dx
    d0 = depth_change(pred, dx) / 0.5 - target[..., 0]
    inner = np.zeros(d0.shape[1:], bool)
    inner[1:-1, 2:-1] = True  # depth error on the cells only continuity updates
    d0 = np.where(inner, d0, 0.0)
    d1 = pred[..., 2] - target[..., 1]
    d2 = pred[..., 3] - target[..., 2]
    loss = float((np.sum(d0 * d0) + np.sum(d1 * d1) + np.sum(d2 * d2)) / count)
    e = 2.0 * d0 / count
    ee = np.pad(e, ((0, 0), (0, 0), (0, 1)))[:, :, 1:]
    en = np.pad(e, ((0, 0), (0, 1), (0, 0)))[:, 1:, :]
    gout = np.zeros(pred.shape[:3] + (C,))
    gout[..., 0] = (c / 0.5) * (ee - e)
    gout[..., 1] = (c / 0.5) * (en - e)
    gout[..., 2] = 2.0 * d1 / count
    gout[..., 3] = 2.0 * d2 / count
    grads = np.zeros(p.size)

    def put(l, x_in, dy):
        grads[l * LAYER:l * LAYER + TAP] = conv_oracle.wgrad(x_in, dy, DIL[l]).reshape(-1)
        grads[l * LAYER + TAP:(l + 1) * LAYER] = dy.reshape(-1, C).sum(0)

    put(17, acts["a8"], gout)
    w, _ = unpack(p, 17)
    g = conv_oracle.conv3x3(gout, conv_oracle.dgrad_weights(w), DIL[17]) * (acts["a8"] > 0)
    for k in range(7, -1, -1):
        put(2 + 2 * k, acts[f"h{k}"], g)
        w2, _ = unpack(p, 2 + 2 * k)
        dh = conv_oracle.conv3x3(g, conv_oracle.dgrad_weights(w2), DIL[2 + 2 * k]) * (acts[f"h{k}"] > 0)
        put(1 + 2 * k, acts[f"a{k}"], dh)
        w1, _ = unpack(p, 1 + 2 * k)
        g = (conv_oracle.conv3x3(dh, conv_oracle.dgrad_weights(w1), DIL[1 + 2 * k]) + g) * (acts[f"a{k}"] > 0)
    put(0, x, g)
    return loss, grads, pred


def consistency(pred, qx, qy, terrain, no_value, dx=3.0):
    """Fallback indicator of one call (fip_sg_consistency): per image, the sum over the inner cells
    [2, W-2] x [1, H-2] (not no_data) of |dh_F - dh_q|, dh_F from the face discharges (continuity)
    and dh_q from the mean discharges q + dq / 2 of the four faces. pred: [N, H, W, 4]."""
    c = 60.0 / dx
    dhf = depth_change(pred.astype(np.float64), dx)
    fx = qx.astype(np.float64) + 0.5 * pred[..., 2]
    fy = qy.astype(np.float64) + 0.5 * pred[..., 3]
    fxw = np.pad(fx, ((0, 0), (0, 0), (1, 0)))[:, :, :-1]
    fys = np.pad(fy, ((0, 0), (1, 0), (0, 0)))[:, :-1, :]
    dhq = -c * (fx - fxw + fy - fys)
    N, H, W = qx.shape
    inner = np.zeros((H, W), bool)
    inner[1:H - 1, 2:W - 1] = True
    m = inner[None] & (terrain != no_value)
    return np.array([np.abs(dhf[n] - dhq[n])[m[n]].sum() for n in range(N)])


def level_bound(h, qx, qy, terrain, zcap, no_value, umax):
    """fip_sg_level_bound with clip and hmax: returns (h, qx, qy, excess[N], hmax-fold of the new
    depth over zeros). Depth above zcap[n] - terrain (at least 0) is removed and summed; then
    |q| <= umax * h; no-data cells untouched."""
    h, qx, qy = h.astype(np.float32).copy(), qx.astype(np.float32).copy(), qy.astype(np.float32).copy()
    valid = terrain != no_value
    cap = np.maximum(np.float32(0), zcap.astype(np.float32)[:, None, None] - terrain).astype(np.float32)
    over = valid & (h > cap)
    excess = np.where(over, h.astype(np.float64) - cap.astype(np.float64), 0.0).sum(axis=(1, 2))
    h = np.where(over, cap, h).astype(np.float32)
    qm = (np.float32(umax) * np.maximum(h, np.float32(0))).astype(np.float32)
    qx = np.where(valid, np.minimum(np.maximum(qx, -qm), qm), qx).astype(np.float32)
    qy = np.where(valid, np.minimum(np.maximum(qy, -qm), qm), qy).astype(np.float32)
    return h, qx, qy, excess
