"""FP64 CPU oracle of the surrogate network's forward pass and gradients (test infrastructure
only: tests compare the GPU training kernels with it; the product never calls it).

Same network as fip_b200/surrogate.py, on unpadded NHWC arrays:
  a0 = relu(conv(x, W0) + b0)
  h_k = relu(conv(a_k, W_{2k+1}) + b_{2k+1}),  a_{k+1} = relu(conv(h_k, W_{2k+2}) + b_{2k+2} + a_k)
  pred = conv(a_8, W17)[..., :3] + b17[:3]
  loss = mean((pred - target)^2)
Gradients by reverse-mode differentiation of the same expressions (conv_oracle supplies the
convolution and its two adjoints).
"""
import numpy as np

import conv_oracle

C, TAP = 64, 9 * 64 * 64
LAYER = TAP + C


def unpack(p, l):
    w = p[l * LAYER:l * LAYER + TAP].reshape(9, C, C).astype(np.float64)
    b = p[l * LAYER + TAP:(l + 1) * LAYER].astype(np.float64)
    return w, b


def forward(p, x):
    acts = {}
    w, b = unpack(p, 0)
    a = np.maximum(conv_oracle.conv3x3(x, w) + b, 0)
    acts["a0"] = a
    for k in range(8):
        w1, b1 = unpack(p, 1 + 2 * k)
        w2, b2 = unpack(p, 2 + 2 * k)
        h = np.maximum(conv_oracle.conv3x3(a, w1) + b1, 0)
        a = np.maximum(conv_oracle.conv3x3(h, w2) + b2 + a, 0)
        acts[f"h{k}"] = h
        acts[f"a{k + 1}"] = a
    w, b = unpack(p, 17)
    pred = conv_oracle.conv3x3(a, w)[..., :4] + b[:4]
    return pred, acts


def loss_and_grads(p, x, target):
    """target: [N, H, W, 3]; returns (loss, grads shaped like p)."""
    pred, acts = forward(p, x)
    count = target.size
    d = pred[..., :3] - target
    loss = float(np.sum(d * d) / count)
    gout = np.zeros(pred.shape[:3] + (C,))
    gout[..., :3] = 2.0 * d / count
    grads = np.zeros(p.size)

    def put(l, x_in, dy):
        grads[l * LAYER:l * LAYER + TAP] = conv_oracle.wgrad(x_in, dy).reshape(-1)
        grads[l * LAYER + TAP:(l + 1) * LAYER] = dy.reshape(-1, C).sum(0)

    put(17, acts["a8"], gout)
    w, _ = unpack(p, 17)
    g = conv_oracle.conv3x3(gout, conv_oracle.dgrad_weights(w)) * (acts["a8"] > 0)
    for k in range(7, -1, -1):
        put(2 + 2 * k, acts[f"h{k}"], g)
        w2, _ = unpack(p, 2 + 2 * k)
        dh = conv_oracle.conv3x3(g, conv_oracle.dgrad_weights(w2)) * (acts[f"h{k}"] > 0)
        put(1 + 2 * k, acts[f"a{k}"], dh)
        w1, _ = unpack(p, 1 + 2 * k)
        g = (conv_oracle.conv3x3(dh, conv_oracle.dgrad_weights(w1)) + g) * (acts[f"a{k}"] > 0)
    put(0, x, g)
    return loss, grads, pred
