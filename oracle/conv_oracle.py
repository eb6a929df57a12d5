"""FP64 CPU oracle of the surrogate's 3x3 convolutions (test infrastructure only: the tests
compare the tcgen05 kernels of libfip_b200 with it; nothing in the product calls it).

The surrogate has no counterpart in the reference; these are the textbook definitions, for a
dilation d:
  forward  y[n, i, j, o] = sum over dy, dx in {-1, 0, 1} and c of x[n, i + d dy, j + d dx, c] * w[t, o, c]
           with t = (dy + 1) * 3 + (dx + 1) and x = 0 outside the image;
  dgrad    dx[n, i, j, c] = sum over t, o of dy[n, i - d dy_t, j - d dx_t, o] * w[t, o, c]
           (the forward convolution with weights w'[8 - t, c, o] = w[t, o, c]);
  wgrad    dw[t, o, c] = sum over n, i, j of x[n, i + d dy_t, j + d dx_t, c] * dy[n, i, j, o].
Tensors here are unpadded NHWC float arrays; `pad` adds the zero border of the device layout.
"""
import numpy as np


PAD = 8  # zero border of the device tensors (FIP_SG_PAD)


def pad(x, p=PAD):
    return np.pad(x, ((0, 0), (p, p), (p, p), (0, 0)))


def conv3x3(x, w, d=1):
    x = np.asarray(x, np.float64)
    w = np.asarray(w, np.float64)
    N, H, W, _ = x.shape
    xp = pad(x, d)
    y = np.zeros((N, H, W, w.shape[1]))
    for t in range(9):
        dy, dx = (t // 3 - 1) * d, (t % 3 - 1) * d
        y += xp[:, d + dy:d + dy + H, d + dx:d + dx + W, :] @ w[t].T
    return y


def dgrad_weights(w):
    """w'[t] = w[8 - t]^T: the dgrad as a forward convolution."""
    w = np.asarray(w)
    return np.stack([w[8 - t].T for t in range(9)])


def wgrad(x, dy, d=1):
    x = np.asarray(x, np.float64)
    g = np.asarray(dy, np.float64)
    N, H, W, _ = x.shape
    xp = pad(x, d)
    dw = np.zeros((9, g.shape[3], x.shape[3]))
    for t in range(9):
        a, b = (t // 3 - 1) * d, (t % 3 - 1) * d
        xs = xp[:, d + a:d + a + H, d + b:d + b + W, :].reshape(-1, x.shape[3])
        dw[t] = g.reshape(-1, g.shape[3]).T @ xs
    return dw
