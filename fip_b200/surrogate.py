"""Learned surrogate of the slim shallow-water step: a residual CNN that advances z/qx/qy by 60
simulated seconds per call, trained on trajectories the solver itself generates.

Network (every convolution 3x3, BF16 operands, FP32 accumulation on the tcgen05 tensor cores,
libfip_b200 kernels of include/fip_surrogate.h):
  input  6 features per cell (terrain, kSt, water level, qx, qy, wet mask), zero-padded to 64
  stem   conv 64 -> 64 + ReLU
  8 residual blocks   a' = relu(a + conv_d(relu(conv_d(a))))      (16 convolutions)
  head   conv 64 -> 4: mean discharges through each cell's east and north faces over the next
         60 s (Fx, Fy) and the changes of qx and qy; the depth changes by the discrete
         continuity equation dh = -(60 / dx) (Fx - Fx_west + Fy - Fy_south), so the surrogate
         moves water between neighbours and through the domain edge only (mass conserving)
The 3x3 kernels of block k are dilated by d = 1, 2, 4, 8, 1, 2, 4, 8: the network sees 62 cells
(186 m) around a cell, about as far as a flood front travels in 60 s; undilated it would see 18.
Tensors carry a zero border of 8 pixels (FIP_SG_PAD) so that every dilated tap stays inside.
The head starts at zero, so an untrained network is persistence (nothing changes); training
learns the change. Cells held by boundary conditions are reset to their condition's values
after every call (`pin`). AdamW on an FP32 master copy; the bf16 weights of the forward and of
the input-gradient convolutions are re-cast after every update.

PyTorch only provides device memory (tensors as buffers) and the current stream; every
arithmetic step runs in the library's own kernels.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np

from . import _lib

C = 64
PAD = 8
TAP = 9 * C * C
LAYER = TAP + C  # weights then biases of one layer
N_LAYERS = 18    # stem, 8 x 2 block convolutions, head
DIL = [1] + [d for d in (1, 2, 4, 8, 1, 2, 4, 8) for _ in range(2)] + [1]
EPI_BIAS_RELU, EPI_BIAS_RES_RELU, EPI_HEAD, EPI_MASK, EPI_RES_MASK, EPI_PLAIN = range(6)
OUT_Z, OUT_Q = 0.5, 1.0


def _torch():
    import torch

    return torch


def _ptr(t, offset_elems: int = 0) -> ctypes.c_void_p:
    return ctypes.c_void_p(t.data_ptr() + offset_elems * t.element_size())


def _stream():
    return ctypes.c_void_p(_torch().cuda.current_stream().cuda_stream)


def init_params(seed: int = 0) -> np.ndarray:
    """He-normal weights ([tap][out][in]); the second convolution of each block and the head
    start small / at zero so the untrained network is close to the identity map of the state."""
    rng = np.random.default_rng(seed)
    p = np.zeros(N_LAYERS * LAYER, np.float32)
    for l in range(N_LAYERS):
        w = np.zeros((9, C, C), np.float32)
        if l == 0:
            w[:, :, :6] = rng.standard_normal((9, C, 6)) * math.sqrt(2.0 / (9 * 6))
        elif l == N_LAYERS - 1:
            pass  # head: zero -> persistence
        else:
            std = math.sqrt(2.0 / (9 * C)) * (0.1 if l % 2 == 0 else 1.0)
            w[:] = rng.standard_normal((9, C, C)) * std
        p[l * LAYER:l * LAYER + TAP] = w.reshape(-1)
    return p


class Surrogate:
    """The network, its optimiser state and its activation buffers on one GPU."""

    def __init__(self, device: int = 0, seed: int = 0, params: np.ndarray | None = None):
        torch = _torch()
        self.torch = torch
        self.dev = torch.device("cuda", device)
        self.L = _lib.lib()
        p = init_params(seed) if params is None else np.asarray(params, np.float32)
        assert p.size == N_LAYERS * LAYER
        self.p = torch.from_numpy(p.copy()).to(self.dev)
        self.g = torch.zeros_like(self.p)
        self.m = torch.zeros_like(self.p)
        self.v = torch.zeros_like(self.p)
        self.wf = torch.empty(N_LAYERS * TAP, dtype=torch.bfloat16, device=self.dev)
        self.wd = torch.empty_like(self.wf)
        self.err = torch.zeros(1, dtype=torch.int32, device=self.dev)
        self.loss_acc = torch.zeros(1, dtype=torch.float64, device=self.dev)
        self.steps = 0
        self._bufs = {}
        self.cast()

    # ---- parameters ------------------------------------------------------------------------
    def cast(self):
        _lib.check(self.L.fip_sg_cast_weights(_ptr(self.p), N_LAYERS, _ptr(self.wf), _ptr(self.wd), _stream()))

    def params(self) -> np.ndarray:
        return self.p.cpu().numpy().copy()

    def check_device(self):
        self.torch.cuda.synchronize(self.dev)
        code = int(self.err.item())
        if code:
            raise RuntimeError(f"surrogate kernel: a device-side wait ran out (code {code})")

    # ---- buffers -----------------------------------------------------------------------------
    def _buffers(self, N, H, W, train):
        key = (N, H, W, train)
        if key not in self._bufs:
            torch = self.torch
            shape = (N, H + 2 * PAD, W + 2 * PAD, C)
            act = lambda: torch.zeros(shape, dtype=torch.bfloat16, device=self.dev)  # noqa: E731
            b = {"x": act(),
                 "pred": torch.zeros((N, H + 2 * PAD, W + 2 * PAD, 4), dtype=torch.float32, device=self.dev)}
            b["e"] = torch.zeros((N, H, W), dtype=torch.float32, device=self.dev)
            if train:
                b["a"] = [act() for _ in range(9)]
                b["h"] = [act() for _ in range(8)]
                b["g"] = [act() for _ in range(3)]
            else:
                b["a"] = [act(), act()]
                b["h"] = [act()]
            self._bufs = {k: v for k, v in self._bufs.items() if k[3] != train}  # keep one shape per mode
            self._bufs[key] = b
        return self._bufs[key]

    def _conv(self, src, layer, epi, out, N, H, W, res=None, mask=None, grad=False):
        w = _ptr(self.wd if grad else self.wf, layer * TAP)
        bias = None if grad or epi in (EPI_MASK, EPI_RES_MASK, EPI_PLAIN) else _ptr(self.p, layer * LAYER + TAP)
        _lib.check(self.L.fip_sg_conv3x3(_ptr(src), w, bias, _ptr(res) if res is not None else None,
                                         _ptr(mask) if mask is not None else None, _ptr(out), N, H, W, DIL[layer],
                                         epi, _ptr(self.err), _stream()))

    # ---- forward / backward ------------------------------------------------------------------
    def pack(self, h, qx, qy, terrain, kst, zref, no_value, N, H, W, train=False):
        b = self._buffers(N, H, W, train)
        _lib.check(self.L.fip_sg_pack_input(_ptr(h), _ptr(qx), _ptr(qy), _ptr(terrain), _ptr(kst), _ptr(zref), N, H, W,
                                            float(no_value), _ptr(b["x"]), _stream()))
        return b

    def forward(self, N, H, W, train=False):
        b = self._buffers(N, H, W, train)
        x, A, Hb = b["x"], b["a"], b["h"]
        self._conv(x, 0, EPI_BIAS_RELU, A[0], N, H, W)
        for k in range(8):
            a_in = A[k] if train else A[k % 2]
            a_out = A[k + 1] if train else A[(k + 1) % 2]
            hb = Hb[k] if train else Hb[0]
            self._conv(a_in, 1 + 2 * k, EPI_BIAS_RELU, hb, N, H, W)
            self._conv(hb, 2 + 2 * k, EPI_BIAS_RES_RELU, a_out, N, H, W, res=a_in)
        self._conv(A[8] if train else A[0], N_LAYERS - 1, EPI_HEAD, b["pred"], N, H, W)
        return b["pred"]

    def backward(self, N, H, W):
        """Gradients of the loss whose output gradient sits in g[0] (after loss()) into self.g."""
        b = self._buffers(N, H, W, True)
        A, Hb, G = b["a"], b["h"], b["g"]
        L, st, err = self.L, _stream(), _ptr(self.err)
        self.g.zero_()
        n_pix = N * (H + 2 * PAD) * (W + 2 * PAD)

        def wgrad(x, dy, layer):
            _lib.check(L.fip_sg_conv3x3_wgrad(_ptr(x), _ptr(dy), _ptr(self.g, layer * LAYER), N, H, W, DIL[layer],
                                              err, st))
            _lib.check(L.fip_sg_bias_grad(_ptr(dy), n_pix, _ptr(self.g, layer * LAYER + TAP), st))

        gout = G[0]
        wgrad(A[8], gout, N_LAYERS - 1)
        g, spare = G[1], G[2]
        self._conv(gout, N_LAYERS - 1, EPI_MASK, g, N, H, W, mask=A[8], grad=True)
        for k in range(7, -1, -1):
            l1, l2 = 1 + 2 * k, 2 + 2 * k
            wgrad(Hb[k], g, l2)
            dh = G[0]
            self._conv(g, l2, EPI_MASK, dh, N, H, W, mask=Hb[k], grad=True)
            wgrad(A[k], dh, l1)
            self._conv(dh, l1, EPI_RES_MASK, spare, N, H, W, res=g, mask=A[k], grad=True)
            g, spare = spare, g
        wgrad(b["x"], g, 0)

    def loss(self, tgt, N, H, W, dx: float = 3.0) -> None:
        """Adds the summed squared error of (dh / 0.5 m, dqx, dqy) to self.loss_acc and puts
        d(mse)/d(pred) into g[0]."""
        b = self._buffers(N, H, W, True)
        b["g"][0].zero_()
        _lib.check(self.L.fip_sg_loss(_ptr(b["pred"]), _ptr(tgt), N, H, W, float(dx), _ptr(b["e"]), _ptr(b["g"][0]),
                                      _ptr(self.loss_acc), _stream()))

    def update(self, lr=3e-4, betas=(0.9, 0.999), eps=1e-8, weight_decay=1e-4):
        self.steps += 1
        _lib.check(self.L.fip_sg_adamw(_ptr(self.p), _ptr(self.g), _ptr(self.m), _ptr(self.v), self.p.numel(), lr,
                                       betas[0], betas[1], eps, weight_decay, self.steps, _stream()))
        self.cast()

    # ---- one surrogate call ------------------------------------------------------------------
    def advance(self, state, pins=None, hmax=None, resid=None, bound=None):
        """state: dict of device tensors h, qx, qy, terrain, kst [N][H][W], zref [N], no_value;
        h/qx/qy advance by 60 s in place (hmax, if given, folds the new depths; resid, a device
        double [N], accumulates the call's consistency residual, fip_sg_consistency). bound =
        (zcap [N], excess [N] double, umax): the level bound of fip_sg_level_bound is applied to
        the new state (depths above zcap cut back, |q| <= umax h) and the depth it removed is
        added to excess. Returns the per-image depth-sum change of the inner cells (device double
        [N])."""
        h, qx, qy = state["h"], state["qx"], state["qy"]
        N, H, W = h.shape
        self.pack(h, qx, qy, state["terrain"], state["kst"], state["zref"], state["no_value"], N, H, W)
        pred = self.forward(N, H, W)
        if resid is not None:
            _lib.check(self.L.fip_sg_consistency(_ptr(pred), N, H, W, float(state.get("dx", 3.0)),
                                                 _ptr(state["terrain"]), float(state["no_value"]), _ptr(qx),
                                                 _ptr(qy), _ptr(resid), _stream()))
        dvol = self.torch.zeros(N, dtype=self.torch.float64, device=self.dev)
        fold_in_apply = hmax is not None and bound is None
        _lib.check(self.L.fip_sg_apply(_ptr(pred), N, H, W, float(state.get("dx", 3.0)), _ptr(state["terrain"]),
                                       float(state["no_value"]), _ptr(h), _ptr(qx), _ptr(qy), _ptr(dvol),
                                       _ptr(hmax) if fold_in_apply else None, _stream()))
        if bound is not None:
            zcap, excess, umax = bound
            _lib.check(self.L.fip_sg_level_bound(_ptr(h), _ptr(qx), _ptr(qy), _ptr(state["terrain"]), _ptr(zcap), N, H,
                                                 W, float(state["no_value"]), 1, float(umax), _ptr(excess),
                                                 _ptr(hmax) if hmax is not None else None, _stream()))
        sides = state.get("sides")
        if sides is not None:  # (left, right, top, bottom): 0 none, 1 close, 2 open
            _lib.check(self.L.fip_sg_edges(_ptr(h), _ptr(state["terrain"]), N, H, W, *[int(t) for t in sides],
                                           float(state["no_value"]), _stream()))
        if pins is not None:
            _lib.check(self.L.fip_sg_pin(_ptr(pins["mask"]), _ptr(pins["h"]), _ptr(pins["qx"]), _ptr(pins["qy"]),
                                         h.numel(), _ptr(h), _ptr(qx), _ptr(qy), _stream()))
        return dvol

    def pin(self, state, pins):
        """Cells held by boundary conditions get their condition's values."""
        h = state["h"]
        _lib.check(self.L.fip_sg_pin(_ptr(pins["mask"]), _ptr(pins["h"]), _ptr(pins["qx"]), _ptr(pins["qy"]),
                                     h.numel(), _ptr(h), _ptr(state["qx"]), _ptr(state["qy"]), _stream()))

    def edge_flux(self, qx, qy):
        N, H, W = qx.shape
        f = self.torch.zeros(N, dtype=self.torch.float64, device=self.dev)
        _lib.check(self.L.fip_sg_edge_flux(_ptr(qx), _ptr(qy), N, H, W, _ptr(f), _stream()))
        return f

    def target(self, s0, s1, terrain, no_value, out):
        n = s0["h"].numel()
        _lib.check(self.L.fip_sg_target(_ptr(s0["h"]), _ptr(s0["qx"]), _ptr(s0["qy"]), _ptr(s1["h"]), _ptr(s1["qx"]),
                                        _ptr(s1["qy"]), _ptr(terrain), n, float(no_value), _ptr(out), _stream()))


def bench_convs(N: int = 32, H: int = 512, W: int = 512, iters: int = 20, device: int = 0) -> dict:
    """Device time of one 64 -> 64 3x3 convolution (forward with the bias + ReLU epilogue, input
    gradient, weight gradient) on an N x H x W batch, CUDA events on the launching stream,
    after warm-up. FLOPs are the algorithmic 2 * 9 * 64 * 64 per interior pixel."""
    torch = _torch()
    net = Surrogate(device=device)
    L, st, err = net.L, _stream(), _ptr(net.err)
    b = net._buffers(N, H, W, True)
    x, y = b["a"][0], b["a"][1]
    gen = torch.Generator(device=net.dev)
    gen.manual_seed(0)
    x.copy_((torch.rand(x.shape, device=net.dev, generator=gen) - 0.5).to(torch.bfloat16))
    dw = torch.zeros(TAP, dtype=torch.float32, device=net.dev)
    flop = 2.0 * 9 * C * C * N * H * W
    res = {}
    runs = {
        "forward": lambda: L.fip_sg_conv3x3(_ptr(x), _ptr(net.wf, TAP), _ptr(net.p, LAYER + TAP), None, None, _ptr(y),
                                            N, H, W, 1, EPI_BIAS_RELU, err, st),
        "dgrad": lambda: L.fip_sg_conv3x3(_ptr(x), _ptr(net.wd, TAP), None, None, _ptr(x), _ptr(y), N, H, W, 1,
                                          EPI_MASK, err, st),
        "wgrad": lambda: L.fip_sg_conv3x3_wgrad(_ptr(x), _ptr(y), _ptr(dw), N, H, W, 1, err, st),
    }
    for name, fn in runs.items():
        for _ in range(3):
            _lib.check(fn())
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(iters):
            _lib.check(fn())
        e1.record()
        e1.synchronize()
        ms = e0.elapsed_time(e1) / iters
        res[name] = {"ms": ms, "tflops": flop / (ms * 1e-3) / 1e12}
    net.check_device()
    return res
