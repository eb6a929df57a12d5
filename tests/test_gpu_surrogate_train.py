"""Training kernels of the surrogate: forward pass, loss and every parameter gradient of the
18-layer network (dilated convolutions, mass-conserving flux head) against the FP64 CPU oracle
(oracle/surrogate_oracle.py), and a short training run that must reduce the loss."""
import numpy as np
import pytest

import surrogate_oracle as so

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _bf16_round(a):
    return torch.from_numpy(np.ascontiguousarray(a, np.float32)).to(torch.bfloat16).float().numpy()


def _net(seed):
    from fip_b200 import surrogate

    p = surrogate.init_params(seed)
    rng = np.random.default_rng(seed + 1)
    L = so.LAYER
    # a non-zero head and biases so that every gradient path carries signal
    p[17 * L:17 * L + so.TAP] = (rng.standard_normal(so.TAP) * 0.02).astype(np.float32)
    for l in range(18):
        p[l * L + so.TAP:(l + 1) * L] = (rng.standard_normal(64) * 0.05).astype(np.float32)
    for l in range(18):  # the GPU computes with bf16 weights: compare on the same weights
        p[l * L:l * L + so.TAP] = _bf16_round(p[l * L:l * L + so.TAP])
    return p


def test_gradients_match_fp64_oracle():
    from fip_b200.surrogate import Surrogate

    N, H, W = 2, 12, 14
    rng = np.random.default_rng(3)
    p = _net(5)
    x = np.zeros((N, H, W, 64), np.float32)
    x[..., :6] = _bf16_round(rng.standard_normal((N, H, W, 6)) * 0.7)
    tgt = (rng.standard_normal((N, H, W, 3)) * 0.1).astype(np.float32)
    net = Surrogate(params=p)
    b = net._buffers(N, H, W, True)
    xp = np.pad(x, ((0, 0), (8, 8), (8, 8), (0, 0)))
    b["x"].copy_(torch.from_numpy(xp).to(torch.bfloat16))
    pred = net.forward(N, H, W, train=True)
    dt = torch.from_numpy(tgt).cuda()
    net.loss_acc.zero_()
    net.loss(dt, N, H, W)
    net.backward(N, H, W)
    net.check_device()
    ref_loss, ref_g, ref_pred = so.loss_and_grads(p.astype(np.float64), x.astype(np.float64), tgt.astype(np.float64))
    got_pred = pred.cpu().numpy()[:, 8:-8, 8:-8, :4]
    assert np.max(np.abs(got_pred - ref_pred[..., :4])) <= 0.02 * np.max(np.abs(ref_pred[..., :4]))
    got_loss = float(net.loss_acc.item()) / tgt.size
    assert abs(got_loss - ref_loss) <= 0.02 * ref_loss
    g = net.g.cpu().numpy().astype(np.float64)
    # activations and gradients are stored in bf16 (8-bit mantissa) between all 18 layers, and
    # the head's continuity operator scales the output gradient by 60 s / dx / 0.5 m = 40: each
    # layer's gradient must agree with the FP64 oracle to 10% (relative L2 norm)
    for l in range(18):
        sl = slice(l * so.LAYER, (l + 1) * so.LAYER)
        num = np.linalg.norm(g[sl] - ref_g[sl])
        den = np.linalg.norm(ref_g[sl])
        assert num <= 0.10 * den, (l, num / den)


def test_training_reduces_loss():
    from fip_b200.surrogate import Surrogate

    N, H, W = 4, 32, 40
    rng = np.random.default_rng(9)
    x = np.zeros((N, H + 16, W + 16, 64), np.float32)
    x[:, 8:-8, 8:-8, :6] = rng.standard_normal((N, H, W, 6)) * 0.5
    # a smooth function of the inputs the network can fit
    xi = x[:, 8:-8, 8:-8]
    tgt = np.stack([np.tanh(xi[..., 0] + xi[..., 2]), 0.5 * xi[..., 3], -0.3 * xi[..., 4]], -1).astype(np.float32)
    net = Surrogate(seed=1)
    b = net._buffers(N, H, W, True)
    b["x"].copy_(torch.from_numpy(x).to(torch.bfloat16))
    dt = torch.from_numpy(tgt).cuda()
    losses = []
    for it in range(120):
        net.forward(N, H, W, train=True)
        net.loss_acc.zero_()
        net.loss(dt, N, H, W)
        net.backward(N, H, W)
        net.update(lr=2e-3)
        if it % 20 == 0 or it == 119:
            losses.append(float(net.loss_acc.item()) / tgt.size)
    net.check_device()
    assert losses[-1] < 0.2 * losses[0], losses


def test_consistency_indicator_matches_oracle():
    """fip_sg_consistency (the fallback indicator) against its FP64 restatement."""
    import ctypes

    from fip_b200 import _lib

    N, H, W = 3, 37, 29
    rng = np.random.default_rng(11)
    pred = (rng.standard_normal((N, H + 16, W + 16, 4)) * 0.3).astype(np.float32)
    pred[:, :8] = pred[:, -8:] = 0.0  # the network output's zero border
    pred[:, :, :8] = pred[:, :, -8:] = 0.0
    qx = (rng.standard_normal((N, H, W)) * 0.5).astype(np.float32)
    qy = (rng.standard_normal((N, H, W)) * 0.5).astype(np.float32)
    terr = rng.standard_normal((N, H, W)).astype(np.float32)
    terr[1, 10:13, 5:9] = -9999.0
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    res = torch.zeros(N, dtype=torch.float64, device="cuda")
    p = lambda t: ctypes.c_void_p(t.data_ptr())
    tp, tq, tr, tt = dev(pred), dev(qx), dev(qy), dev(terr)
    rc = _lib.lib().fip_sg_consistency(p(tp), N, H, W, 3.0, p(tt), -9999.0, p(tq), p(tr), p(res),
                                       ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == 0, _lib.last_error()
    ref = so.consistency(pred[:, 8:-8, 8:-8].astype(np.float64), qx, qy, terr, -9999.0)
    got = res.cpu().numpy()
    assert np.allclose(got, ref, rtol=1e-5), (got, ref)


def test_level_bound_matches_oracle():
    """fip_sg_level_bound (the rollout limiter and mass residual) against its restatement."""
    import ctypes

    from fip_b200 import _lib

    N, H, W = 3, 33, 41
    rng = np.random.default_rng(7)
    terr = rng.uniform(0.0, 3.0, (N, H, W)).astype(np.float32)
    terr[2, 5:8, 9:12] = -9999.0
    h = rng.uniform(0.0, 4.0, (N, H, W)).astype(np.float32)
    qx = (rng.standard_normal((N, H, W)) * 20).astype(np.float32)
    qy = (rng.standard_normal((N, H, W)) * 20).astype(np.float32)
    zcap = np.array([3.5, 2.0, 4.2], np.float32)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    th, tqx, tqy, tt, tz = dev(h), dev(qx), dev(qy), dev(terr), dev(zcap)
    ex = torch.zeros(N, dtype=torch.float64, device="cuda")
    p = lambda t: ctypes.c_void_p(t.data_ptr())
    rc = _lib.lib().fip_sg_level_bound(p(th), p(tqx), p(tqy), p(tt), p(tz), N, H, W, -9999.0, 1, 10.0, p(ex), None,
                                       ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == 0, _lib.last_error()
    rh, rqx, rqy, rex = so.level_bound(h, qx, qy, terr, zcap, -9999.0, 10.0)
    assert np.array_equal(th.cpu().numpy(), rh)
    assert np.array_equal(tqx.cpu().numpy(), rqx) and np.array_equal(tqy.cpu().numpy(), rqy)
    assert np.allclose(ex.cpu().numpy(), rex, rtol=1e-9)
