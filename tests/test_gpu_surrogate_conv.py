"""tcgen05 BF16 3x3 convolutions of the surrogate (fip_sg_conv3x3, fip_sg_conv3x3_wgrad) against
the FP64 CPU oracle (oracle/conv_oracle.py), through the C ABI. Inputs are bf16-exact, the
kernels accumulate in fp32; tolerances: bf16 outputs within 1% of the output scale, fp32
outputs (head, weight gradient) within 0.1%."""
import ctypes

import numpy as np
import pytest

import conv_oracle
from fip_b200 import _lib

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _L():
    return _lib.lib()


def _bf16(a):
    return torch.from_numpy(np.ascontiguousarray(a, np.float32)).to(torch.bfloat16)


def _dev_padded(x):  # unpadded NHWC float -> padded bf16 device tensor
    return _bf16(conv_oracle.pad(x)).cuda().contiguous()


P = conv_oracle.PAD


def _unpad(t):
    return t.float().cpu().numpy()[:, P:-P, P:-P, :]


def _border_zero(o):
    return (np.all(o[:, :P] == 0) and np.all(o[:, -P:] == 0) and np.all(o[:, :, :P] == 0)
            and np.all(o[:, :, -P:] == 0))


def _check_err(err):
    torch.cuda.synchronize()
    assert int(err.item()) == 0, f"device wait ran out: code {int(err.item())}"


SHAPES = [(2, 11, 37), (1, 64, 64), (3, 30, 130)]
DILS = [1, 2, 8]


@pytest.mark.parametrize("dil", DILS)
@pytest.mark.parametrize("N,H,W", SHAPES)
def test_forward_epilogues(N, H, W, dil):
    L = _L()
    rng = np.random.default_rng(N * 1000 + H * 10 + W)
    x = np.float32(_bf16(rng.standard_normal((N, H, W, 64)) * 0.5).float().numpy())
    w = np.float32(_bf16(rng.standard_normal((9, 64, 64)) * 0.06).float().numpy())
    res = np.float32(_bf16(rng.standard_normal((N, H, W, 64)) * 0.5).float().numpy())
    bias = (rng.standard_normal(64) * 0.1).astype(np.float32)
    ref = conv_oracle.conv3x3(x, w, dil)
    dx_, dw_, dres = _dev_padded(x), _bf16(w).cuda(), _dev_padded(res)
    db = torch.from_numpy(bias).cuda()
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    Hp, Wp = H + 2 * P, W + 2 * P
    for epi, expect in ((5, ref), (0, np.maximum(ref + bias, 0)), (1, np.maximum(ref + bias + res, 0)),
                        (3, ref * (res > 0)), (4, (ref + res) * (res > 0))):
        out = torch.full((N, Hp, Wp, 64), 7.0, dtype=torch.bfloat16, device="cuda")
        rc = L.fip_sg_conv3x3(dx_.data_ptr(), dw_.data_ptr(), db.data_ptr(), dres.data_ptr(), dres.data_ptr(),
                              out.data_ptr(), N, H, W, dil, epi, err.data_ptr(), None)
        assert rc == 0, _lib.last_error()
        _check_err(err)
        o = out.float().cpu().numpy()
        assert _border_zero(o)
        scale = max(1e-6, float(np.max(np.abs(expect))))
        got = o[:, P:-P, P:-P]
        assert np.max(np.abs(got - expect)) <= 1e-2 * scale, (epi, np.max(np.abs(got - expect)))
    head = torch.full((N, Hp, Wp, 4), 7.0, dtype=torch.float32, device="cuda")
    rc = L.fip_sg_conv3x3(dx_.data_ptr(), dw_.data_ptr(), db.data_ptr(), None, None, head.data_ptr(), N, H, W, dil, 2,
                          err.data_ptr(), None)
    assert rc == 0
    _check_err(err)
    hd = head.cpu().numpy()
    exp_h = ref[..., :4] + bias[:4]
    assert np.max(np.abs(hd[:, P:-P, P:-P] - exp_h)) <= 1e-3 * np.max(np.abs(exp_h))
    assert _border_zero(hd)


@pytest.mark.parametrize("dil", DILS)
@pytest.mark.parametrize("N,H,W", SHAPES)
def test_dgrad_and_wgrad(N, H, W, dil):
    L = _L()
    rng = np.random.default_rng(7 + N + H + W)
    x = np.float32(_bf16(rng.standard_normal((N, H, W, 64)) * 0.5).float().numpy())
    g = np.float32(_bf16(rng.standard_normal((N, H, W, 64)) * 0.5).float().numpy())
    w = np.float32(_bf16(rng.standard_normal((9, 64, 64)) * 0.06).float().numpy())
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    # dgrad = forward convolution of dy with the flipped, transposed weights
    wd = conv_oracle.dgrad_weights(w)
    # keep every device tensor referenced until the kernels ran (a freed temporary's memory is
    # handed to the next allocation)
    dg, dwd, dxx = _dev_padded(g), _bf16(wd).cuda(), _dev_padded(x)
    out = torch.empty((N, H + 2 * P, W + 2 * P, 64), dtype=torch.bfloat16, device="cuda")
    rc = L.fip_sg_conv3x3(dg.data_ptr(), dwd.data_ptr(), None, None, None, out.data_ptr(),
                          N, H, W, dil, 5, err.data_ptr(), None)
    assert rc == 0
    _check_err(err)
    # the oracle's dgrad: adjoint of the forward convolution, checked through <conv(x), g> = <x, dgrad(g)>
    ref_dx = conv_oracle.conv3x3(g, wd, dil)
    assert abs(np.sum(conv_oracle.conv3x3(x, w, dil) * g) - np.sum(x * ref_dx)) < 1e-6 * np.sum(np.abs(x * ref_dx))
    assert np.max(np.abs(_unpad(out) - ref_dx)) <= 1e-2 * np.max(np.abs(ref_dx))
    dw = torch.zeros((9, 64, 64), dtype=torch.float32, device="cuda")
    rc = L.fip_sg_conv3x3_wgrad(dxx.data_ptr(), dg.data_ptr(), dw.data_ptr(), N, H, W, dil, err.data_ptr(), None)
    assert rc == 0, _lib.last_error()
    _check_err(err)
    ref_dw = conv_oracle.wgrad(x, g, dil)
    assert np.max(np.abs(dw.cpu().numpy() - ref_dw)) <= 1e-3 * np.max(np.abs(ref_dw))
