"""fip_rmg_step_noalloc: the rmg step for callers that cannot allocate device memory (a host
driving the step from its own loop while other streams keep the GPU busy, since cudaFree
synchronises the whole device, or a host whose memory pool owns the device). Its scratch is a
static device array, so the test checks it through the C ABI against the handle API's step
(fip_step, the same stencil kernel on the same inputs: bit for bit), on two calls in a row: the
second call must not see stale scratch from the first. Both roughness forms are covered: a kSt
grid and the uniform kSt (no grid pointer).

This file is collected last on purpose: a failure here leaves every other test already run.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

UNIFORM_KST = 33.0


def _closed_case(tmp, W, H, seed, kst_var=True):
    from fip_b200 import synth

    rng = np.random.default_rng(seed)
    y = np.arange(H, dtype=np.float32)[:, None]
    x = np.arange(W, dtype=np.float32)[None, :]
    terr = (0.3 * np.sin(x / 11.0) * np.cos(y / 9.0) + 0.001 * x).astype(np.float32)
    depth = np.clip(0.6 + 0.3 * rng.standard_normal((H, W)), 0, None).astype(np.float32)
    depth[rng.random((H, W)) < 0.2] = 0.0
    qx = (0.2 * rng.standard_normal((H, W)) * (depth > 0)).astype(np.float32)
    qy = (0.2 * rng.standard_normal((H, W)) * (depth > 0)).astype(np.float32)
    kst = np.where(rng.random((H, W)) < 0.5, 25.0, 40.0).astype(np.float32)
    files = {}
    for k, a in (("terrain", terr), ("z", terr + depth), ("qx", qx), ("qy", qy), ("kst", kst)):
        files[k] = str(tmp / f"na_{k}.bin")
        synth.write_grid(files[k], a)
    cfg = {"name": str(tmp / "na"), "terrain": [files["terrain"], 0], "z": [files["z"], 0],
           "qx": [files["qx"], 0], "qy": [files["qy"], 0],
           "W": W, "H": H, "dx": 2.0, "dt": 0.02, "duration": 100, "variable_dt": False}
    if kst_var:
        cfg["kSt_var"] = [files["kst"], 0]
    else:
        cfg["kSt"] = UNIFORM_KST
    path = str(tmp / "na.yml")
    synth.write_yaml(path, cfg)
    return path, terr, kst


@pytest.mark.parametrize("kst_var", [True, False])
def test_no_alloc_step_matches_handle_step(tmp_path, kst_var):
    import torch

    from fip_b200 import Simulation, _lib

    W, H = 1000, 150  # 3 x 5 tiles, ragged in both directions
    path, terr, kst = _closed_case(tmp_path, W, H, seed=3, kst_var=kst_var)
    sim = Simulation(path, quiet=True, all_tiles=True)
    dt = sim.time()[1]
    P = (W + 3) // 4 * 4
    dev = torch.device("cuda", 0)

    def pitched(a):
        t = torch.zeros((H + 3, P), dtype=torch.float32, device=dev)
        t[:H, :W] = torch.from_numpy(np.ascontiguousarray(a)).to(dev)
        return t

    state = [pitched(sim.field(k)) for k in ("h", "qx", "qy")]
    out = [s.clone() for s in state]  # output cells the step does not write keep the input state
    t_terr, t_kst = pitched(terr), pitched(kst)
    cfl = torch.zeros(1, dtype=torch.float32, device=dev)
    L = _lib.lib()
    ptr = lambda t: ctypes.c_void_p(t.data_ptr())
    torch.cuda.synchronize()
    for call in range(2):  # two calls in a row share the static scratch
        kst_arg = ptr(t_kst) if kst_var else None
        rc = L.fip_rmg_step_noalloc(ptr(state[0]), ptr(state[1]), ptr(state[2]), ptr(t_terr), kst_arg, UNIFORM_KST,
                                    ptr(out[0]), ptr(out[1]), ptr(out[2]), W, H, P, 2.0, dt, -9999.0, ptr(cfl),
                                    ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
        assert rc == 0, _lib.last_error()
        torch.cuda.synchronize()
        sim.step(1)
        for k, o in zip(("h", "qx", "qy"), out):
            ref = sim.field(k)
            got = o[:H, :W].cpu().numpy()
            same = ref.view(np.uint32) == got.view(np.uint32)
            assert same.all(), f"call {call} {k}: {int((~same).sum())} cells differ, max |d| = {np.abs(ref - got).max()}"
        assert float(cfl.item()) == sim.info().last_cfl
        state, out = out, [s.clone() for s in out]
    sim.close()


def test_no_alloc_rejects_grids_beyond_its_scratch():
    from fip_b200 import _lib

    L = _lib.lib()
    one = ctypes.c_void_p(16)  # never dereferenced: the size check comes first
    rc = L.fip_rmg_step_noalloc(one, one, one, one, None, 30.0, one, one, one, 480 * 200, 32 * 200, 480 * 200,
                                2.0, 0.1, -9999.0, None, None)
    assert rc == -7 and "static scratch holds at most 32768" in _lib.last_error()
