"""Failure detection on the device without a GPU fault: every shared-memory wait of the stencil
has a 2-s limit, after which the kernel records FIP_DEVERR_* in the control block and returns.
The test hook fip_inject_wait_timeout makes one CTA leave its first row unstaged (a barrier that
nothing completes); the step must come back with FIP_ERR_DEVICE_TIMEOUT within seconds, and the
CUDA context must stay usable: a new handle on the same device runs and matches a clean run."""
import time

import numpy as np
import pytest

from fip_b200 import FipError, Simulation, _lib, synth

pytestmark = pytest.mark.gpu


def test_wait_timeout_is_reported_and_context_survives(tmp_path):
    sc = synth.scenario1(str(tmp_path), W=512, H=384, seed=6, duration=3600.0, name="f")
    with Simulation(sc.yaml_path, quiet=True, all_tiles=True) as a:
        a.step(20)
        a.inject_wait_timeout()
        t0 = time.perf_counter()
        with pytest.raises(FipError) as e:
            a.step(5)
        assert e.value.code == _lib.FIP_ERR_DEVICE_TIMEOUT
        assert time.perf_counter() - t0 < 30.0
    with Simulation(sc.yaml_path, quiet=True, all_tiles=True) as b:
        b.step(40)
        got = {k: b.field(k) for k in ("h", "qx", "qy")}
    with Simulation(sc.yaml_path, quiet=True, all_tiles=True) as c:
        c.step(40)
        ref = {k: c.field(k) for k in ("h", "qx", "qy")}
    for k in ref:
        assert np.array_equal(got[k], ref[k]), k
