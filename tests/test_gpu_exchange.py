"""Pipelined state exchange (fip_stage_state / fip_step_exchange / fip_exchange_wait) against the
sequential calls it overlaps (fip_set_field x 3, fip_step, fip_get_field x 3): the same states,
bit for bit, whatever the copies overlap with."""
import numpy as np
import pytest

from test_gpu_parity import random_case

pytestmark = pytest.mark.gpu


def _states(W, H, n, seed):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        d = np.clip(0.4 + 0.3 * rng.standard_normal((H, W)), 0, None).astype(np.float32)
        d[rng.random((H, W)) < 0.3] = 0.0
        qx = (0.2 * rng.standard_normal((H, W)) * (d > 0)).astype(np.float32)
        qy = (0.2 * rng.standard_normal((H, W)) * (d > 0)).astype(np.float32)
        out.append((d, qx, qy))
    return out


def test_exchange_matches_sequential_calls(tmp_path):
    from fip_b200 import Simulation

    W, H, K, n = 530, 140, 37, 5
    y = random_case(tmp_path, W, H, seed=4, dt=0.02, variable_dt=True)
    states = _states(W, H, n, seed=8)
    seq = []
    with Simulation(y, quiet=True) as s:
        for st in states:
            for k, a in zip(("h", "qx", "qy"), st):
                s.set_field(k, a)
            s.step(K)
            seq.append((tuple(s.field(k) for k in ("h", "qx", "qy")), s.time()))
    outs = [tuple(np.empty((H, W), np.float32) for _ in range(3)) for _ in range(n)]
    times = []
    with Simulation(y, quiet=True) as s:
        s.stage_state(*states[0])
        for i in range(n):
            if i + 1 < n:
                s.stage_state(*states[i + 1])
            s.step_exchange(K, outs[i])
            times.append(s.time())
        s.exchange_wait()
    for i in range(n):
        assert times[i] == seq[i][1], (i, times[i], seq[i][1])
        for f in range(3):
            assert np.array_equal(outs[i][f].view(np.uint32), seq[i][0][f].view(np.uint32)), (i, f)


def test_exchange_limits(tmp_path):
    from fip_b200 import FipError, Simulation

    W, H = 64, 40
    y = random_case(tmp_path, W, H, seed=5)
    st = _states(W, H, 1, seed=1)[0]
    with Simulation(y, quiet=True) as s:
        s.stage_state(*st)
        s.stage_state(*st)
        with pytest.raises(FipError):
            s.stage_state(*st)  # two states wait already
        s.step_exchange(3)  # takes one, no download
        s.step_exchange(0)  # takes the other, runs nothing
        s.step_exchange(2)  # nothing staged: steps the current state
        s.exchange_wait()
        assert s.iteration == 5
