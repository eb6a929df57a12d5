"""What the trained network gains over the method without it: trained for a few hundred steps on
trajectories the batched solver generates, the surrogate's 60-s prediction of the water depth
on held-out scenarios must beat persistence (no change over the call, the untrained network's
output) by a clear margin, and its closed-loop depth after several calls too."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
pytest.importorskip("torch")


def test_trained_network_beats_persistence(tmp_path):
    from fip_b200 import surrogate_run as sr
    from fip_b200.surrogate import Surrogate

    tr = sr.config3_members(str(tmp_path), 8, 256, seed=11, duration=1800.0)
    btr = sr.Batch(tr)
    snaps, _, _ = sr.solver_trajectories(tr, 20)
    net = Surrogate(seed=3)
    log, _ = sr.train(net, btr, snaps, 300, bs=8, lr=1e-3, log_every=100)
    assert log[-1][1] < log[0][1]
    ev = sr.config3_members(str(tmp_path), 4, 256, seed=12, duration=1800.0)
    bev = sr.Batch(ev)
    esn, _, _ = sr.solver_trajectories(ev, 20)
    one = sr.evaluate_one_call(net, bev, esn)
    assert one["rmse_depth_net_m"] < 0.95 * one["rmse_depth_persistence_m"], one
    st, _, _, _, _, _ = sr.rollout(net, bev, 5, esn["h"][0], esn["qx"][0], esn["qy"][0])
    ref = esn["h"][5].cpu().numpy().astype(np.float64)
    got = st["h"].cpu().numpy()
    pers = esn["h"][0].cpu().numpy()
    assert np.sqrt(np.mean((got - ref) ** 2)) < np.sqrt(np.mean((pers - ref) ** 2)), "5-call rollout"
