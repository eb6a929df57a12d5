"""Known-answer properties of the CPU oracle itself (no reference run needed)."""
import numpy as np
import pytest

import pyoracle


def _closed_box(W, H, seed, precision, wet=True):
    rng = np.random.default_rng(seed)
    y = np.arange(H, dtype=np.float32)[:, None]
    x = np.arange(W, dtype=np.float32)[None, :]
    terr = (0.05 * np.sin(x / 5.0) + 0.04 * np.cos(y / 7.0)).astype(np.float32)
    h0 = np.maximum(0.0, 0.6 + 0.2 * rng.standard_normal((H, W)) * wet).astype(np.float32)
    o = pyoracle.Oracle(W, H, ((W * 4 + 511) // 512) * 128, 2.0, 0.05, False, 30.0, -9999.0, terr, h0,
                        None, None, None, precision=precision)
    return o, terr, h0


@pytest.mark.parametrize("precision", [64, 32])
def test_lake_at_rest(precision):
    """A flat water surface over uneven terrain stays at rest (pressure balances bed slope)."""
    W, H = 40, 36
    y = np.arange(H, dtype=np.float32)[:, None]
    x = np.arange(W, dtype=np.float32)[None, :]
    terr = (0.3 * np.sin(x / 4.0) * np.cos(y / 6.0)).astype(np.float32)
    h0 = (1.5 - terr).astype(np.float32)
    o = pyoracle.Oracle(W, H, 128, 3.0, 0.1, False, 30.0, -9999.0, terr, h0, None, None, None,
                        precision=precision)
    o.simulate(200)
    h = o.field(pyoracle.F_H)
    tol = 2.5e-7 if precision == 64 else 2e-5  # fp64: one float32 ulp at 1.5 m after read-out
    assert np.max(np.abs(h - h0)[1:-1, 1:-1]) < tol
    assert np.max(np.abs(o.field(pyoracle.F_QX))) < (1e-6 if precision == 64 else 1e-4)  # float32 inputs


def test_closed_box_conserves_volume():
    """Without boundary conditions the domain edges are walls: total volume is conserved."""
    o, _, _ = _closed_box(48, 44, 3, 64)
    v0 = o.volume()
    o.simulate(300)
    assert abs(o.volume() - v0) / v0 < 1e-10


def test_dt_controller_step_sequence():
    """controlTimestep: +0.1 % per step while below half the CFL minimum (at most 1 s)."""
    o, _, _ = _closed_box(32, 30, 1, 64, wet=False)
    o2 = pyoracle.Oracle(32, 30, 128, 2.0, 0.1, True, 30.0, -9999.0, o.terrain,
                         np.zeros((30, 32), np.float32), None, None, None)
    dts = []
    for _ in range(5):
        o2.simulate(1)
        dts.append(o2.dt)
    exp = []
    d = np.float32(0.1)
    for _ in range(6):
        d = np.float32(d * np.float32(1.001))
        exp.append(float(d))
    assert dts == exp[:5]  # controlTimestep runs at the start of each simulate()


def test_read_series_formats(tmp_path):
    p = tmp_path / "s.csv"
    p.write_text("time;value\n0;1\n10.5;2\n20;3\n")
    t, v = pyoracle.read_series(str(p), 0, 1)
    assert list(t) == [0.0, 10.5, 20.0] and list(v) == [1.0, 2.0, 3.0]
    p2 = tmp_path / "d.csv"
    p2.write_text("when;q\n14.07.2021 00:00:00;5\n14.07.2021 01:00:00;7\n")
    t, v = pyoracle.read_series(str(p2), 0, 1)
    assert list(t) == [0.0, 3600.0] and list(v) == [5.0, 7.0]
