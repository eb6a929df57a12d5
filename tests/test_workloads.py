"""The synthetic workloads (fip_b200.synth) against the configurations they stand in for: the
1024 x 1024 plain-solver case, the 5667 x 6500 large grid and the batched ensemble, read back
through the library's own parameter-file loader (fip_config_json, no GPU)."""
import numpy as np
import pytest

from fip_b200 import config_json, synth


def _bcs(cfg):
    return {b["side"]: b for b in cfg["boundary_conditions"]}


def test_plain_solver_case(tmp_path):
    """1024 x 1024, dx 3 m; plane sloping 0.001 in -x with 40 bumps and a 30-cell, 2 m deep
    channel along y = 512; kSt 30; dry start; left z over rows 480-544 at the lowest terrain of
    those rows + 2.5 m, right open, top and bottom closed; fixed dt 0.1 s for 10 000 steps; state
    dumped every 1 000 steps."""
    sc = synth.scenario0(str(tmp_path))
    cfg = config_json(sc.yaml_path)
    assert (cfg["W"], cfg["H"], cfg["dx"], cfg["dt"]) == (1024, 1024, 3.0, pytest.approx(0.1))
    assert cfg["variable_dt"] is False and cfg["kSt"] == 30.0 and not cfg["kst_var"] and cfg["h0_sum"] == 0
    assert round(cfg["target_duration"] / 0.1) == 10000
    assert [float(t) for t in cfg["save_state"]] == [100.0 * k for k in range(1, 11)]
    b = _bcs(cfg)
    assert (b["left"]["type"], b["left"]["from"], b["left"]["to"]) == ("z", 480, 544)
    assert b["left"]["z"] == pytest.approx(float(sc.terrain[480:545, 0].min()) + 2.5, abs=1e-4)
    assert (b["right"]["type"], b["top"]["type"], b["bottom"]["type"]) == ("open", "close", "close")
    t = sc.terrain.astype(np.float64)
    # channel rows 497-526: a 2 m step at both banks
    assert np.median(t[497] - t[496]) == pytest.approx(-2.0, abs=0.05)
    assert np.median(t[527] - t[526]) == pytest.approx(2.0, abs=0.05)


def test_large_grid_case(tmp_path):
    """5667 x 6500, dx 3 m; fBm terrain with a carved channel; kSt_var 25 on a 30% mask, 40
    elsewhere; no_data -1 on about 5% of the cells along the border; variable dt; left q inflow
    over 200 cells with a triangular hydrograph 0 -> 1500 (6 h) -> 200 m3/s and the stage series
    the q type requires; bottom open; 24 simulated hours."""
    sc = synth.scenario1(str(tmp_path), seed=1)
    cfg = config_json(sc.yaml_path)
    assert (cfg["W"], cfg["H"], cfg["dx"]) == (5667, 6500, 3.0)
    assert cfg["variable_dt"] is True and cfg["kst_var"] and cfg["target_duration"] == 86400.0
    assert cfg["no_data"] == -1.0
    nd = sc.terrain == -1.0
    assert 0.03 < nd.mean() < 0.07
    assert not nd[: 6500 // 2, : 5667 // 2].any()  # a border band (top and right edges)
    k = sc.kst_var
    assert set(np.unique(k).tolist()) == {25.0, 40.0} and abs(float((k == 25.0).mean()) - 0.3) < 0.01
    b = _bcs(cfg)
    left = b["left"]
    assert left["type"] == "q" and left["series"] and left["to"] - left["from"] + 1 == 200
    qt, qv = np.array(left["q_t"]), np.array(left["q_v"])
    assert qv[0] == 0.0 and qv.max() == pytest.approx(1500.0) and qt[qv.argmax()] == 6 * 3600.0
    assert qv[-1] == pytest.approx(200.0) and qt[-1] == 86400.0
    assert len(left["z_t"]) == len(qt) and b["bottom"]["type"] == "open"
    assert set(b) == {"left", "bottom"}


def test_ensemble_members(tmp_path):
    """Members of the batched ensemble: W, H ~ U[256, 2048], own fBm terrain, uniform kSt ~
    U[20, 45], q inflow with a hydrograph peaking at U[200, 2000] m3/s at U[1, 8] h, variable dt,
    6 simulated hours (the first 8 of the 64 seeded members)."""
    members = synth.ensemble2(str(tmp_path), n=8)
    sizes = set()
    for sc in members:
        cfg = config_json(sc.yaml_path)
        assert 256 <= cfg["W"] <= 2048 and 256 <= cfg["H"] <= 2048
        sizes.add((cfg["W"], cfg["H"]))
        assert 20.0 <= cfg["kSt"] <= 45.0 and not cfg["kst_var"]
        assert cfg["variable_dt"] is True and cfg["target_duration"] == 6 * 3600.0
        left = _bcs(cfg)["left"]
        assert left["type"] == "q" and left["series"]
        qt, qv = np.array(left["q_t"]), np.array(left["q_v"])
        peak, t_peak = sc.info["q_peak"], sc.info["t_peak"]
        assert 200.0 <= peak <= 2000.0 and 3600.0 <= t_peak <= 8 * 3600.0
        assert qv[0] == 0.0 and qv.max() <= peak * (1 + 1e-6)
    assert len(sizes) == len(members)  # uneven sizes
    assert len({round(float(sc.terrain[5, 5]), 4) for sc in members}) == len(members)  # own terrains
