"""GPU parity of the sm_100a solver, through the C ABI (fip_b200.Simulation -> libfip_b200.so).

* against the reference binary's own dumps and sampling rows (tests/golden/*.npz), with the
  accuracy gates: |dz| <= 1e-4 m, |dq| <= 1e-4 m^2/s (plus a relative term for the reference's
  pitch-scaled top/bottom outflow, whose depths reach hundreds of metres), identical wet sets and
  the same step count;
* against the CPU oracle (FP32 and FP64 builds) on random wet states with every boundary type,
  several tiles and ragged sizes, for the current state, the ping-pong partner and hmax;
* dry-tile skipping and graph batching against the all-tiles / eager runs: bit-identical.
"""
import glob
import os

import numpy as np
import pytest

import plan_rule
import pyoracle
from golden_util import Golden, cases

pytestmark = pytest.mark.gpu

KINDS = ("ah", "qx", "qy", "flood_plains")


def _sim(*a, **k):
    from fip_b200 import Simulation

    return Simulation(*a, **k)


def _read_dump(path):
    with open(path, "rb") as f:
        w, h = np.frombuffer(f.read(16), dtype=np.uint64)
        return np.frombuffer(f.read(), dtype=np.float32).reshape(int(h), int(w))


def _close(ref, got, atol=1e-4, rtol=1e-6):
    d = np.abs(ref.astype(np.float64) - got.astype(np.float64))
    return float(np.nanmax(d)) if d.size else 0.0, bool(np.all(d <= atol + rtol * np.abs(ref)))


@pytest.mark.parametrize("name", cases())
def test_matches_reference_binary(name, tmp_path):
    g = Golden(name)
    y = g.materialize(str(tmp_path))
    samples = tmp_path / "samples.csv"
    sim = _sim(y, sample_path=str(samples))
    assert sim.pitch == g.pitch_elems  # same cudaMallocPitch row pitch as the reference
    sim.run()
    it = sim.iteration
    sim.close()
    assert it == int(g.meta["stderr"].split("Finished ")[1].split(" ")[0])
    prefix = os.path.join(str(tmp_path), os.path.basename(g.meta["name"]))
    exact = total = 0
    for t in g.dump_times():
        for kind in KINDS:
            files = glob.glob(f"{prefix}_{kind}_{t}_*")
            assert len(files) == 1, (kind, t, files)
            got = _read_dump(files[0])
            ref = g.dump(kind, t)
            worst, ok = _close(ref, got)
            assert ok, f"{name} t={t} {kind}: max |d| = {worst}"
            exact += int(np.sum(ref.view(np.uint32) == got.view(np.uint32)))
            total += ref.size
            if kind == "ah":
                assert np.array_equal(ref > 1e-6, got > 1e-6)
    ref_rows = [r for r in g.stdout.split("\n") if r]
    got_rows = [r for r in samples.read_text().split("\n") if r] if ref_rows else []
    assert len(ref_rows) == len(got_rows)
    for a, b in zip(ref_rows[1:], got_rows[1:]):
        va = [float(x) for x in a.split(";") if x]
        vb = [float(x) for x in b.split(";") if x]
        assert va[0] == vb[0] and np.allclose(va[1:], vb[1:], atol=1e-4, rtol=1e-6)
    print(f"{name}: {exact}/{total} dumped values bit-identical to the reference")


def random_case(tmp, W, H, seed, bcs=None, kst_var=True, no_data=True, dt=0.02, variable_dt=False,
                name="rnd", kst_zero=0.0):
    """Wet start with random velocities, terrain relief, kSt_var (a fraction kst_zero of it 0:
    infinite friction), no_data holes."""
    from fip_b200 import synth

    rng = np.random.default_rng(seed)
    y = np.arange(H, dtype=np.float32)[:, None]
    x = np.arange(W, dtype=np.float32)[None, :]
    terr = (0.4 * np.sin(x / 9.0 + seed) * np.cos(y / 7.0) + 0.002 * x).astype(np.float32)
    depth = np.clip(0.5 + 0.4 * rng.standard_normal((H, W)), 0, None).astype(np.float32)
    depth[rng.random((H, W)) < 0.15] = 0.0
    qx = (0.3 * rng.standard_normal((H, W)) * (depth > 0)).astype(np.float32)
    qy = (0.3 * rng.standard_normal((H, W)) * (depth > 0)).astype(np.float32)
    if no_data:  # holes away from the border band the boundary conditions write
        hole = rng.random((H, W)) < 0.02
        hole[:3, :] = hole[-3:, :] = False
        hole[:, :3] = hole[:, -3:] = False
        terr[hole] = -9999.0
    files = {}
    for k, a in (("terrain", terr), ("z", terr + depth), ("qx", qx), ("qy", qy)):
        files[k] = str(tmp / f"{name}_{k}.bin")
        synth.write_grid(files[k], a)
    cfg = {"name": str(tmp / name), "terrain": [files["terrain"], 0], "z": [files["z"], 0],
           "qx": [files["qx"], 0], "qy": [files["qy"], 0], "W": W, "H": H, "dx": 2.0, "dt": dt,
           "duration": 1000, "variable_dt": variable_dt}
    if kst_var:
        k = np.where(rng.random((H, W)) < 0.4, 25.0, 40.0).astype(np.float32)
        if kst_zero:
            k[rng.random((H, W)) < kst_zero] = 0.0
        files["kst"] = str(tmp / f"{name}_kst.bin")
        synth.write_grid(files["kst"], k)
        cfg["kSt_var"] = [files["kst"], 0]
    else:
        cfg["kSt"] = 33
    if bcs is None:
        bcs = [{"side": "left", "type": "z", "z": float(terr[H // 2, 0] + 0.8), "from": 1, "to": H - 2},
               {"side": "right", "type": "open"},
               {"side": "top", "type": "close"},
               {"side": "bottom", "type": "close", "from": 2, "to": W - 3}]
    cfg["boundary_conditions"] = bcs
    path = str(tmp / f"{name}.yml")
    synth.write_yaml(path, cfg)
    return path


FIELDS = (("h", pyoracle.F_H), ("qx", pyoracle.F_QX), ("qy", pyoracle.F_QY), ("h_prev", pyoracle.F_H_OTHER),
          ("qx_prev", pyoracle.F_QX_OTHER), ("qy_prev", pyoracle.F_QY_OTHER), ("hmax", pyoracle.F_HMAX))


@pytest.mark.parametrize("W,H,steps", [(100, 90, 150), (1000, 100, 120), (481, 33, 101), (37, 5, 60), (4, 4, 30),
                                       (131, 70, 205)])
def test_matches_oracle_random_state(W, H, steps, tmp_path):
    y = random_case(tmp_path, W, H, seed=W * 7 + H)
    sim = _sim(y, quiet=True)
    sim.step(steps)
    got = {k: sim.field(k) for k, _ in FIELDS}
    vol = sim.volume()
    pitch = sim.pitch
    sim.close()
    # FP32 oracle: every field within the gates, identical wet set
    o = pyoracle.Oracle.from_yaml(y, pitch, precision=32)
    o.simulate(steps)
    for k, which in FIELDS:
        worst, ok = _close(o.field(which), got[k], atol=1e-4, rtol=1e-5)
        assert ok, f"fp32 {k}: max |d| = {worst}"
    assert np.array_equal(o.field(pyoracle.F_H) > 1e-6, got["h"] > 1e-6)
    # FP64 oracle: total volume within 1e-6 relative; fields only loosely (the white-noise start
    # puts some upwind switches at near-ties, where FP32 and FP64 can take different branches)
    o = pyoracle.Oracle.from_yaml(y, pitch, precision=64)
    o.simulate(steps)
    assert abs(vol - o.volume()) <= 1e-6 * abs(o.volume())
    worst, ok = _close(o.field(pyoracle.F_H), got["h"], atol=2e-2, rtol=0)
    assert ok, f"fp64 h: max |d| = {worst}"


def test_infinite_friction_matches_oracle(tmp_path):
    """kSt_var with zeros (5% of the cells): dt G / kSt^2 is infinite there, the reference's
    select gives a friction factor of 0 where both discharges vanish and an infinite one (the
    discharge becomes 0) elsewhere. Against the FP32 oracle."""
    W, H, steps = 300, 70, 120
    y = random_case(tmp_path, W, H, seed=41, kst_zero=0.05)
    sim = _sim(y, quiet=True)
    sim.step(steps)
    got = {k: sim.field(k) for k, _ in FIELDS}
    pitch = sim.pitch
    sim.close()
    o = pyoracle.Oracle.from_yaml(y, pitch, precision=32)
    o.simulate(steps)
    for k, which in FIELDS:
        worst, ok = _close(o.field(which), got[k], atol=1e-4, rtol=1e-5)
        assert ok, f"fp32 {k}: max |d| = {worst}"
    assert np.array_equal(o.field(pyoracle.F_H) > 1e-6, got["h"] > 1e-6)


def test_pitch_scaled_open_outflow(tmp_path):
    """The reference's open boundary on the top/bottom sides multiplies the outflow by the row
    pitch (sign = idx - idx_neighbor); the resulting strong sink is reproduced (FP32 oracle, the
    dynamics there are too sensitive for an FP64 comparison)."""
    bcs = [{"side": "bottom", "type": "open", "from": 2}, {"side": "top", "type": "open"},
           {"side": "left", "type": "close"}]
    y = random_case(tmp_path, 96, 70, seed=9, bcs=bcs)
    sim = _sim(y, quiet=True)
    sim.step(60)
    got = {k: sim.field(k) for k, _ in FIELDS}
    pitch = sim.pitch
    sim.close()
    o = pyoracle.Oracle.from_yaml(y, pitch, precision=32)
    o.simulate(60)
    assert got["h"].min() < -1.0  # the sink drives row 1 far below zero depth
    for k, which in FIELDS:
        worst, ok = _close(o.field(which), got[k], atol=1e-4, rtol=1e-5)
        assert ok, f"{k}: max |d| = {worst}"


@pytest.mark.parametrize("bc_type", ["z", "q", "close", "open"])
@pytest.mark.parametrize("side", ["left", "right", "top", "bottom"])
def test_boundary_fragments(side, bc_type, tmp_path):
    """Each side x type alone (constant values) against the oracle."""
    W, H = 70, 64
    bc = {"side": side, "type": bc_type}
    if bc_type in ("z", "q"):
        bc["z"] = 1.2
    if bc_type == "q":
        bc["q"] = 3.0
    y = random_case(tmp_path, W, H, seed=5, bcs=[bc], kst_var=False, no_data=False)
    sim = _sim(y, quiet=True)
    sim.step(80)
    got = {k: sim.field(k) for k, _ in FIELDS[:3]}
    pitch = sim.pitch
    sim.close()
    o = pyoracle.Oracle.from_yaml(y, pitch, precision=32)
    o.simulate(80)
    for k, which in FIELDS[:3]:
        worst, ok = _close(o.field(which), got[k], atol=1e-4, rtol=1e-5)
        assert ok, f"{side}/{bc_type} {k}: max |d| = {worst}"


def test_dry_tile_skipping_is_exact(tmp_path):
    """Dry-start scenario on a grid of many tiles: skipping quiescent tiles changes no bit."""
    from fip_b200 import synth

    sc = synth.scenario0(str(tmp_path), W=1500, H=700, duration=60, save_every=0, name="skip",
                         bc_rows=(300, 360))
    res = []
    for all_tiles, graphs in ((True, False), (False, True), (False, False)):
        sim = _sim(sc.yaml_path, quiet=True, all_tiles=all_tiles, use_graphs=graphs)
        sim.step(250)
        inf = sim.info()
        res.append(({k: sim.field(k) for k, _ in FIELDS}, inf.active_tiles, inf.n_tiles))
        sim.close()
    ref = res[0][0]
    for fields, active, n in res[1:]:
        assert active < n  # some tiles were skipped
        for k, _ in FIELDS:
            assert np.array_equal(ref[k].view(np.uint32), fields[k].view(np.uint32)), k


def test_dry_tile_skipping_across_strip_edges(tmp_path):
    """Water short of the edge bands of a strip on either side (the first and last thread's four
    columns of a 480-column tile, which hold the two columns the stencil reaches), and a pond
    across a strip edge: the strip beside a pond is planned only once water reaches its facing
    band. The plan of the second step has exactly the tiles that rule names (fewer than "any
    nonzero cell in the 3 x 3 tile neighbourhood" would), and runs with dry-tile skipping stay
    bit-identical to every-tile runs while the fronts cross the strip edges."""
    from fip_b200 import synth

    W, H = 1500, 192
    y = np.arange(H, dtype=np.float32)[:, None]
    x = np.arange(W, dtype=np.float32)[None, :]
    terr = (0.05 * np.sin(x / 29.0) * np.cos(y / 17.0)).astype(np.float32)
    depth = np.zeros((H, W), np.float32)
    depth[40:80, 466:474] = 1.0      # after one step still west of strip 0's east band (476-479)
    depth[100:140, 966:980] = 0.9    # after one step still east of strip 2's west band (960-963)
    depth[150:170, 478:490] = 0.7    # across the edge of strips 0 and 1
    files = {}
    for k, a in (("terrain", terr), ("z", terr + depth)):
        files[k] = str(tmp_path / f"e_{k}.bin")
        synth.write_grid(files[k], a)
    cfg = {"name": str(tmp_path / "e"), "terrain": [files["terrain"], 0], "z": [files["z"], 0], "W": W, "H": H,
           "dx": 2.0, "dt": 0.05, "duration": 1000, "kSt": 30, "variable_dt": False}
    path = str(tmp_path / "e.yml")
    synth.write_yaml(path, cfg)
    res = []
    for all_tiles, graphs in ((True, False), (False, True), (False, False)):
        sim = _sim(path, quiet=True, all_tiles=all_tiles, use_graphs=graphs)
        sim.step(1)
        st = {k: sim.field(k) for k, _ in FIELDS}
        planned = sim.info().active_tiles  # plan of step 2
        sim.step(239)
        res.append(({k: sim.field(k) for k, _ in FIELDS}, st, planned, sim.info().n_tiles))
        sim.close()
    ref = res[0][0]
    # both fronts crossed into strip 1
    assert float(np.abs(ref["h"][40:80, 480:482]).max()) > 0 and float(np.abs(ref["h"][100:140, 958:960]).max()) > 0
    for fields, st, planned, n in res[1:]:
        cur = (st["h"] != 0) | (st["qx"] != 0) | (st["qy"] != 0)
        prev = (st["h_prev"] != 0) | (st["qx_prev"] != 0) | (st["qy_prev"] != 0)
        want = int(plan_rule.planned(cur, prev, 480, 32).sum())
        n3 = int(plan_rule.planned_3x3(cur, prev, 480, 32).sum())
        assert planned == want < n3 <= n, (planned, want, n3, n)
        for k, _ in FIELDS:
            assert np.array_equal(ref[k].view(np.uint32), fields[k].view(np.uint32)), k


def test_variable_dt_matches_oracle(tmp_path):
    y = random_case(tmp_path, 120, 96, seed=11, dt=0.05, variable_dt=True)
    sim = _sim(y, quiet=True)
    sim.step(300)
    d, dt, it = sim.time()
    h = sim.field("h")
    pitch = sim.pitch
    sim.close()
    o = pyoracle.Oracle.from_yaml(y, pitch, precision=32)
    o.simulate(300)
    assert it == 300
    assert abs(d - o.duration) < 1e-6 and abs(dt - o.dt) < 1e-6
    worst, ok = _close(o.field(pyoracle.F_H), h, atol=1e-4, rtol=1e-5)
    assert ok, worst


def test_nonfinite_is_reported(tmp_path):
    """A q inflow whose level is below every boundary cell divides by a zero wet sum (the
    reference propagates the NaN); with stop_on_nonfinite the run stops with a status."""
    bc = [{"side": "left", "type": "q", "z": -50.0, "q": 1.0}]
    y = random_case(tmp_path, 64, 40, seed=2, bcs=bc, kst_var=False, no_data=False)
    from fip_b200 import FipError

    sim = _sim(y, quiet=True, stop_on_nonfinite=True)
    with pytest.raises(FipError) as e:
        sim.step(50)
    assert e.value.code == -5
    assert sim.info().nonfinite == 1
    sim.close()


def test_dry_tile_skipping_unconfigured_sides(tmp_path):
    """Only the tiles a boundary condition writes near are always computed: sides without a
    condition keep their edge cells as they are, so their dry tiles are skipped, while water lying
    on edge cells the step never writes keeps the tiles within reach active. Runs with dry-tile
    skipping stay bit-identical to every-tile runs."""
    from fip_b200 import synth

    W, H = 1500, 700
    rng = np.random.default_rng(17)
    y = np.arange(H, dtype=np.float32)[:, None]
    x = np.arange(W, dtype=np.float32)[None, :]
    terr = (0.002 * x + 0.3 * np.sin(x / 37.0) * np.cos(y / 23.0)).astype(np.float32)
    depth = np.zeros((H, W), np.float32)
    depth[250:420, 0:300] = 0.8                      # pond against the left side (z inflow rows 300-360)
    depth[H - 3:H, 700:760] = 0.5                    # water on the top edge rows (never written there)
    depth[100:140, W - 2:W] = 0.3                    # and on the right edge columns
    depth[500:530, 900:960] = 0.6                    # an inland pond
    wet = depth > 0
    qx = (0.05 * rng.standard_normal((H, W)) * wet).astype(np.float32)
    qy = (0.05 * rng.standard_normal((H, W)) * wet).astype(np.float32)
    files = {}
    for k, a in (("terrain", terr), ("z", terr + depth), ("qx", qx), ("qy", qy)):
        files[k] = str(tmp_path / f"u_{k}.bin")
        synth.write_grid(files[k], a)
    cfg = {"name": str(tmp_path / "u"), "terrain": [files["terrain"], 0], "z": [files["z"], 0],
           "qx": [files["qx"], 0], "qy": [files["qy"], 0], "W": W, "H": H, "dx": 2.0, "dt": 0.05,
           "duration": 1000, "kSt": 30, "variable_dt": False,
           "boundary_conditions": [{"side": "left", "type": "z", "z": float(terr[330, 0] + 1.2), "from": 300,
                                    "to": 360}]}
    path = str(tmp_path / "u.yml")
    synth.write_yaml(path, cfg)
    res = []
    for all_tiles, graphs in ((True, False), (False, True), (False, False)):
        sim = _sim(path, quiet=True, all_tiles=all_tiles, use_graphs=graphs)
        first = sim.info().active_tiles
        sim.step(300)
        inf = sim.info()
        res.append(({k: sim.field(k) for k, _ in FIELDS}, first, inf.active_tiles, inf.n_tiles))
        sim.close()
    ref = res[0][0]
    for fields, first, active, n in res[1:]:
        # 4 x 22 tiles, 48 of them on the edge: the dry edge tiles away from the water and from
        # the inflow are skipped from the first step on
        assert first < n and active < n, (first, active, n)
        for k, _ in FIELDS:
            assert np.array_equal(ref[k].view(np.uint32), fields[k].view(np.uint32)), k
