"""Parity on the full-size workloads, through the C ABI (fip_b200.Simulation -> libfip_b200.so).

* The 1024 x 1024 plain-solver case exactly as specified (dt 0.1 s, 10 000 steps, a dump every
  100 simulated s = 1 000 steps) against the reference binary itself (oracle/_ref/fip_ref_nomask,
  src/kernels.cu with the wet/dry mask off, deterministic): every dump of depth, qx, qy and flood
  plains within |dz|, |dq| <= 1e-4, identical wet sets, the same step count.
* The 5667 x 6500 large grid (2448 tiles of 480 x 32 cells: five plan chunks, so the kernels' walk
  over a multi-chunk active-tile list is exercised) from a flooded start with smooth seeded
  discharges, fixed dt, 50 steps, against the FP32 oracle: h, qx, qy, both ping-pong partners and
  hmax within the gates, identical wet sets; FP64 volume within 1e-6 relative; and the dry-tile
  skipping run bit-identical to the every-tile run.
* The 5667 x 6500 grid as specified (dry start), variable dt, against the reference binary with a
  synchronised CFL readback (oracle/_ref/fip_ref_sync): the same step count and dumps within the
  gates.
The reference binaries are built from the reference's sources by oracle/ref.mk; tests that need
them are skipped (with the reason) where they were not built.
"""
import os
import shutil

import numpy as np
import pytest

import pyoracle
import refbin

pytestmark = pytest.mark.gpu

FIELDS = (("h", pyoracle.F_H), ("qx", pyoracle.F_QX), ("qy", pyoracle.F_QY), ("h_prev", pyoracle.F_H_OTHER),
          ("qx_prev", pyoracle.F_QX_OTHER), ("qy_prev", pyoracle.F_QY_OTHER), ("hmax", pyoracle.F_HMAX))


def _need(name):
    if refbin.binary(name) is None:
        pytest.skip(f"oracle/_ref/{name} not built (make -f oracle/ref.mk REF=<reference sources>)")


def _gate(ref, got, atol=1e-4, rtol=1e-6):
    """max |d| and whether every cell is within atol + rtol |ref| (the relative term covers the
    reference's pitch-scaled top/bottom outflow, whose depths reach hundreds of metres)."""
    d = np.abs(ref.astype(np.float64) - got.astype(np.float64))
    return float(d.max()) if d.size else 0.0, bool(np.all(d <= atol + rtol * np.abs(ref.astype(np.float64))))


def _two_copies(tmp_path, make):
    """The same seeded scenario generated twice (own `name` prefix each, so dumps do not mix)."""
    a, b = tmp_path / "ref", tmp_path / "ours"
    return make(str(a)), make(str(b))


def _compare_dumps(ref_prefix, got_prefix, label):
    ref, got = refbin.dumps(ref_prefix), refbin.dumps(got_prefix)
    assert ref, f"{label}: the reference wrote no dumps"
    assert sorted(ref) == sorted(got), f"{label}: dump sets differ: {sorted(ref)} vs {sorted(got)}"
    exact = total = 0
    for key in sorted(ref):
        worst, ok = _gate(ref[key], got[key])
        assert ok, f"{label} {key}: max |d| = {worst}"
        exact += int(np.sum(ref[key].view(np.uint32) == got[key].view(np.uint32)))
        total += ref[key].size
        if key[0] == "ah":
            assert np.array_equal(ref[key] > 1e-6, got[key] > 1e-6), f"{label} {key}: wet sets differ"
    return exact, total


def test_config0_full_run_matches_reference_binary(tmp_path):
    """1024 x 1024, dt 0.1 s, 10 000 steps, 10 dumps: the reference binary against fip_run."""
    _need("fip_ref_nomask")
    from fip_b200 import Simulation, synth

    mk = lambda d: synth.scenario0(d, W=1024, H=1024, dt=0.1, duration=1000.0, save_every=100.0, name="cfg0")
    sref, sours = _two_copies(tmp_path, mk)
    r = refbin.run("fip_ref_nomask", sref.yaml_path)
    with Simulation(sours.yaml_path, quiet=True) as sim:
        sim.run()
        it = sim.iteration
    assert it == r["iterations"] == 10000
    exact, total = _compare_dumps(str(tmp_path / "ref" / "cfg0"), str(tmp_path / "ours" / "cfg0"), "config0")
    print(f"config0: {exact}/{total} dumped values bit-identical to the reference binary")


def _flood1(d, **kw):
    from fip_b200 import synth

    return synth.scenario1(d, wet_start=True, dt=0.1, name="cfg1", **kw)


def test_config1_full_grid_fixed_dt_matches_oracle(tmp_path):
    """5667 x 6500 flooded start, fixed dt 0.1 s, 50 steps: FP32 oracle, FP64 volume, and dry-tile
    skipping over the five-chunk tile list against the every-tile run, bit for bit."""
    from fip_b200 import Simulation

    sc = _flood1(str(tmp_path), variable_dt=False, duration=3600.0)
    steps = 50
    runs = {}
    for all_tiles in (True, False):
        with Simulation(sc.yaml_path, quiet=True, all_tiles=all_tiles) as sim:
            inf = sim.info()
            assert inf.n_tiles == 12 * 204
            sim.step(steps)
            runs[all_tiles] = ({k: sim.field(k) for k, _ in FIELDS}, sim.volume(), sim.info().active_tiles)
            pitch = sim.pitch
    got, vol, _ = runs[True]
    skip, vol_skip, active = runs[False]
    assert 0 < active < 12 * 204
    for k, _ in FIELDS:
        assert np.array_equal(got[k].view(np.uint32), skip[k].view(np.uint32)), f"skip vs all tiles: {k}"
    assert vol == vol_skip
    o = pyoracle.Oracle.from_yaml(sc.yaml_path, pitch, precision=32)
    o.simulate(steps)
    for k, which in FIELDS:
        worst, ok = _gate(o.field(which), got[k])
        assert ok, f"fp32 oracle {k}: max |d| = {worst}"
    assert np.array_equal(o.field(pyoracle.F_H) > 1e-6, got["h"] > 1e-6)
    del o
    o = pyoracle.Oracle.from_yaml(sc.yaml_path, pitch, precision=64)
    o.simulate(steps)
    assert abs(vol - o.volume()) <= 1e-6 * abs(o.volume()), (vol, o.volume())


def test_config1_full_grid_variable_dt_matches_reference_binary(tmp_path):
    """5667 x 6500 as specified (dry start, q inflow hydrograph, open bottom, kSt_var, no_data
    border), variable dt, the first 300 simulated s (about 600 steps): the reference with a
    synchronised CFL readback against fip_run (same step count, dumps within the gates)."""
    _need("fip_ref_sync")
    from fip_b200 import Simulation, synth

    mk = lambda d: synth.scenario1(d, duration=300.0, name="cfg1", save_state=["150", "300"])
    sref, sours = _two_copies(tmp_path, mk)
    r = refbin.run("fip_ref_sync", sref.yaml_path)
    with Simulation(sours.yaml_path, quiet=True) as sim:
        sim.run()
        it = sim.iteration
    assert it == r["iterations"], (it, r["iterations"])
    exact, total = _compare_dumps(str(tmp_path / "ref" / "cfg1"), str(tmp_path / "ours" / "cfg1"), "config1")
    print(f"config1 variable dt: {it} steps, {exact}/{total} dumped values bit-identical to the reference binary")
    shutil.rmtree(tmp_path / "ref", ignore_errors=True)
