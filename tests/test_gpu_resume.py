"""Exact resume (fip_checkpoint / fip_restore) and restarts from save_state dumps.

The reference restarts only by feeding dumps back as z/qx/qy input files (src/main.cpp:154-202,
src/simdata.cpp:266-274), which mixes up depth and level and loses the step state. A checkpoint
must let a run continue bit for bit; the dump route (through fip_b200.restart) must restart the
dumped depths to FP32 rounding and the discharges exactly.
"""
import glob
import os

import numpy as np
import pytest

from fip_b200 import FipError, Simulation, synth
from fip_b200 import restart

pytestmark = pytest.mark.gpu

FIELDS = ("h", "qx", "qy", "h_prev", "qx_prev", "qy_prev", "hmax")


def _state(sim):
    return {k: sim.field(k) for k in FIELDS}, sim.time()


@pytest.mark.parametrize("first", [0, 137, 200])
def test_checkpoint_restore_is_exact(tmp_path, first):
    """Checkpoints before the first step, in mid-run and at a flood-plain iteration (200)."""
    sc = synth.scenario1(str(tmp_path), W=230, H=190, seed=4, duration=7200.0, name="r")
    ck = str(tmp_path / "state.ckpt")
    with Simulation(sc.yaml_path, quiet=True) as a:
        a.step(first) if first else None
        a.checkpoint(ck)
        a.step(170)
        ref, ref_t = _state(a)
    with Simulation(sc.yaml_path, quiet=True) as b:
        b.step(25)  # some other state first: restore must replace all of it
        b.restore(ck)
        b.step(170)
        got, got_t = _state(b)
    assert got_t == ref_t
    for k in FIELDS:
        assert np.array_equal(got[k], ref[k]), (k, float(np.max(np.abs(got[k] - ref[k]))))


def test_restore_rejects_another_scenario(tmp_path):
    a = synth.scenario1(str(tmp_path), W=120, H=100, seed=4, duration=600.0, name="a")
    b = synth.scenario1(str(tmp_path), W=120, H=100, seed=5, duration=600.0, name="b")
    ck = str(tmp_path / "a.ckpt")
    with Simulation(a.yaml_path, quiet=True) as s:
        s.step(10)
        s.checkpoint(ck)
    with Simulation(b.yaml_path, quiet=True) as s:
        with pytest.raises(FipError, match="different terrain"):
            s.restore(ck)
    with open(ck, "r+b") as f:  # a truncated file is an I/O error, not a crash
        f.truncate(200)
    with Simulation(a.yaml_path, quiet=True) as s:
        with pytest.raises(FipError):
            s.restore(ck)


def test_restart_from_dump_as_level_file(tmp_path):
    sc = synth.scenario0(str(tmp_path), W=150, H=110, duration=60.0, save_every=0, name="d")
    prefix = str(tmp_path / "dump")
    with Simulation(sc.yaml_path, quiet=True) as s:
        s.step(300)
        s.save(prefix, current=True)
        h, qx, qy = s.field("h"), s.field("qx"), s.field("qy")
    ah = glob.glob(prefix + "_ah_*")[0]
    fqx = glob.glob(prefix + "_qx_*")[0]
    fqy = glob.glob(prefix + "_qy_*")[0]
    assert np.array_equal(restart.read_dump(ah), h)
    level = str(tmp_path / "level.bin")
    restart.level_file_from_dump(ah, os.path.join(str(tmp_path), "d_terrain.bin"), 0, level)
    y2 = str(tmp_path / "d_restart.yml")
    with open(sc.yaml_path) as f:
        text = f.read()
    with open(y2, "w") as f:
        f.write(text + f"z: [{level}, 16]\nqx: [{fqx}, 16]\nqy: [{fqy}, 16]\n")
    with Simulation(y2, quiet=True) as r:
        assert np.array_equal(r.field("qx"), qx) and np.array_equal(r.field("qy"), qy)
        h2 = r.field("h")
        terr = r.field("terrain")
        # (h + terrain) - terrain: exact up to the rounding of the level
        tol = np.spacing(np.abs(h + terr).astype(np.float32)).astype(np.float64)
        assert np.all(np.abs(h2.astype(np.float64) - h) <= tol)
