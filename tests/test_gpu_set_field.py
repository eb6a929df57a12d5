"""fip_set_field: the state a host writes into a running simulation.

A caller that drives the step from its own loop (coupling, data assimilation, the end-to-end
benchmark) uploads h, qx and qy between steps. The upload must land in both ping-pong buffers
unchanged, continuing after re-uploading the current state must give what continuing without it
gives, and a negative depth in the upload must switch the hmax fold to the whole grid (the
initial-state rule of fip_init), which the checkpoint header records.
"""
import struct

import numpy as np
import pytest

from fip_b200 import Simulation, synth

pytestmark = pytest.mark.gpu

CKPT_HEADER_BYTES = 88
CKPT_HMAX_FULL_OFFSET = 84  # last int32 of the checkpoint header


def _hmax_full(path):
    with open(path, "rb") as f:
        hd = f.read(CKPT_HEADER_BYTES)
    assert hd[:8] == b"FIPCKPT1"
    assert struct.unpack_from("<I", hd, 12)[0] == CKPT_HEADER_BYTES
    return struct.unpack_from("<i", hd, CKPT_HMAX_FULL_OFFSET)[0]


def test_upload_lands_in_both_buffers(tmp_path):
    sc = synth.scenario0(str(tmp_path), W=300, H=210, duration=60, save_every=0, name="u")
    rng = np.random.default_rng(1)
    with Simulation(sc.yaml_path, quiet=True) as s:
        s.step(30)
        for name in ("h", "qx", "qy"):
            v = (s.field(name) + rng.uniform(0.0, 0.5, (s.H, s.W))).astype(np.float32)
            s.set_field(name, v)
            assert np.array_equal(s.field(name), v), name
            assert np.array_equal(s.field(name + "_prev"), v), name + "_prev"


def test_reupload_of_the_current_state_changes_nothing(tmp_path):
    sc = synth.scenario0(str(tmp_path), W=300, H=210, duration=60, save_every=0, name="c")
    with Simulation(sc.yaml_path, quiet=True) as a, Simulation(sc.yaml_path, quiet=True) as b:
        a.step(40)
        b.step(40)
        for name in ("h", "qx", "qy"):
            b.set_field(name, b.field(name))
        a.step(60)
        b.step(60)
        for name in ("h", "qx", "qy"):
            ra, rb = a.field(name), b.field(name)
            assert np.max(np.abs(ra - rb)) <= 1e-4, name
        assert np.array_equal(a.field("h") > 1e-6, b.field("h") > 1e-6)
        assert a.time()[0] == b.time()[0]


def test_negative_upload_sets_the_full_hmax_fold(tmp_path):
    sc = synth.scenario0(str(tmp_path), W=300, H=210, duration=60, save_every=0, name="n")
    with Simulation(sc.yaml_path, quiet=True) as s:
        s.step(10)
        s.checkpoint(str(tmp_path / "a.ckpt"))
        assert _hmax_full(str(tmp_path / "a.ckpt")) == 0
        h = s.field("h")
        s.set_field("h", h)  # no negative depth: the flag stays clear
        s.checkpoint(str(tmp_path / "b.ckpt"))
        assert _hmax_full(str(tmp_path / "b.ckpt")) == 0
        h[150, 277] = -0.25  # one cell, far from the water
        s.set_field("h", h)
        s.checkpoint(str(tmp_path / "c.ckpt"))
        assert _hmax_full(str(tmp_path / "c.ckpt")) == 1
        s.step(5)
