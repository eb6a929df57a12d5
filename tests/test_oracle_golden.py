"""The CPU oracle against the reference binary's own outputs (tests/golden/*.npz).

The fixtures were produced by tests/golden/make_golden.py, which runs the reference built from
its sources (oracle/ref.mk) on a B200. This pins the oracle: same dumps within FP rounding, the
same wet/dry sets, the same sampling rows and, for variable dt, the same number of steps.
"""
import numpy as np
import pytest

import pyoracle
from golden_util import Golden, cases

KINDS = ("ah", "qx", "qy", "flood_plains")


def _compare(ref, got, atol, rtol):
    d = np.abs(ref.astype(np.float64) - got.astype(np.float64))
    lim = atol + rtol * np.abs(ref.astype(np.float64))
    return float(np.max(d)), bool(np.all(d <= lim))


def _iterations_of(stderr: str) -> int:
    # "Finished N iterations after S s (x s/it)" (src/main.cpp:253)
    return int(stderr.split("Finished ")[1].split(" ")[0])


@pytest.mark.parametrize("precision", [64, 32])
@pytest.mark.parametrize("name", cases())
def test_oracle_matches_reference(name, precision, tmp_path):
    g = Golden(name)
    y = g.materialize(str(tmp_path))
    o = pyoracle.Oracle.from_yaml(y, g.pitch_elems, precision=precision)
    o.run_to(o.target_duration)
    assert o.iteration == _iterations_of(g.meta["stderr"])
    dumps = o.dumps()
    assert [int(t) for t, _ in dumps] == g.dump_times()
    for t, fs in dumps:
        for kind, f in zip(KINDS, fs):
            ref = g.dump(kind, int(t))
            worst, ok = _compare(ref, f, atol=2e-5, rtol=1e-6)
            assert ok, f"{name} t={t} {kind}: max |d| {worst}"
            if kind == "ah":
                assert np.array_equal(ref > 1e-6, f > 1e-6), f"{name} t={t}: wet sets differ"
    # sampling rows: same times, values within rounding
    ref_rows = [r for r in g.stdout.split("\n")[1:] if r]
    got_rows = [r for r in o.sample_text().split("\n") if r]
    assert len(ref_rows) == len(got_rows)
    for a, b in zip(ref_rows, got_rows):
        va = [float(x) for x in a.split(";") if x]
        vb = [float(x) for x in b.split(";") if x]
        assert va[0] == vb[0]
        assert np.allclose(va[1:], vb[1:], atol=2e-5, rtol=1e-5)


def test_mask_on_reference_agrees_on_wet_cells(tmp_path):
    """The shipped reference (wet/dry mask on) against the oracle (mask off): the mask only
    skips strips whose cells are all dry, so wet cells and the wet set agree."""
    g = Golden("g0_z_open_close_mask")
    y = g.materialize(str(tmp_path))
    o = pyoracle.Oracle.from_yaml(y, g.pitch_elems, precision=64)
    o.run_to(o.target_duration)
    for t, fs in o.dumps():
        ref = g.dump("ah", int(t))
        wet = ref > 1e-6
        assert np.array_equal(wet, fs[0] > 1e-6)
        assert np.max(np.abs(ref[wet] - fs[0][wet])) < 2e-5
