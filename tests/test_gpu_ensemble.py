"""Batched ensembles (fip_ensemble_* in include/fip.h) against single-scenario runs.

Every member of an ensemble must compute exactly what fip_init + fip_step compute for its own
parameter file: same depths and discharges in both ping-pong buffers, same flood-plain map, same
simulated time, dt and step count, bit for bit, whatever the tile shape and however the
autotuner switches shapes during the run. The members differ in size (ragged, narrower and
wider than one tile), boundary types (z, q with time series, open on a side and on the bottom,
close), roughness (uniform kSt and a kSt_var grid with no_data cells) and dt control (fixed and
variable).
"""
import numpy as np
import pytest

from fip_b200 import Ensemble, Simulation, synth

pytestmark = pytest.mark.gpu

FIELDS = ("h", "qx", "qy", "h_prev", "qx_prev", "qy_prev", "hmax")


def _members(d, long=False):
    f = 4.0 if long else 1.0
    return [
        synth.ensemble_member(str(d), 300, 170, seed=5, kst=33.3, q_peak=40.0, t_peak=300.0, duration=900.0 * f,
                              name="a").yaml_path,
        synth.ensemble_member(str(d), 97, 211, seed=6, kst=21.0, q_peak=15.0, t_peak=200.0, duration=600.0 * f,
                              name="b", right="close", bottom="open").yaml_path,
        synth.scenario0(str(d), W=130, H=90, duration=40.0 * f, save_every=0, name="c").yaml_path,
        synth.scenario1(str(d), W=200, H=180, seed=3, duration=3600.0 * f, name="d").yaml_path,
        synth.ensemble_member(str(d), 517, 45, seed=7, kst=44.0, q_peak=30.0, t_peak=100.0, duration=300.0 * f,
                              name="e").yaml_path,
    ]


def _single(path, steps=None):
    with Simulation(path, quiet=True) as s:
        if steps is None:
            s.run()
        else:
            s.step(steps)
        return {k: s.field(k) for k in FIELDS}, s.time()


def _check_member(e, m, ref, ref_time):
    for k in FIELDS:
        got = e.field(m, k)
        assert np.array_equal(got, ref[k]), (m, k, float(np.max(np.abs(got - ref[k]))))
    d, dt, it = e.time(m)
    assert (d, dt, it) == ref_time, (m, (d, dt, it), ref_time)


def test_ensemble_members_match_single_runs(tmp_path):
    paths = _members(tmp_path, long=True)
    K = 230  # every member is still short of its target duration
    with Ensemble(paths) as e:
        e.step(K)
        inf = e.info()
        assert inf.n_members == len(paths) and inf.active_members == len(paths) and inf.iteration == K
        for m, p in enumerate(paths):
            ref, rt = _single(p, K)
            _check_member(e, m, ref, rt)


@pytest.mark.parametrize("kw,rows,nc", [(4, 32, 4), (4, 16, 4), (4, 64, 4), (2, 32, 4), (2, 16, 4), (2, 64, 4),
                                        (4, 32, 2), (4, 16, 2), (4, 64, 2)])
def test_ensemble_tile_shapes_are_exact(tmp_path, kw, rows, nc):
    paths = _members(tmp_path, long=True)[:4]
    K = 120
    with Ensemble(paths) as e:
        e.set_shape(kw, rows, nc)
        e.step(K)
        inf = e.info()
        assert inf.tile_rows == rows and inf.consumer_warps == kw and inf.cols_per_thread == nc
        assert inf.tile_cols == 30 * nc * kw
        for m, p in enumerate(paths):
            ref, rt = _single(p, K)
            _check_member(e, m, ref, rt)


def test_ensemble_run_to_target_and_autotune(tmp_path):
    """Members end at different times (a member that reached its target stops while the others
    go on); the autotuner switches shapes mid-run without changing any result."""
    paths = _members(tmp_path)
    with Ensemble(paths) as e:
        e.step(30)
        res = e.autotune(steps_per_shape=8)
        assert len(res) >= 1 and all(r["ms_per_step"] > 0 for r in res)
        e.run()
        assert e.info().active_members == 0
        for m, p in enumerate(paths):
            ref, rt = _single(p)
            _check_member(e, m, ref, rt)


def test_ensemble_all_tiles_matches(tmp_path):
    paths = _members(tmp_path, long=True)[:3]
    K = 64
    with Ensemble(paths, all_tiles=True) as e:
        e.step(K)
        assert e.info().active_tiles == e.info().n_tiles
        for m, p in enumerate(paths):
            ref, rt = _single(p, K)
            _check_member(e, m, ref, rt)


@pytest.mark.parametrize("all_tiles,shape", [(True, (4, 32)), (False, (2, 16)), (False, (4, 16, 2))])
def test_large_ensemble_multi_chunk_members_match_single_runs(tmp_path, all_tiles, shape):
    """Members of 0.5 to 3 M cells whose tiles together fill several 512-tile chunks of the
    concatenated plan (1 131 tiles of 480 x 32, 3 957 of 240 x 16): every member still computes
    exactly what its single run computes."""
    sizes = [(2048, 1500), (1900, 1300), (1200, 2000), (2000, 900), (700, 1800), (1500, 1500), (1024, 1024)]
    paths = [synth.ensemble_member(str(tmp_path), W, H, seed=40 + i, kst=22.0 + 3 * i, q_peak=800.0 + 150 * i,
                                   t_peak=600.0, duration=3600.0, name=f"L{i}").yaml_path
             for i, (W, H) in enumerate(sizes)]
    K = 150
    with Ensemble(paths, all_tiles=all_tiles) as e:
        e.set_shape(*shape)
        e.step(K)
        inf = e.info()
        assert inf.n_tiles > 1024
        for m, p in enumerate(paths):
            ref, rt = _single(p, K)
            _check_member(e, m, ref, rt)
