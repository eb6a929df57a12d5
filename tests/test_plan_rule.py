"""The dry-tile plan's exactness argument, on the CPU.

Skipping a tile is exact when the step computes zeros there: every state cell within the
stencil's reach of the tile is zero, and so is the tile in the output buffer (the previous
state). The plan (restated in tests/plan_rule.py) reads per-tile flags with edge bands of 4
columns (2 for two-column threads) and whole tiles above and below. These tests check, against
the CPU oracle, that one step reads no state cell more than 2 cells away (the reach), and that
the band rule plans every tile a reach of 2 makes necessary, for random sparse states and every
tile shape the library uses; a planted band of 1 column is caught.
"""
import numpy as np
import pytest

import plan_rule
import pyoracle


def _wet_state(W, H, seed):
    rng = np.random.default_rng(seed)
    y = np.arange(H, dtype=np.float32)[:, None]
    x = np.arange(W, dtype=np.float32)[None, :]
    terr = (0.3 * np.sin(x / 5.0 + seed) * np.cos(y / 4.0) + 0.01 * x).astype(np.float32)
    h = (0.5 + 0.2 * rng.standard_normal((H, W))).clip(0.05, None).astype(np.float32)
    qx = (0.2 * rng.standard_normal((H, W))).astype(np.float32)
    qy = (0.2 * rng.standard_normal((H, W))).astype(np.float32)
    kst = np.where(rng.random((H, W)) < 0.5, 25.0, 40.0).astype(np.float32)
    return terr, h, qx, qy, kst


def _step(terr, h, qx, qy, kst, precision):
    H, W = h.shape
    o = pyoracle.Oracle(W, H, 128 * -(-W // 128), 2.0, 0.02, False, 30.0, -9999.0, terr, h, qx, qy, kst_var=kst,
                        precision=precision)
    o.simulate(1)
    return [o.field(k) for k in (pyoracle.F_H, pyoracle.F_QX, pyoracle.F_QY)]


@pytest.mark.parametrize("precision", [32, 64])
@pytest.mark.parametrize("field", [0, 1, 2])  # perturb h, qx or qy
def test_step_reads_two_cells_around_each_cell(precision, field):
    """Changing one state cell changes the next state only within 2 cells of it, and at
    distance 2 too (the bound is the reach, not a loose one)."""
    W, H = 40, 36
    terr, h, qx, qy, kst = _wet_state(W, H, seed=5 + field)
    base = _step(terr, h, qx, qy, kst, precision)
    far = 0
    for (pr, pc) in ((17, 19), (9, 30), (26, 8)):
        st = [h.copy(), qx.copy(), qy.copy()]
        st[field][pr, pc] += 0.3
        got = _step(terr, *st, kst, precision)
        diff = np.zeros((H, W), bool)
        for a, b in zip(base, got):
            diff |= a.view(np.uint32) != b.view(np.uint32)
        rr, cc = np.nonzero(diff)
        assert rr.size > 0
        dist = np.maximum(np.abs(rr - pr), np.abs(cc - pc))
        assert dist.max() <= 2, (pr, pc, list(zip(rr[dist > 2], cc[dist > 2])))
        far += int((dist == 2).sum())
    assert far > 0


def _sparse_mask(W, H, rng, n_blobs):
    m = np.zeros((H, W), bool)
    for _ in range(n_blobs):
        r, c = int(rng.integers(0, H)), int(rng.integers(0, W))
        hr, hc = int(rng.integers(0, 6)), int(rng.integers(0, 6))
        m[max(r - hr, 0):r + hr + 1, max(c - hc, 0):c + hc + 1] = True
    return m


# tile shapes of the library: single grids 480 x 32 with 4-column threads; ensembles 240 / 480
# columns, 16 / 32 / 64 rows, 4- or 2-column threads (edge bands of 4 or 2 columns)
SHAPES = [(480, 32, 4), (240, 16, 4), (240, 32, 2), (480, 64, 4), (240, 64, 2)]


@pytest.mark.parametrize("tc,tr,band", SHAPES)
@pytest.mark.parametrize("seed", range(6))
def test_band_rule_plans_every_tile_the_reach_needs(tc, tr, band, seed):
    rng = np.random.default_rng(seed)
    W, H = 1503, 205  # ragged last strip and tile row
    for n_blobs in (1, 4, 20):
        cur = _sparse_mask(W, H, rng, n_blobs)
        prev = _sparse_mask(W, H, rng, 1) & (rng.random() < 0.5)
        need = plan_rule.needed(cur, prev, tc, tr, reach=2)
        plan = plan_rule.planned(cur, prev, tc, tr, band=band)
        wide = plan_rule.planned_3x3(cur, prev, tc, tr)
        assert not (need & ~plan).any()   # sound: no needed tile is skipped
        assert not (plan & ~wide).any()   # never more than the 3 x 3 rule


def test_band_rule_with_water_at_strip_edges():
    """Water 2 cells from a strip edge needs the neighbouring strip; the band rule plans it and a
    band of 1 column (a planted mistake in the restatement) would not; water 5 cells away needs
    it not, and the band rule skips it where the 3 x 3 rule would not."""
    W, H, tc, tr = 1500, 96, 480, 32
    cur = np.zeros((H, W), bool)
    cur[40, 478] = True      # 2 cells west of strip 1
    need = plan_rule.needed(cur, cur, tc, tr)
    assert need[1, 1] and not (need & ~plan_rule.planned(cur, cur, tc, tr, band=4)).any()
    assert (need & ~plan_rule.planned(cur, cur, tc, tr, band=1)).any()
    cur[:] = False
    cur[40, 475] = True      # 5 cells west of strip 1
    assert not plan_rule.needed(cur, cur, tc, tr)[1].any()
    assert not plan_rule.planned(cur, cur, tc, tr, band=4)[1].any()
    assert plan_rule.planned_3x3(cur, cur, tc, tr)[1].any()
