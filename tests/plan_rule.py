"""Host restatement of the dry-tile plan, for the tests.

The library plans the tiles of the next step on the device (`fip_plan` / `fip_ens_plan` in
fip_b200/csrc/bc_codegen.cpp) from one flag byte per tile and state, set by the stencil and by
`init_tiles_kernel` (fip_b200/csrc/rmg_stencil.cu): ANY (some cell nonzero), WEST / EAST (some
cell of the tile's first / last `band` columns nonzero). A tile is planned when it had a nonzero
cell in the previous state, when it or the tile above or below it has one in the current state,
or when one of the three tiles beside it in a neighbouring strip has one in its facing band.

The rule is exact only if the step's result on a tile depends on no state cell further than
`band` columns beside it and one tile above or below it; the stencil reaches 2 cells
(tests/test_plan_rule.py checks that against the oracle), so `band` >= 2 suffices.
"""
from __future__ import annotations

import numpy as np


def _grid(nz, tc, tr):
    H, W = nz.shape
    return -(-W // tc), -(-H // tr)


def tile_flags(nz, tc, tr, band):
    """any / west / east flags, (n_sx, n_ty) bool arrays, of a nonzero mask (H, W)."""
    H, W = nz.shape
    n_sx, n_ty = _grid(nz, tc, tr)
    f = {k: np.zeros((n_sx, n_ty), bool) for k in ("any", "west", "east")}
    for s in range(n_sx):
        c0, c1 = s * tc, min((s + 1) * tc, W)
        for t in range(n_ty):
            blk = nz[t * tr:(t + 1) * tr, c0:c1]
            f["any"][s, t], f["west"][s, t], f["east"][s, t] = blk.any(), blk[:, :band].any(), blk[:, -band:].any()
    return f


def planned(cur, prev, tc, tr, band=4):
    """Tiles the band rule plans for the next step (no sticky tiles): (n_sx, n_ty) bool."""
    f, p = tile_flags(cur, tc, tr, band), tile_flags(prev, tc, tr, band)
    n_sx, n_ty = f["any"].shape
    act = np.zeros((n_sx, n_ty), bool)
    for s in range(n_sx):
        for t in range(n_ty):
            rows = slice(max(t - 1, 0), t + 2)
            own = p["any"][s, t] or f["any"][s, rows].any()
            side = (s > 0 and f["east"][s - 1, rows].any()) or (s + 1 < n_sx and f["west"][s + 1, rows].any())
            act[s, t] = own or side
    return act


def planned_3x3(cur, prev, tc, tr):
    """Tiles the rule "some nonzero cell in the 3 x 3 tile neighbourhood" would plan."""
    f, p = tile_flags(cur, tc, tr, 1), tile_flags(prev, tc, tr, 1)
    n_sx, n_ty = f["any"].shape
    act = np.zeros((n_sx, n_ty), bool)
    for s in range(n_sx):
        for t in range(n_ty):
            act[s, t] = p["any"][s, t] or f["any"][max(s - 1, 0):s + 2, max(t - 1, 0):t + 2].any()
    return act


def needed(cur, prev, tc, tr, reach=2):
    """Tiles whose step is not the identity on zeros: a nonzero cell of the current state within
    `reach` cells of the tile, or of the previous state (the output buffer) in the tile."""
    H, W = cur.shape
    n_sx, n_ty = _grid(cur, tc, tr)
    p = tile_flags(prev, tc, tr, 1)
    need = np.zeros((n_sx, n_ty), bool)
    for s in range(n_sx):
        c0, c1 = s * tc, min((s + 1) * tc, W)
        for t in range(n_ty):
            r0, r1 = t * tr, min((t + 1) * tr, H)
            box = cur[max(r0 - reach, 0):r1 + reach, max(c0 - reach, 0):c1 + reach]
            need[s, t] = p["any"][s, t] or box.any()
    return need
