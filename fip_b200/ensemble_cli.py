"""Runs a batched ensemble of synthetic scenarios and prints its timing as JSON.

    python -m fip_b200.ensemble_cli [--members 64 --size-lo 256 --size-hi 2048 --steps 200
                                     --all-tiles --autotune --spinup 0]

Members come from synth.ensemble2 (fBm valleys, uniform kSt ~ U[20, 45], triangular inflow
hydrographs, variable dt). The timed steps run through fip_ensemble_step_timed (CUDA events on
the ensemble's stream).
"""
from __future__ import annotations

import argparse
import json
import os
import tempfile

from . import Ensemble, synth


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--members", type=int, default=64)
    ap.add_argument("--size-lo", type=int, default=256)
    ap.add_argument("--size-hi", type=int, default=2048)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--spinup", type=int, default=0)
    ap.add_argument("--all-tiles", action="store_true")
    ap.add_argument("--autotune", action="store_true")
    ap.add_argument("--seed", type=int, default=2)
    ap.add_argument("--to-target", action="store_true",
                    help="run every member to its target duration (6 simulated hours) and time it")
    a = ap.parse_args(argv)
    d = tempfile.mkdtemp(prefix="fip_ens_")
    members = synth.ensemble2(os.path.join(d, "m"), n=a.members, seed=a.seed, size_lo=a.size_lo, size_hi=a.size_hi)
    cells = sum(m.W * m.H for m in members)
    import time

    with Ensemble([m.yaml_path for m in members], all_tiles=a.all_tiles) as e:
        if a.to_target:
            t0 = time.perf_counter()
            tune = e.autotune(10) if a.autotune else None
            retunes = []
            # re-tune as the flood grows: the fastest tile shape changes with the active fraction
            while e.info().active_members:
                e.step(5000)
                if a.autotune and e.info().active_members:
                    best = e.autotune(10)
                    retunes.append(min(best, key=lambda r: r["ms_per_step"]) if best else None)
            wall = time.perf_counter() - t0
            inf = e.info()
            times = [e.time(m) for m in range(a.members)]
            print(json.dumps({"members": a.members, "cells": cells, "ensemble_steps": inf.iteration,
                              "wall_s": wall, "sim_hours": [round(t[0] / 3600, 3) for t in times][:4],
                              "member_steps_min_max": [min(t[2] for t in times), max(t[2] for t in times)],
                              "whole_ensemble_cell_updates_per_s": sum(
                                  m.W * m.H * t[2] for m, t in zip(members, times)) / wall,
                              "first_tune": tune, "retunes": retunes}))
            return 0
        if a.spinup:
            e.step(a.spinup)
        tune = e.autotune(10) if a.autotune else None
        e.step(3)
        ms = e.step_timed(a.steps)
        inf = e.info()
    print(json.dumps({"members": a.members, "cells": cells, "steps": a.steps, "ms_per_step": ms / a.steps,
                      "whole_ensemble_cell_updates_per_s": cells * a.steps / (ms / 1e3),
                      "active_tiles": inf.active_tiles, "n_tiles": inf.n_tiles,
                      "shape": [inf.consumer_warps, inf.tile_rows], "autotune": tune}))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
