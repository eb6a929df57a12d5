#!/usr/bin/env python
"""Benchmark of the slim shallow-water step on the large-grid scenario (5667 x 6500, kSt_var,
no_data border, variable dt, q inflow hydrograph, open bottom), FP32, one B200 per rank.

    python bench.py [--gpus N --steps K --warmup W] [--impl fip_b200|reference]

Metric: cell-updates/s. A step is one simulate() of the whole grid (every tile computed, no
dry-tile skipping in the headline number). `value` is device time of K steps run as one CUDA
graph with the state resident in HBM (the 1.18 GB working set of a step is far larger than the
126 MB L2, so no flush is needed); `e2e` runs the same steps through the C ABI with the state
uploaded from and downloaded to pinned host buffers around every batch of steps. The roofline
uses 32 algorithmic bytes per cell update (read h, qx, qy, terrain, kSt; write h, qx, qy) and the
stencil kernel's average launch time, from CUDA events around every stencil launch in a second
graph of K steps (event nodes between the launches keep them from overlapping, so the headline
graph has none). With N > 1 (torchrun) every rank runs an independent replica ("replicas only").

--impl reference times the reference's algorithm on the host cores: the reference's path is CUDA
only, so its CPU stand-in is the FP64 restatement (oracle port) of the whole scenario (every
cell, its boundary conditions and dt control) with all host threads.

Two informational objects ride on the same line (N = 1 only): `ensemble` (64 scenarios of
W, H ~ U[256, 2048] as one batched ensemble, every tile computed, autotuned tile shape, against
the same scenarios run one at a time, plus a flooded state with dry-tile skipping) and
`surrogate` (the tcgen05 convolutions of the learned surrogate against the measured bf16 GEMM
peak, and a reduced train / evaluate / screen run of fip_b200.surrogate_run).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

BYTES_PER_CELL = 32  # kSt_var workload: 5 float reads + 3 float writes
METRIC = "cell-updates/s"


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profile_traffic():
    """DRAM bytes per stencil launch from the committed ncu summary, scaled to this grid."""
    try:
        with open(os.path.join(ROOT, "profiles", "rmg_step_traffic.json")) as f:
            t = json.load(f)
        return float(t["dram_bytes_per_cell"])
    except Exception:
        return None


class Clocks:
    """SM clock, power and throttle reasons sampled during the timed region: NVML read-only
    queries every 2 ms from a thread (a timed region of a few milliseconds still gets samples),
    else nvidia-smi every 100 ms."""

    NAMES = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.samples = []  # (sm_mhz, sm_max_mhz, power_w, reasons tuple)
        self._stop = threading.Event()
        self._t = None
        self.source = None

    def __enter__(self):
        try:
            import pynvml

            pynvml.nvmlInit()
            dev = pynvml.nvmlDeviceGetHandleByIndex(self.index)
            bits = (pynvml.nvmlClocksEventReasonHwSlowdown, pynvml.nvmlClocksEventReasonHwThermalSlowdown,
                    pynvml.nvmlClocksEventReasonSwThermalSlowdown, pynvml.nvmlClocksEventReasonSwPowerCap)
            mx = pynvml.nvmlDeviceGetMaxClockInfo(dev, pynvml.NVML_CLOCK_SM)

            def read():
                sm = pynvml.nvmlDeviceGetClockInfo(dev, pynvml.NVML_CLOCK_SM)
                pw = pynvml.nvmlDeviceGetPowerUsage(dev) / 1000.0
                r = pynvml.nvmlDeviceGetCurrentClocksEventReasons(dev)
                return (float(sm), float(mx), pw, tuple(n for n, b in zip(self.NAMES, bits) if r & b))

            read()
            self.source = "nvml 2 ms"
            self._read = read
            self._t = threading.Thread(target=self._poll_nvml, daemon=True)
            self._t.start()
        except Exception:
            self._start_smi()
        return self

    def _poll_nvml(self):
        while not self._stop.is_set():
            try:
                self.samples.append(self._read())
            except Exception:
                pass
            time.sleep(0.002)

    def _start_smi(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self._p = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                        "--format=csv,noheader,nounits", "-lms", "100"],
                                       stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            return
        self.source = "nvidia-smi 100 ms"

        def reader():
            for line in self._p.stdout:
                p = [x.strip() for x in line.split(",")]
                if len(p) >= 7:
                    try:
                        self.samples.append((float(p[0]), float(p[1]), float(p[2]),
                                             tuple(n for n, v in zip(self.NAMES, p[3:7]) if v.lower() == "active")))
                    except ValueError:
                        pass

        self._t = threading.Thread(target=reader, daemon=True)
        self._t.start()
        t0 = time.time()  # keep nvidia-smi's start-up out of the timed region
        while not self.samples and time.time() - t0 < 10:
            time.sleep(0.05)

    def __exit__(self, *exc):
        self._stop.set()
        if getattr(self, "_p", None):
            self._p.terminate()
            try:
                self._p.wait(timeout=5)
            except Exception:
                self._p.kill()
        if self._t is not None:
            self._t.join(timeout=2)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        return {"sm_mhz": statistics.median(s[0] for s in self.samples),
                "sm_max_mhz": max(s[1] for s in self.samples),
                "power_w_max": max(s[2] for s in self.samples),
                "reasons": sorted({r for s in self.samples for r in s[3]}),
                "samples": len(self.samples), "source": self.source}


def make_workload(args, rank):
    from fip_b200 import synth

    d = os.path.join(tempfile.gettempdir(), f"fip_bench_{os.getpid()}_{rank}")
    sc = synth.scenario1(d, W=args.W, H=args.H, seed=1)
    return sc


def _pitch(W):
    return ((W * 4 + 511) // 512) * 128  # cudaMallocPitch's 512-byte row alignment, in floats


def cpu_baseline(sc, seconds: float):
    """FP64 oracle port (the restatement of the reference's kernel, boundary conditions and dt
    control) on the whole scenario: all host threads for about `seconds`, then one thread for a
    few steps."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle

    threads = os.cpu_count() or 1
    cells = sc.W * sc.H
    o = pyoracle.Oracle.from_yaml(sc.yaml_path, _pitch(sc.W), precision=64)
    o.set_threads(threads)
    t0 = time.perf_counter()
    o.simulate(1)
    per = time.perf_counter() - t0
    n = max(2, int(seconds / max(per, 1e-6)))
    t0 = time.perf_counter()
    o.simulate(n)
    dt = time.perf_counter() - t0
    o.set_threads(1)
    n1 = max(1, int(min(seconds / 3, 8.0) / max(per * threads, 1e-6)))
    t0 = time.perf_counter()
    o.simulate(n1)
    dt1 = time.perf_counter() - t0
    return {"value": cells * n / dt, "unit": METRIC, "cores": threads, "kind": "port",
            "single_thread_value": cells * n1 / dt1,
            "sample": f"FP64 oracle, whole {sc.W}x{sc.H} scenario with its boundary conditions and variable dt: "
                      f"{n} steps in {dt:.1f} s on {threads} threads, then {n1} steps in {dt1:.1f} s on 1 thread"}


def cpu_baseline_config0():
    """The 1024 x 1024 plain-solver case over its full 10 000 steps (dt 0.1 s), FP64 oracle port,
    all host threads; one thread timed on its first 200 steps."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle

    from fip_b200 import synth

    d = os.path.join(tempfile.gettempdir(), f"fip_bench_c0_{os.getpid()}")
    sc = synth.scenario0(d, W=1024, H=1024, dt=0.1, duration=1000.0, save_every=0, name="c0")
    threads = os.cpu_count() or 1
    o = pyoracle.Oracle.from_yaml(sc.yaml_path, _pitch(1024), precision=64)
    o.set_threads(threads)
    t0 = time.perf_counter()
    o.run_to(1000.0)
    dt = time.perf_counter() - t0
    steps = o.iteration
    o1 = pyoracle.Oracle.from_yaml(sc.yaml_path, _pitch(1024), precision=64)
    o1.set_threads(1)
    t0 = time.perf_counter()
    o1.simulate(200)
    dt1 = time.perf_counter() - t0
    return {"workload": "1024x1024 plain-solver case, dt 0.1 s, 10000 steps", "steps": steps,
            "wall_s": dt, "cores": threads, "cell_updates_per_s": 1024 * 1024 * steps / dt,
            "single_thread_cell_updates_per_s": 1024 * 1024 * 200 / dt1,
            "single_thread_wall_s_extrapolated": dt1 * steps / 200}


def gpu_reference_baseline(args, local_rank, duration):
    """Baseline leg: the reference's own CUDA kernels on this GPU. oracle/_ref holds the reference
    built from its own sources (the parity pin of the tests; oracle/ref.mk): fip_ref_nomask computes
    every strip (mask off), fip_ref skips dry strips with its wet/dry mask. Both run the large-grid
    scenario for its first `duration` simulated seconds and report the reference's own timing line
    (CUDA events around its whole simulate() loop, src/main.cpp:238-253). This library runs the same
    parameter file through fip_run, timed around the loop (wall clock, the loop ends synchronised),
    with every tile computed and with dry-tile skipping. Per-step time includes each side's host
    work per step (the reference's host dt controller and launches; the graphs and device-side dt
    control here)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import refbin

    from fip_b200 import Simulation, synth

    d = os.path.join(tempfile.gettempdir(), f"fip_bench_ref_{os.getpid()}")
    sc = synth.scenario1(d, W=args.W, H=args.H, seed=1, duration=duration, name="refcmp")
    cells = sc.W * sc.H
    out = {"workload": f"scenario1 {sc.W}x{sc.H}, variable dt, first {duration:g} simulated s (dry start)",
           "source": "oracle/_ref binaries built from the reference's sources by oracle/ref.mk"}
    for name, key in (("fip_ref_nomask", "reference_every_cell"), ("fip_ref", "reference_wet_dry_mask")):
        if refbin.binary(name) is None:
            out[key] = {"unavailable": f"oracle/_ref/{name} not built"}
            continue
        try:
            r = refbin.run(name, sc.yaml_path, timeout=600)
            out[key] = {"binary": f"oracle/_ref/{name}", "iterations": r["iterations"], "seconds": r["seconds"],
                        "s_per_it": r["seconds"] / r["iterations"],
                        "cell_updates_per_s": cells * r["iterations"] / r["seconds"]}
        except Exception as exc:
            out[key] = {"error": f"{type(exc).__name__}: {exc}"[:300]}
    for all_tiles, key in ((True, "fip_b200_every_tile"), (False, "fip_b200_dry_skip")):
        with Simulation(sc.yaml_path, device=local_rank, quiet=True, all_tiles=all_tiles) as sim:
            t0 = time.perf_counter()
            sim.run()
            sec = time.perf_counter() - t0
            it = sim.iteration
        out[key] = {"iterations": it, "seconds": sec, "s_per_it": sec / it, "cell_updates_per_s": cells * it / sec}
    a, b = out.get("reference_every_cell", {}), out.get("reference_wet_dry_mask", {})
    if "s_per_it" in a:
        out["speedup_every_cell"] = a["s_per_it"] / out["fip_b200_every_tile"]["s_per_it"]
    if "s_per_it" in b:
        out["speedup_dry_skip_vs_mask"] = b["s_per_it"] / out["fip_b200_dry_skip"]["s_per_it"]
    return out


def ensemble_measure(args, local_rank):
    """Batched ensemble of 64 scenarios (W, H ~ U[256, 2048], own fBm terrain, kSt ~ U[20, 45],
    triangular inflow peaking at U[200, 2000] m3/s after U[1, 8] h, variable dt), FP32.

    * batched: one Ensemble, every tile computed, tile shape autotuned, `ens_steps` ensemble
      steps timed with CUDA events (graphs of 64 steps);
    * sequential: the same members one at a time as single-scenario runs (the reference runs one
      scenario per process), every tile computed, `ens_seq_steps` steps each, device time;
    * flooded: the ensemble with dry-tile skipping after `ens_spinup` steps (whole-ensemble
      cell updates per second, i.e. every member's every cell, and the active-tile fraction).
    Speed-up = per-step time of the sequential runs summed over members / batched per-step time.
    """
    from fip_b200 import Ensemble, Simulation, synth

    d = os.path.join(tempfile.gettempdir(), f"fip_bench_ens_{os.getpid()}")
    t0 = time.perf_counter()
    members = synth.ensemble2(d, n=args.ens_members, seed=2)
    gen_s = time.perf_counter() - t0
    paths = [m.yaml_path for m in members]
    cells = sum(m.W * m.H for m in members)
    out = {"workload": f"ensemble of {len(paths)} scenarios, W,H ~ U[256,2048], kSt ~ U[20,45], variable dt",
           "members": len(paths), "cells": cells, "input_gen_s": round(gen_s, 1)}
    t0 = time.perf_counter()
    with Ensemble(paths, device=local_rank, all_tiles=True) as e:
        out["init_s"] = round(time.perf_counter() - t0, 1)
        e.step(3)
        tune = e.autotune(steps_per_shape=10)
        inf = e.info()
        e.step_timed(8)
        ms = e.step_timed(args.ens_steps)
    out["autotune"] = [{k: (round(v, 4) if isinstance(v, float) else v) for k, v in r.items()} for r in tune]
    out["shape"] = {"consumer_warps": inf.consumer_warps, "tile_cols": inf.tile_cols, "tile_rows": inf.tile_rows}
    batched_ms = ms / args.ens_steps
    out["batched_ms_per_step"] = batched_ms
    out["batched_cell_updates_per_s"] = cells / (batched_ms / 1e3)
    out["batched_roofline_frac"] = cells * 28 / (batched_ms / 1e3) / 1e9 / peaks()[0]
    seq_ms = 0.0
    t0 = time.perf_counter()
    for pth in paths:
        with Simulation(pth, device=local_rank, quiet=True, all_tiles=True) as s:
            s.step_timed(3)
            tot, _, _ = s.step_timed(args.ens_seq_steps)
            seq_ms += tot / args.ens_seq_steps
    out["sequential_ms_per_step"] = seq_ms
    out["sequential_wall_s"] = round(time.perf_counter() - t0, 1)
    out["sequential_cell_updates_per_s"] = cells / (seq_ms / 1e3)
    out["speedup_batched_vs_sequential"] = seq_ms / batched_ms
    if args.ens_spinup > 0:
        with Ensemble(paths, device=local_rank) as e:
            e.step(args.ens_spinup)
            e.autotune(steps_per_shape=10)
            inf = e.info()
            ms = e.step_timed(args.ens_steps)
            t_sim = [e.time(m)[0] for m in range(len(paths))]
        out["flooded"] = {"after_steps": args.ens_spinup, "sim_time_s_median": float(np.median(t_sim)),
                          "active_tile_fraction": inf.active_tiles / max(inf.n_tiles, 1),
                          "shape": [inf.consumer_warps, inf.tile_rows],
                          "ms_per_step": ms / args.ens_steps,
                          "whole_ensemble_cell_updates_per_s": cells * args.ens_steps / (ms / 1e3)}
    return out


def bf16_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["bf16_tflops"]), "measured"
    except Exception:
        return 1590.0, "fallback"


def surrogate_measure(args):
    """Learned surrogate: throughput of its tcgen05 convolutions (32 x 512 x 512 x 64, CUDA
    events) against the measured bf16 GEMM peak, and a reduced train / evaluate / screen run of
    fip_b200.surrogate_run (trajectories from the batched solver; see that module)."""
    from fip_b200 import surrogate_run
    from fip_b200.surrogate import bench_convs

    peak, kind = bf16_peak()
    conv = bench_convs(32, 512, 512, 10)
    out = {"conv_32x512x512": {k: {"ms": round(v["ms"], 4), "tflops": round(v["tflops"], 1),
                                   "frac_of_bf16_peak": round(v["tflops"] / peak, 3)} for k, v in conv.items()},
           "bf16_peak_tflops": peak, "peak_source": f"{kind} (MEASURED_PEAKS.json bf16_tflops)"}
    res = surrogate_run.main(["--members", str(args.sg_members), "--size", str(args.sg_size), "--hours",
                              str(args.sg_hours), "--steps", str(args.sg_steps), "--batch", str(args.sg_batch),
                              "--eval-members", "4", "--screen-members", str(args.sg_members), "--screen-size",
                              str(args.sg_size), "--screen-hours", str(args.sg_hours)], emit=False)
    out["pipeline"] = {k: v for k, v in res.items() if k != "config"}
    out["pipeline"]["config"] = {"members": args.sg_members, "size": args.sg_size, "hours": args.sg_hours,
                                 "train_steps": args.sg_steps, "batch": args.sg_batch}
    return out


def workload_config(W, H):
    """The `config` object of both arms' lines: the same workload, whichever arm measures it."""
    return {"workload": f"scenario1 large grid {W}x{H}, dx 3 m, kSt_var, no_data border, "
                        "variable dt, q inflow + open bottom; every cell computed",
            "grid_cells": W * H, "bytes_per_cell": BYTES_PER_CELL}


def run_reference(args, rank, world):
    """The reference's algorithm on the host cores: the whole scenario (every cell, its boundary
    conditions and variable dt), FP64 restatement of the reference's kernel with all host
    threads. The reference's own path is CUDA only (no CPU implementation exists)."""
    if rank != 0:
        return 0
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle

    sc = make_workload(args, rank)
    threads = os.cpu_count() or 1
    o = pyoracle.Oracle.from_yaml(sc.yaml_path, _pitch(sc.W), precision=64)
    o.set_threads(threads)
    o.simulate(max(args.warmup, 1))
    t0 = time.perf_counter()
    o.simulate(args.steps)
    dt = time.perf_counter() - t0
    value = sc.W * sc.H * args.steps / dt
    cpu = {"value": value, "unit": METRIC, "cores": threads, "kind": "port",
           "sample": f"FP64 oracle (restatement of the reference's kernel, boundary conditions and dt control), "
                     f"whole {sc.W}x{sc.H} grid, {args.steps} steps after {max(args.warmup, 1)} warm-up steps, "
                     f"{dt:.1f} s, {threads} threads"}
    cfg = workload_config(sc.W, sc.H)
    cfg["arm"] = "CPU: FP64 oracle port on the host cores (the reference has no CPU path)"
    cfg["parallelism"] = f"{threads} host threads"
    line = {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": cfg,
            "impl": "reference", "cpu_baseline": cpu,
            "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_gpu(args, rank, world, local_rank):
    import torch

    from fip_b200 import Simulation

    from fip_b200 import replicas

    torch.cuda.set_device(local_rank)
    dist = replicas.init("nccl")
    sc = make_workload(args, rank)
    W, H = sc.W, sc.H
    cells = W * H

    # ---- realistic flood state with dry-tile skipping (informational) ----
    active = None
    if args.spinup > 0:
        with Simulation(sc.yaml_path, device=local_rank, quiet=True) as sim:
            t0 = time.perf_counter()
            while sim.duration < args.spinup:
                sim.step(2000)
            spin_wall = time.perf_counter() - t0
            inf = sim.info()
            tot, st_ms, po_ms = sim.step_timed(args.steps)
            inf2 = sim.info()
            wet = float(np.mean(sim.field("h") > 1e-6))
            active = {"sim_time_s": round(inf2.duration, 1), "active_tile_fraction": inf.active_tiles / inf.n_tiles,
                      "wet_cell_fraction": wet, "whole_grid_equiv_cell_updates_per_s": cells * args.steps / (tot / 1e3),
                      "ms_per_step": tot / args.steps, "spinup_wall_s": round(spin_wall, 2)}

    # ---- headline: every tile computed ----
    sim = Simulation(sc.yaml_path, device=local_rank, quiet=True, all_tiles=True)
    sim.step_timed(max(args.warmup, 3))  # warm-up (graph build, clocks, TLB)
    replicas.barrier(dist)
    torch.cuda.synchronize()
    with Clocks(local_rank) as clk:
        total_ms, stencil_ms, post_ms = sim.step_timed(args.steps)
    torch.cuda.synchronize()
    total_ms = replicas.max_over_ranks(dist, total_ms, device="cuda")
    value = world * cells * args.steps / (total_ms / 1e3)

    # ---- e2e through the C ABI with pinned host buffers ----
    # every e2e step: the state (h, qx, qy) from pinned host buffers, `inner` solver steps, the
    # state back into pinned host buffers; the pipelined exchange (fip_stage_state /
    # fip_step_exchange) overlaps the next upload and the last download with the steps
    inner = args.e2e_inner
    pin = lambda: torch.empty((H, W), dtype=torch.float32, pin_memory=True).numpy()
    hin = [sim.field(k, out=pin()) for k in ("h", "qx", "qy")]
    hout = [[pin() for _ in range(3)] for _ in range(2)]
    reps = max(args.e2e_reps, args.steps // inner)
    sim.stage_state(*hin)  # warm the path once
    sim.step_exchange(inner, hout[0])
    sim.exchange_wait()
    replicas.barrier(dist)
    t0 = time.perf_counter()
    sim.stage_state(*hin)
    for i in range(reps):
        if i + 1 < reps:
            sim.stage_state(*hin)
        sim.step_exchange(inner, hout[i % 2])
    sim.exchange_wait()
    e2e_s = time.perf_counter() - t0
    e2e_s = replicas.max_over_ranks(dist, e2e_s, device="cuda")
    e2e_value = world * cells * inner * reps / e2e_s
    sim.close()

    peak, peak_kind = peaks()
    achieved = cells * BYTES_PER_CELL / (stencil_ms / 1e3) / 1e9
    tpc = profile_traffic()
    roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else "fallback 6.65 TB/s",
            "traffic": tpc * cells if tpc else None, "kernel": "rmg_step_kernel<true>",
            "bytes_per_launch": cells * BYTES_PER_CELL, "stencil_ms_per_launch": stencil_ms,
            "post_ms_per_launch": post_ms}
    clocks = clk.summary()
    ens = None
    if world == 1 and args.ens_members > 0:
        try:
            ens = ensemble_measure(args, local_rank)
        except Exception as exc:  # reported in the line; the headline stands on its own
            ens = {"error": f"{type(exc).__name__}: {exc}"}
    sgm = None
    if world == 1 and args.sg_members > 0:
        try:
            sgm = surrogate_measure(args)
        except Exception as exc:
            sgm = {"error": f"{type(exc).__name__}: {exc}"}
    gref = None
    if world == 1 and args.gpu_ref_seconds > 0:
        try:
            gref = gpu_reference_baseline(args, local_rank, args.gpu_ref_seconds)
        except Exception as exc:
            gref = {"error": f"{type(exc).__name__}: {exc}"[:300]}
    if rank == 0:
        base = None
        if world == 1 and not args.no_cpu_baseline:
            base = cpu_baseline(sc, args.cpu_seconds)
            if args.cpu_config0:
                base["config0"] = cpu_baseline_config0()
        line = {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": dict(workload_config(W, H), parallelism=f"replicas x{world}",
                               l2="working set 1.18 GB per step >> 126 MB L2 (no flush needed)"),
                "e2e": {"value": e2e_value, "unit": METRIC, "h2d_bytes_per_step": 3 * cells * 4,
                        "d2h_bytes_per_step": 3 * cells * 4,
                        "note": f"{reps} e2e steps, each = upload of h,qx,qy from pinned host + {inner} solver "
                                "steps + download into pinned host (fip_stage_state / fip_step_exchange: the "
                                "copies of one e2e step overlap the solver steps of its neighbours)"},
                "gpu_launches": 2 * args.steps, "roofline": roof, "clocks": clocks,
                "cpu_baseline": base, "gpu_reference": gref, "active_tiles": active, "ensemble": ens,
                "surrogate": sgm}
        print(json.dumps(line), flush=True)
    replicas.finish(dist)
    return 0


def time_to_solution(args):
    """The large-grid scenario over its whole duration (24 simulated hours, variable dt, dry-tile
    skipping) through fip_run, and optionally reference binaries (oracle/_ref) on the same
    parameter file: wall seconds and steps, and the final save_state dumps compared (flood
    plains and depth). Prints one JSON object (not a bench line)."""
    from fip_b200 import Simulation, synth

    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import refbin

    dur = args.tts_hours * 3600.0
    base = os.path.join(tempfile.gettempdir(), f"fip_tts_{os.getpid()}")

    def scenario(tag):
        return synth.scenario1(os.path.join(base, tag), W=args.W, H=args.H, seed=1, duration=dur, name="tts",
                               save_state=[f"{dur:g}"])

    sc = scenario("ours")
    out = {"workload": f"scenario1 {sc.W}x{sc.H}, {args.tts_hours:g} simulated hours, variable dt"}
    with Simulation(sc.yaml_path, quiet=True) as sim:
        t0 = time.perf_counter()
        sim.run()
        wall = time.perf_counter() - t0
        inf = sim.info()
        out["fip_b200"] = {"wall_s": wall, "steps": sim.iteration, "s_per_step": wall / sim.iteration,
                           "final_dt": sim.time()[1], "active_tile_fraction_end": inf.active_tiles / inf.n_tiles}
    ours = refbin.dumps(os.path.join(base, "ours", "tts"))
    for name in [x for x in args.tts_reference.split(",") if x]:
        sr = scenario(name)
        r = refbin.run(name, sr.yaml_path, timeout=7200)
        o = {"seconds": r["seconds"], "steps": r["iterations"], "s_per_step": r["seconds"] / r["iterations"],
             "speedup_wall": r["seconds"] / wall}
        ref = refbin.dumps(os.path.join(base, name, "tts"))
        for kind in ("flood_plains", "ah"):
            key = [k for k in ref if k[0] == kind]
            if key and key[0] in ours:
                a_, b_ = ref[key[0]].astype(np.float64), ours[key[0]].astype(np.float64)
                d = np.abs(a_ - b_)
                wa, wb = a_ > 0.05, b_ > 0.05
                u = np.logical_or(wa, wb).sum()
                o[kind] = {"max_abs_diff": float(d.max()), "rmse": float(np.sqrt((d ** 2).mean())),
                           "cells_over_1e-4": float((d > 1e-4).mean()),
                           "extent_iou_5cm": float(np.logical_and(wa, wb).sum() / u) if u else 1.0}
        out[name] = o
    print(json.dumps(out), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="fip_b200", choices=["fip_b200", "reference"])
    ap.add_argument("--W", type=int, default=5667)
    ap.add_argument("--H", type=int, default=6500)
    ap.add_argument("--spinup", type=float, default=7200.0, help="simulated s before the active-tile measurement")
    ap.add_argument("--e2e-inner", type=int, default=100)
    ap.add_argument("--e2e-reps", type=int, default=8, help="e2e steps (at least; more when --steps is larger)")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-config0", action="store_true",
                    help="also time the oracle port over the full 1024x1024, 10000-step case")
    ap.add_argument("--gpu-ref-seconds", type=float, default=120.0,
                    help="simulated s of the reference-binary baseline on this GPU (0: skip)")
    ap.add_argument("--ens-members", type=int, default=64, help="batched-ensemble measurement (0: skip)")
    ap.add_argument("--ens-steps", type=int, default=200)
    ap.add_argument("--ens-seq-steps", type=int, default=20)
    ap.add_argument("--ens-spinup", type=int, default=3000)
    ap.add_argument("--sg-members", type=int, default=16, help="surrogate measurement (0: skip)")
    ap.add_argument("--sg-size", type=int, default=512)
    ap.add_argument("--sg-hours", type=float, default=0.5)
    ap.add_argument("--sg-steps", type=int, default=300)
    ap.add_argument("--sg-batch", type=int, default=16)
    ap.add_argument("--tts", action="store_true", help="only the time-to-solution run of the large grid")
    ap.add_argument("--tts-hours", type=float, default=24.0)
    ap.add_argument("--tts-reference", default="",
                    help="comma-separated reference binaries (oracle/_ref) to run for --tts, e.g. fip_ref_sync")
    args = ap.parse_args()
    if args.tts:
        return time_to_solution(args)
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)
    return run_gpu(args, rank, world, local_rank)


if __name__ == "__main__":
    sys.exit(main())
