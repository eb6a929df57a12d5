"""Runs the fip reference binaries built by oracle/ref.mk (oracle/_ref/). TEST INFRASTRUCTURE ONLY.

The reference has no tests or golden vectors, so its own binary is the parity pin: tests/ run it
on the same parameter file as the CUDA path and compare dumps, sampling rows and step counts;
bench.py's baseline legs run it to time the reference's own CUDA kernels beside the CPU oracle.
The product never calls anything here.

Binaries (see oracle/ref.mk):
  fip_ref         as shipped (wet/dry mask on; the host reads the CFL slots unsynchronised)
  fip_ref_nomask  ENABLE_MASK 0 (every strip computed; deterministic for fixed dt)
  fip_ref_sync    nomask + a synchronised CFL readback (deterministic for variable dt)

The headless reference prints `Finished N iterations after S s (x s/it)` on stderr, S being CUDA
event time around its whole `while (duration < target_duration) simulate();` loop
(src/main.cpp:238-253); `run()` parses it.
"""
from __future__ import annotations

import glob
import os
import re
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(_HERE, "_ref")
KINDS = ("ah", "qx", "qy", "flood_plains")
_FINISHED = re.compile(r"Finished (\d+) iterations after ([0-9.eE+-]+) s \(([0-9.eE+-]+) s/it\)")


def binary(name: str) -> str | None:
    """Path of oracle/_ref/<name> when it was built, else None."""
    p = os.path.join(REF_DIR, name)
    return p if os.access(p, os.X_OK) else None


def parse_finished(stderr: str):
    """(iterations, seconds, s_per_it) from the reference's stderr timing line, or None."""
    m = None
    for m in _FINISHED.finditer(stderr):
        pass
    if m is None:
        return None
    return int(m.group(1)), float(m.group(2)), float(m.group(3))


def run(name: str, yaml_path: str, cwd: str | None = None, timeout: float = 900.0) -> dict:
    """Runs reference binary `name` on `yaml_path`; raises if it is missing or fails."""
    exe = binary(name)
    if exe is None:
        raise FileNotFoundError(f"reference binary oracle/_ref/{name} not built (make -f oracle/ref.mk)")
    p = subprocess.run([exe, yaml_path], cwd=cwd or os.path.dirname(os.path.abspath(yaml_path)),
                       capture_output=True, text=True, timeout=timeout)
    if p.returncode != 0:
        raise RuntimeError(f"{name} exited {p.returncode}: {p.stderr[-2000:]}")
    fin = parse_finished(p.stderr)
    if fin is None:
        raise RuntimeError(f"{name}: no timing line on stderr: {p.stderr[-2000:]}")
    it, sec, spi = fin
    return {"iterations": it, "seconds": sec, "s_per_it": spi, "stdout": p.stdout, "stderr": p.stderr}


def read_dump(path: str) -> np.ndarray:
    """A save_state file: size_t W, size_t H (16 bytes) + W*H float32 (src/main.cpp:154-170)."""
    with open(path, "rb") as f:
        w, h = np.frombuffer(f.read(16), dtype=np.uint64)
        return np.frombuffer(f.read(), dtype=np.float32).reshape(int(h), int(w))


def dumps(prefix: str) -> dict:
    """{(kind, int_time): array} of every dump written under `prefix` (the YAML `name`)."""
    base = os.path.basename(prefix)
    out = {}
    for kind in KINDS:
        for f in sorted(glob.glob(f"{prefix}_{kind}_*")):
            t = int(os.path.basename(f)[len(base) + len(kind) + 2:].split("_")[0])
            out[(kind, t)] = read_dump(f)
    return out
