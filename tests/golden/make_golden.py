"""Generate the golden fixtures in tests/golden/ by running the fip reference itself.

The reference has no tests, golden vectors or example inputs, so its own binary is the only pin:
oracle/ref.mk builds it from the reference sources into oracle/_ref/ (fip_ref as shipped,
fip_ref_nomask with the wet/dry mask off, fip_ref_sync = nomask + synchronised CFL readback).
This script needs a GPU: it writes small seeded scenarios, runs those binaries on them and
packs inputs, the stdout sampling CSV and every save_state dump into one .npz per case.

    python tests/golden/make_golden.py --out /tmp/golden      (then copy the .npz files here)

Grid sizes avoid the reference's two halo-lane defects (W mod 28 in {2,3,5}, H mod 50 in {2,3}).
The cudaMallocPitch row pitch of each W is recorded, since the reference's open boundary on the
top/bottom sides multiplies its outflow by it.
"""
from __future__ import annotations

import argparse
import ctypes
import glob
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from fip_b200 import synth  # noqa: E402

REF_DIR = os.path.join(ROOT, "oracle", "_ref")


def malloc_pitch(width_bytes: int, height: int) -> int:
    rt = ctypes.CDLL("libcudart.so")
    ptr = ctypes.c_void_p()
    pitch = ctypes.c_size_t()
    rc = rt.cudaMallocPitch(ctypes.byref(ptr), ctypes.byref(pitch), ctypes.c_size_t(width_bytes),
                            ctypes.c_size_t(height))
    if rc != 0:
        raise RuntimeError(f"cudaMallocPitch failed: {rc}")
    rt.cudaFree(ptr)
    return int(pitch.value)


def read_dump(path: str):
    with open(path, "rb") as f:
        w, h = np.frombuffer(f.read(16), dtype=np.uint64)
        a = np.frombuffer(f.read(), dtype=np.float32)
    return a.reshape(int(h), int(w))


def input_files(yaml_path: str, work: str) -> dict:
    """Every file the YAML names, stored verbatim so a test can re-create the case."""
    with open(yaml_path) as f:
        text = f.read()
    files = {}
    for fn in sorted(os.listdir(work)):
        full = os.path.join(work, fn)
        if os.path.isfile(full) and full in text:
            with open(full, "rb") as f:
                files["file:" + fn] = np.frombuffer(f.read(), dtype=np.uint8)
    return files


def run_case(name: str, binary: str, yaml_path: str, work: str, meta: dict, arrays: dict, out: str):
    exe = os.path.join(REF_DIR, binary)
    arrays = dict(arrays, **input_files(yaml_path, work))
    meta = dict(meta, workdir=work)
    p = subprocess.run([exe, yaml_path], cwd=work, capture_output=True, text=True, timeout=600)
    if p.returncode != 0:
        raise RuntimeError(f"{name}: {binary} exited {p.returncode}\n{p.stderr}")
    prefix = meta["name"]
    dumps = {}
    for kind in ("ah", "qx", "qy", "flood_plains"):
        for f in sorted(glob.glob(f"{prefix}_{kind}_*")):
            t = int(os.path.basename(f)[len(os.path.basename(prefix)) + len(kind) + 2:].split("_")[0])
            dumps[f"dump_{kind}_{t}"] = read_dump(f)
    with open(yaml_path) as f:
        ytext = f.read()
    meta = dict(meta, binary=binary, stderr=p.stderr.strip().splitlines()[-1] if p.stderr.strip() else "")
    np.savez_compressed(os.path.join(out, f"{name}.npz"), yaml=np.array(ytext), stdout=np.array(p.stdout),
                        meta=np.array(json.dumps(meta)), **arrays, **dumps)
    print(f"{name}: {binary} ok, {len(dumps)} dump fields, stdout {len(p.stdout)} bytes")


def case_g0(work: str, out: str, binary: str, tag: str):
    s = synth.scenario0(work, W=100, H=90, duration=30, save_every=10, sampling_interval=5,
                        name=f"g0{tag}")
    meta = {"W": 100, "H": 90, "pitch_bytes": malloc_pitch(100 * 4, 93), "name": os.path.join(work, f"g0{tag}"),
            "steps": 300}
    run_case(f"g0_z_open_close{tag}", binary, s.yaml_path, work, meta, {}, out)


def case_g2(work: str, out: str):
    s = synth.scenario0(work, W=100, H=90, duration=60, save_every=20, sampling_interval=10,
                        variable_dt=True, name="g2")
    meta = {"W": 100, "H": 90, "pitch_bytes": malloc_pitch(100 * 4, 93), "name": os.path.join(work, "g2")}
    run_case("g2_variable_dt", "fip_ref_sync", s.yaml_path, work, meta, {}, out)


def case_g1(work: str, out: str):
    """Wet start with velocities, kSt_var, interior no_data cells, q inflow from CSV series (the z
    series with date stamps), top z, right close, bottom open (outflow scaled by the pitch)."""
    W, H = 72, 64
    rng = np.random.default_rng(42)
    y = np.arange(H, dtype=np.float32)[:, None]
    x = np.arange(W, dtype=np.float32)[None, :]
    terr = (0.02 * y + 0.01 * (W - x) + 0.3 * np.sin(x / 7.0) * np.cos(y / 5.0)).astype(np.float32)
    terr[20:24, 30:33] = -9999.0  # interior no_data block (default no_data value)
    depth = np.clip(0.4 + 0.3 * np.sin(x / 9.0 + y / 11.0) - 0.01 * y, 0.0, None).astype(np.float32)
    depth[rng.random((H, W)) < 0.1] = 0.0
    z0 = (terr + depth).astype(np.float32)
    qx0 = (0.05 * np.cos(y / 6.0) * (depth > 0)).astype(np.float32)
    qy0 = (-0.04 * np.sin(x / 8.0) * (depth > 0)).astype(np.float32)
    kst = np.where(rng.random((H, W)) < 0.3, 25.0, 40.0).astype(np.float32)
    paths = {}
    for k, a, off in (("terrain", terr, 36), ("z", z0, 0), ("qx", qx0, 16), ("qy", qy0, 16), ("kst", kst, 36)):
        paths[k] = os.path.join(work, f"g1_{k}.bin")
        synth.write_grid(paths[k], a, offset=off)
    ts = np.array([0.0, 1.0, 2.5, 4.0, 10.0])
    synth.write_series(os.path.join(work, "g1_q.csv"), ts, [0.0, 2.0, 5.0, 3.0, 1.0], header="t;q")
    synth.write_series(os.path.join(work, "g1_z.csv"), ts, [1.9, 2.0, 2.3, 2.2, 2.0], header="t;z", dates=True)
    cfg = {
        "name": os.path.join(work, "g1"),
        "terrain": [paths["terrain"], 36], "z": [paths["z"], 0], "qx": [paths["qx"], 16],
        "qy": [paths["qy"], 16], "kSt_var": [paths["kst"], 36],
        "W": W, "H": H, "dx": 2.0, "dt": 0.05, "duration": 5, "variable_dt": False,
        "boundary_conditions": [
            {"side": "left", "type": "q", "q": [os.path.join(work, "g1_q.csv"), 0, 1],
             "z": [os.path.join(work, "g1_z.csv"), 0, 1], "from": 10, "to": 40},
            {"side": "bottom", "type": "open", "from": 5, "to": 60},
            {"side": "top", "type": "z", "z": 1.85},
            {"side": "right", "type": "close"},
        ],
        "save_state": ["1", "3", "5"],
        "sampling_interval": 1,
        "sampling": [{"x": 1, "y": 20, "label": "in_z", "type": "z"},
                     {"x": 35, "y": 2, "label": "out_qy", "type": "qy"},
                     {"x": 36, "y": 32, "label": "mid_qx", "type": "qx"},
                     {"x": 36, "y": 62, "label": "top_h", "type": "h"}],
    }
    ypath = os.path.join(work, "g1.yml")
    synth.write_yaml(ypath, cfg)
    meta = {"W": W, "H": H, "pitch_bytes": malloc_pitch(W * 4, H + 3), "name": cfg["name"], "steps": 100}
    run_case("g1_wet_q_open", "fip_ref_nomask", ypath, work, meta, {}, out)


def case_g3(work: str, out: str):
    s = synth.scenario1(work, W=128, H=120, duration=600.0, name="g3",
                        save_state=["200", "400", "600"])
    meta = {"W": 128, "H": 120, "pitch_bytes": malloc_pitch(128 * 4, 123), "name": os.path.join(work, "g3")}
    run_case("g3_scenario1_small", "fip_ref_sync", s.yaml_path, work, meta, {}, out)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True, help="directory for the .npz fixtures")
    args = ap.parse_args()
    os.makedirs(args.out, exist_ok=True)
    with tempfile.TemporaryDirectory() as work:
        case_g0(work, args.out, "fip_ref_nomask", "")
        case_g0(work, args.out, "fip_ref", "_mask")
        case_g1(work, args.out)
        case_g2(work, args.out)
        case_g3(work, args.out)


if __name__ == "__main__":
    main()
