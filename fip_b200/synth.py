"""Seeded synthetic scenarios in fip's input format (YAML + raw float32 grids + `;` CSV series).

The reference ships no example inputs, so every workload here is generated: terrain, roughness,
initial state and hydrographs are written as the files the reference's loader reads
(src/simdata.cpp:143-150: raw float32 W*H at a byte offset; src/timeseries.cpp:28-84: `;`
separated CSV with a header line) and a YAML file with the keys of README.md:46-64.

Scenarios:
  * ``scenario0`` -- the 1024x1024 plain-solver case: plane sloping 0.001 in -x, 40 seeded
    Gaussian bumps (amplitude U[-3,5] m, sigma U[20,120] cells), a 2 m deep channel 30 cells
    wide along y=H/2, kSt 30, dry start, left z inflow on rows 480-544 at the lowest terrain of
    those rows + 2.5 m, right open, top and bottom closed, fixed dt 0.1 s.
  * ``scenario1`` -- the 5667x6500 large grid: fBm terrain (Hurst 0.8, 40 m relief) tilted
    towards the bottom edge with a meandering channel 60 cells wide and 4 m deep, kSt_var (25 on
    a 30% land-use mask, 40 elsewhere), no_data=-1 on a 5% irregular border band along the top
    and right edges, variable dt, left q inflow over 200 cells with a triangular hydrograph
    0 -> 1500 -> 200 m3/s peaking at 6 h (plus the z series the q type requires: channel bed +
    a stage that follows the discharge), bottom open.
Both accept smaller W/H for tests; sizes and every random draw come from the seed.
"""
from __future__ import annotations

import os
from dataclasses import dataclass, field

import numpy as np


@dataclass
class Scenario:
    yaml_path: str
    W: int
    H: int
    terrain: np.ndarray
    h0: np.ndarray | None = None
    qx0: np.ndarray | None = None
    qy0: np.ndarray | None = None
    kst_var: np.ndarray | None = None
    info: dict = field(default_factory=dict)


def write_grid(path: str, arr: np.ndarray, offset: int = 0) -> None:
    """Raw float32 row-major grid, optionally behind `offset` header bytes."""
    a = np.ascontiguousarray(arr, dtype=np.float32)
    with open(path, "wb") as f:
        if offset:
            f.write(b"\0" * offset)
        f.write(a.tobytes())


def write_series(path: str, times, values, header: str = "t;v", dates: bool = False) -> None:
    """`;` separated CSV, header line first (skipped by the reader); time in seconds or as
    %d.%m.%Y %H:%M:%S stamps counted from the first row."""
    import datetime as _dt

    base = _dt.datetime(2021, 7, 14, 0, 0, 0)
    with open(path, "w") as f:
        f.write(header + "\n")
        for t, v in zip(times, values):
            if dates:
                ts = (base + _dt.timedelta(seconds=float(t))).strftime("%d.%m.%Y %H:%M:%S")
                f.write(f"{ts};{v:.9g}\n")
            else:
                f.write(f"{t:.9g};{v:.9g}\n")


def _fmt(v):
    if isinstance(v, bool):
        return "true" if v else "false"
    return str(v)


def write_yaml(path: str, cfg: dict) -> None:
    """Block-style YAML of the reference schema (README.md:46-64)."""
    lines = []
    for k, v in cfg.items():
        if k.startswith("#"):
            lines.append(f"# {v}")
        elif k == "boundary_conditions" or k == "sampling":
            lines.append(f"{k}:")
            for item in v:
                first = True
                for kk, vv in item.items():
                    lead = "  - " if first else "    "
                    first = False
                    if isinstance(vv, (list, tuple)):
                        vv = "[" + ", ".join(_fmt(x) for x in vv) + "]"
                    lines.append(f"{lead}{kk}: {_fmt(vv)}")
        elif k == "save_state":
            lines.append(f"{k}:")
            for item in v:
                lines.append(f"  - {item}")
        elif isinstance(v, (list, tuple)):
            lines.append(f"{k}: [" + ", ".join(_fmt(x) for x in v) + "]")
        else:
            lines.append(f"{k}: {_fmt(v)}")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def terrain0(W: int, H: int, dx: float, seed: int) -> np.ndarray:
    """Plane -0.001*x*dx + 40 Gaussian bumps - a 2 m channel, 30 cells wide, along y=H/2.
    Bump sigmas and the channel width scale with min(W,H)/1024 for small test grids."""
    rng = np.random.default_rng(seed)
    scale = min(W, H) / 1024.0
    x = np.arange(W, dtype=np.float64)[None, :]
    y = np.arange(H, dtype=np.float64)[:, None]
    z = -0.001 * x * dx + 0.0 * y
    for _ in range(40):
        cx, cy = rng.uniform(0, W), rng.uniform(0, H)
        amp = rng.uniform(-3.0, 5.0)
        sig = rng.uniform(20.0, 120.0) * scale
        z = z + amp * np.exp(-((x - cx) ** 2 + (y - cy) ** 2) / (2 * sig * sig))
    half = max(1, int(round(15 * scale)))
    yc = H // 2
    z[max(0, yc - half):yc + half, :] -= 2.0
    return z.astype(np.float32)


def scenario0(outdir: str, W: int = 1024, H: int = 1024, dx: float = 3.0, dt: float = 0.1,
              duration: float = 1000.0, save_every: float = 100.0, seed: int = 0,
              sampling_interval: int = 0, variable_dt: bool = False, name: str = "scenario0",
              bc_rows: tuple[int, int] | None = None, kst: float = 30.0, level_add: float = 0.0) -> Scenario:
    os.makedirs(outdir, exist_ok=True)
    terr = terrain0(W, H, dx, seed)
    if bc_rows is None:
        bc_rows = (480, 544) if (W, H) == (1024, 1024) else (H // 2 - H // 16, H // 2 + H // 16)
    lo, hi = bc_rows
    zbc = float(terr[lo:hi + 1, 0].min()) + 2.5 + level_add
    tpath = os.path.join(outdir, f"{name}_terrain.bin")
    write_grid(tpath, terr)
    cfg = {
        "#0": f"seed {seed}: terrain0(W={W}, H={H}, dx={dx}); left z level = min terrain of rows "
              f"{lo}-{hi} + 2.5 m + {level_add:.6g} m; kSt {kst:.6g}",
        "name": os.path.join(outdir, name),
        "terrain": [tpath, 0],
        "W": W, "H": H, "dx": dx, "dt": dt,
        "duration": duration,
        "kSt": 30 if kst == 30.0 else f"{kst:.9g}",
        "variable_dt": variable_dt,
        "boundary_conditions": [
            {"side": "left", "type": "z", "z": f"{zbc:.9g}", "from": lo, "to": hi},
            {"side": "right", "type": "open"},
            {"side": "top", "type": "close"},
            {"side": "bottom", "type": "close"},
        ],
    }
    if save_every and save_every > 0:
        n = int(round(duration / save_every))
        cfg["save_state"] = [f"{save_every * (k + 1):g}" for k in range(n)]
    if sampling_interval:
        cfg["sampling_interval"] = sampling_interval
        cfg["sampling"] = [
            {"x": 2, "y": (lo + hi) // 2, "label": "inflow", "type": "z"},
            {"x": W // 8, "y": H // 2, "label": "channel_h", "type": "h"},
            {"x": W // 8, "y": H // 2, "label": "channel_qx", "type": "qx"},
            {"x": W // 8, "y": H // 2 + 2, "label": "channel_qy", "type": "qy"},
        ]
    ypath = os.path.join(outdir, f"{name}.yml")
    write_yaml(ypath, cfg)
    return Scenario(ypath, W, H, terr, info={"zbc": zbc, "bc_rows": bc_rows, "kst": kst, "level_add": level_add})


def fbm(W: int, H: int, hurst: float, seed: int) -> np.ndarray:
    """Spectral fractional Brownian surface, zero mean, unit peak-to-peak."""
    rng = np.random.default_rng(seed)
    ky = np.fft.fftfreq(H)[:, None]
    kx = np.fft.rfftfreq(W)[None, :]
    k = np.sqrt(kx * kx + ky * ky).astype(np.float32)
    k[0, 0] = 1.0
    amp = k ** np.float32(-(hurst + 1.0))
    amp[0, 0] = 0.0
    ph = rng.uniform(0, 2 * np.pi, size=amp.shape).astype(np.float32)
    spec = (amp * np.exp(1j * ph)).astype(np.complex64)
    z = np.fft.irfft2(spec, s=(H, W)).astype(np.float32)
    z -= z.min()
    z /= max(float(z.max()), 1e-12)
    return z - 0.5


def scenario1(outdir: str, W: int = 5667, H: int = 6500, dx: float = 3.0, dt: float = 0.5,
              duration: float = 3600.0 * 24, seed: int = 1, name: str = "scenario1",
              inflow_cells: int = 200, q_peak: float = 1500.0, t_peak: float = 6 * 3600.0,
              q_end: float = 200.0, channel_width: int = 60, save_state: list | None = None,
              variable_dt: bool = True, wet_start: bool = False) -> Scenario:
    os.makedirs(outdir, exist_ok=True)
    rng = np.random.default_rng(seed)
    scale = min(W, H) / 5667.0
    relief = 40.0
    z = fbm(W, H, 0.8, seed) * relief
    y = np.arange(H, dtype=np.float32)[:, None]
    x = np.arange(W, dtype=np.float32)[None, :]
    # regional tilt towards the bottom edge and away from the left inflow
    z = z + 0.002 * dx * y + 0.0005 * dx * (W - x) * 0.0
    # meandering channel from the left edge (row 0.6 H) down to the bottom edge (row 0)
    y0 = H * 0.6
    xs = np.arange(W, dtype=np.float32)
    lam = max(64.0, 1800.0 * scale)
    amp_m = 300.0 * scale
    ycl = y0 - (H * 0.75) * (xs / max(W - 1, 1)) ** 1.3 + amp_m * np.sin(2 * np.pi * xs / lam)
    half = max(2, int(round(channel_width * max(scale, 0.05) / 2)))
    bed_start = float(np.percentile(z, 20)) - 4.0
    bed_end = bed_start - 0.0008 * dx * W
    bed = bed_start + (bed_end - bed_start) * xs / max(W - 1, 1)
    dist = np.abs(y - ycl[None, :])
    inch = dist <= half
    z = np.where(inch, np.minimum(z, bed[None, :] + 0.0), z)
    # levee-free floodplain: soften the banks over one channel width
    bank = (dist > half) & (dist <= 3 * half)
    z = np.where(bank, np.minimum(z, bed[None, :] + 4.0 + (dist - half) * (2.0 / max(half, 1))), z)
    z = z.astype(np.float32)
    # no_data: irregular band along the top and right edges, about 5% of the cells
    no_data = -1.0
    noise = fbm(W, H, 0.5, seed + 7)
    band = 0.025 * (1.0 + 1.2 * noise)
    fy = (H - 1 - y) / H
    fx = (W - 1 - x) / W
    mask_nd = (fy < band) | (fx < band)
    z = np.where(mask_nd, np.float32(no_data), z).astype(np.float32)
    # kSt_var: 25 on a 30% land-use mask, 40 elsewhere
    lu = fbm(W, H, 0.6, seed + 11)
    thr = np.quantile(lu[:: max(1, H // 512), :: max(1, W // 512)], 0.7)
    kst = np.where(lu > thr, np.float32(25.0), np.float32(40.0)).astype(np.float32)
    # inflow: left edge, `inflow_cells` rows centred on the channel entry
    n_in = max(4, int(round(inflow_cells * max(scale, 0.02))))
    r0 = int(np.clip(int(ycl[0]) - n_in // 2, 1, H - n_in - 2))
    r1 = r0 + n_in
    terr_in = z[r0:r1, 0]
    bed_in = float(terr_in.min())
    # triangular hydrograph 0 -> q_peak (t_peak) -> q_end (end), 10 min resolution
    ts = np.arange(0.0, duration + 600.0, 600.0)
    qs = np.where(ts <= t_peak, q_peak * ts / t_peak,
                  q_peak + (q_end - q_peak) * (ts - t_peak) / max(duration - t_peak, 1.0))
    qs = np.maximum(qs, 0.0) * (max(scale, 0.02) if scale < 1 else 1.0)
    stage = 0.5 + 3.5 * (qs / max(q_peak, 1e-9)) ** 0.6
    zs = bed_in + stage
    tpath = os.path.join(outdir, f"{name}_terrain.bin")
    kpath = os.path.join(outdir, f"{name}_kst.bin")
    write_grid(tpath, z, offset=16)
    write_grid(kpath, kst, offset=16)
    qpath = os.path.join(outdir, f"{name}_q.csv")
    zpath = os.path.join(outdir, f"{name}_z.csv")
    write_series(qpath, ts, qs, header="time;discharge")
    write_series(zpath, ts, zs, header="time;stage")
    init = {}
    if wet_start:
        # flooded start: water up to a level 1.5 m above the 35th terrain percentile (ponds and the
        # channel), discharges from smooth seeded fields (|u| <= 0.3 m/s) in the wet cells, dry on
        # no_data cells
        level = float(np.percentile(z[~mask_nd], 35)) + 1.5
        depth = np.clip(level - z, 0.0, 6.0).astype(np.float32)
        depth[mask_nd] = 0.0
        wet = depth > 0
        ux = 0.6 * fbm(W, H, 0.9, seed + 23)
        uy = 0.6 * fbm(W, H, 0.9, seed + 29)
        qx0 = np.where(wet, depth * ux, 0.0).astype(np.float32)
        qy0 = np.where(wet, depth * uy, 0.0).astype(np.float32)
        for k, a in (("z", z + depth), ("qx", qx0), ("qy", qy0)):
            path = os.path.join(outdir, f"{name}_{k}0.bin")
            write_grid(path, a.astype(np.float32))
            init[k] = [path, 0]
    cfg = {
        "#0": f"seed {seed}: scenario1(W={W}, H={H}{', wet start' if wet_start else ''}); inflow rows {r0}-{r1 - 1}",
        "name": os.path.join(outdir, name),
        "terrain": [tpath, 16],
        "W": W, "H": H, "dx": dx, "dt": dt,
        "duration": "3600*24" if duration == 3600.0 * 24 else duration,
        "kSt_var": [kpath, 16],
        **init,
        "no_data": no_data,
        "variable_dt": variable_dt,
        "boundary_conditions": [
            {"side": "left", "type": "q", "q": [qpath, 0, 1], "z": [zpath, 0, 1],
             "from": r0, "to": r1 - 1},
            {"side": "bottom", "type": "open"},
        ],
    }
    if save_state:
        cfg["save_state"] = save_state
    ypath = os.path.join(outdir, f"{name}.yml")
    write_yaml(ypath, cfg)
    return Scenario(ypath, W, H, z, kst_var=kst,
                    info={"inflow_rows": (r0, r1 - 1), "no_data": no_data,
                          "series": (ts, qs, zs)})


def ensemble_member(outdir: str, W: int, H: int, seed: int, kst: float = 30.0, q_peak: float = 1000.0,
                    t_peak: float = 3 * 3600.0, duration: float = 6 * 3600.0, dx: float = 3.0, dt: float = 0.5,
                    name: str | None = None, right: str = "open", bottom: str | None = None) -> Scenario:
    """One member of the batched ensemble: fBm valley (Hurst 0.8) draining to the right edge with
    a meandering channel, uniform kSt, dry start, variable dt, left q inflow over the channel
    entry with a triangular hydrograph 0 -> q_peak (at t_peak) -> q_peak / 5 (at the end) plus the
    stage series the q type requires, right edge `right`, top and bottom closed unless `bottom`
    names a type."""
    os.makedirs(outdir, exist_ok=True)
    name = name or f"member{seed}"
    scale = min(W, H) / 1024.0
    y = np.arange(H, dtype=np.float32)[:, None]
    x = np.arange(W, dtype=np.float32)[None, :]
    relief = 6.0 * max(scale, 0.25) ** 0.5
    z = fbm(W, H, 0.8, seed) * relief
    xs = np.arange(W, dtype=np.float32)
    yc = H * 0.5 + 0.2 * H * np.sin(2 * np.pi * xs / max(W * 0.7, 16.0))
    # valley: banks rising away from the channel, the floor falling towards the right edge
    dist = np.abs(y - yc[None, :])
    z = z + 0.004 * dx * dist - 0.001 * dx * x
    half = max(2, int(round(20 * scale)))
    z = np.where(dist <= half, z - 2.5, z).astype(np.float32)
    n_in = max(4, min(H - 4, 2 * half + 4))
    r0 = int(np.clip(int(yc[0]) - n_in // 2, 1, H - n_in - 2))
    r1 = r0 + n_in
    bed_in = float(z[r0:r1, 0].min())
    ts = np.arange(0.0, duration + 600.0, 600.0)
    qs = np.where(ts <= t_peak, q_peak * ts / max(t_peak, 1.0),
                  q_peak + (0.2 * q_peak - q_peak) * (ts - t_peak) / max(duration - t_peak, 1.0))
    qs = np.maximum(qs, 0.0)
    stage = 0.3 + 2.5 * (qs / max(q_peak, 1e-9)) ** 0.6
    zs = bed_in + stage
    tpath = os.path.join(outdir, f"{name}_terrain.bin")
    write_grid(tpath, z)
    qpath = os.path.join(outdir, f"{name}_q.csv")
    zpath = os.path.join(outdir, f"{name}_z.csv")
    write_series(qpath, ts, qs, header="time;discharge")
    write_series(zpath, ts, zs, header="time;stage")
    bcs = [{"side": "left", "type": "q", "q": [qpath, 0, 1], "z": [zpath, 0, 1], "from": r0, "to": r1 - 1},
           {"side": "right", "type": right}]
    if bottom:
        bcs.append({"side": "bottom", "type": bottom})
    cfg = {
        "#0": f"seed {seed}: ensemble_member(W={W}, H={H}, kSt={kst:.4g}, q_peak={q_peak:.6g}, t_peak={t_peak:.6g})",
        "name": os.path.join(outdir, name),
        "terrain": [tpath, 0],
        "W": W, "H": H, "dx": dx, "dt": dt,
        "duration": duration,
        "kSt": f"{kst:.9g}",
        "variable_dt": True,
        "boundary_conditions": bcs,
    }
    ypath = os.path.join(outdir, f"{name}.yml")
    write_yaml(ypath, cfg)
    return Scenario(ypath, W, H, z, info={"inflow_rows": (r0, r1 - 1), "kst": kst, "q_peak": q_peak,
                                          "t_peak": t_peak})


def ensemble2(outdir: str, n: int = 64, seed: int = 2, size_lo: int = 256, size_hi: int = 2048,
              duration: float = 6 * 3600.0) -> list:
    """The batched-ensemble workload: n members with W, H ~ U[size_lo, size_hi], their own fBm
    seeds, kSt ~ U[20, 45], hydrograph peak ~ U[200, 2000] m3/s at U[1, 8] h, 6 simulated hours."""
    rng = np.random.default_rng(seed)
    out = []
    for m in range(n):
        W = int(rng.integers(size_lo, size_hi + 1))
        H = int(rng.integers(size_lo, size_hi + 1))
        kst = float(rng.uniform(20.0, 45.0))
        q_peak = float(rng.uniform(200.0, 2000.0))
        t_peak = float(rng.uniform(1.0, 8.0)) * 3600.0
        out.append(ensemble_member(outdir, W, H, seed=1000 * seed + m, kst=kst, q_peak=q_peak, t_peak=t_peak,
                                   duration=duration, name=f"m{m:03d}"))
    return out
