"""ctypes front-end of the CPU oracle (oracle/liboracle.so). TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference arm import this
module, as the checker: the product never routes through it.

`Oracle.from_yaml` restates the reference's input handling for the oracle side
(src/simdata.cpp:238-310 loadSimData, :98-131 createBoundaryCondition,
src/timeseries.cpp:28-84 fromCsv, src/utils.h:29-43 solveSimpleMathExpression) with PyYAML,
independently of the product's own C++ YAML reader, so the two cross-check each other.
"""
from __future__ import annotations

import ctypes
import math
import os
import time as _time

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

SIDES = {"left": 0, "right": 1, "top": 2, "bottom": 3}
TYPES = {"z": 0, "q": 1, "close": 2, "open": 3}
SAMPLE_TYPES = {"z": 0, "h": 1, "qx": 2, "qy": 3}
F_H, F_QX, F_QY, F_H_OTHER, F_QX_OTHER, F_QY_OTHER, F_HMAX = range(7)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            raise RuntimeError("oracle/liboracle.so missing: run `make -C oracle`")
        L = ctypes.CDLL(path)
        fp = ctypes.POINTER(ctypes.c_float)
        ip = ctypes.POINTER(ctypes.c_int)
        for P in ("ora64_", "ora32_"):
            f = getattr(L, P + "new_sim")
            f.restype = ctypes.c_void_p
            f.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_long, ctypes.c_float, ctypes.c_float,
                          ctypes.c_int, ctypes.c_float, ctypes.c_float, fp, fp, fp, fp, fp]
            f = getattr(L, P + "add_bc")
            f.restype = ctypes.c_int
            f.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                          ctypes.c_int, ctypes.c_float, ctypes.c_float, ctypes.c_int, fp, fp,
                          ctypes.c_int, fp, fp]
            getattr(L, P + "set_sampling").argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ip, ip, ip]
            getattr(L, P + "set_save_times").argtypes = [ctypes.c_void_p, ctypes.c_int,
                                                         ctypes.POINTER(ctypes.c_double)]
            getattr(L, P + "set_threads").argtypes = [ctypes.c_void_p, ctypes.c_int]
            for name, rt in (("simulate", ctypes.c_int), ("run_to", ctypes.c_int)):
                f = getattr(L, P + name)
                f.restype = rt
            getattr(L, P + "simulate").argtypes = [ctypes.c_void_p, ctypes.c_int]
            getattr(L, P + "run_to").argtypes = [ctypes.c_void_p, ctypes.c_double]
            for name, rt in (("duration", ctypes.c_double), ("dt", ctypes.c_float),
                             ("iteration", ctypes.c_int), ("last_cfl", ctypes.c_float),
                             ("volume", ctypes.c_double), ("sample_text", ctypes.c_char_p),
                             ("dump_count", ctypes.c_int)):
                f = getattr(L, P + name)
                f.restype = rt
                f.argtypes = [ctypes.c_void_p]
            f = getattr(L, P + "dump_duration")
            f.restype = ctypes.c_double
            f.argtypes = [ctypes.c_void_p, ctypes.c_int]
            getattr(L, P + "get_field").argtypes = [ctypes.c_void_p, ctypes.c_int, fp]
            getattr(L, P + "dump_field").argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, fp]
            getattr(L, P + "free_sim").argtypes = [ctypes.c_void_p]
        _LIB = L
    return _LIB


def _fptr(a):
    if a is None:
        return None
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def solve_simple_math(expr) -> float:
    """utils::solveSimpleMathExpression (src/utils.h:29-43): products of floats only."""
    s = str(expr)
    if any(ch not in "0123456789.* " for ch in s):
        raise ValueError(f"Unsupported math expression {s}")
    r = 1.0
    for item in s.split("*"):
        r *= float(np.float32(float(item)))
    return r


def read_series(path: str, tcol: int, dcol: int):
    """TimeSeries::fromCsv (src/timeseries.cpp:28-84): header skipped, `;` separated, time in
    float seconds or %d.%m.%Y %H:%M:%S relative to the first stamp; first entry wins on equal
    times (std::map::emplace)."""
    series = {}
    first = None
    with open(path, newline="") as f:
        lines = f.read().split("\n")
    if lines and lines[-1] == "":
        lines = lines[:-1]
    for line in lines[1:]:
        cols = line.split(";")
        tv = cols[tcol]
        try:
            if tv != tv.strip():
                raise ValueError
            t = float(np.float32(float(tv)))
        except ValueError:
            st = _time.strptime(tv, "%d.%m.%Y %H:%M:%S")
            ts = int(_time.mktime(st))
            if first is None:
                first = ts
            t = float(np.float32(ts - first))
        d = float(np.float32(float(cols[dcol].strip().split()[0])))
        t32 = float(np.float32(t))
        if t32 not in series:
            series[t32] = d
    keys = sorted(series)
    return np.array(keys, np.float32), np.array([series[k] for k in keys], np.float32)


class Oracle:
    """One CPU simulation (FP64 by default, precision=32 for the IEEE FP32 build)."""

    def __init__(self, W, H, pitch_elems, dx, dt, variable_dt, kst_fixed, no_value, terrain,
                 h0=None, qx0=None, qy0=None, kst_var=None, precision=64):
        self.L = lib()
        self.P = "ora64_" if precision == 64 else "ora32_"
        self.W, self.H = W, H
        self._keep = [np.ascontiguousarray(a, np.float32) if a is not None else None
                      for a in (terrain, h0, qx0, qy0, kst_var)]
        t, h, qx, qy, k = self._keep
        self.terrain = t
        self.s = getattr(self.L, self.P + "new_sim")(W, H, pitch_elems, dx, dt, int(variable_dt), kst_fixed,
                                                     no_value, _fptr(t), _fptr(h), _fptr(qx), _fptr(qy), _fptr(k))
        if not self.s:
            raise ValueError("oracle rejected the grid (W and H must be >= 4)")

    def _f(self, name):
        return getattr(self.L, self.P + name)

    def add_bc(self, side, type_, frm, to, is_series=False, z=0.0, q=0.0, zs=None, qs=None):
        zt, zv = zs if zs is not None else (np.zeros(0, np.float32), np.zeros(0, np.float32))
        qt, qv = qs if qs is not None else (np.zeros(0, np.float32), np.zeros(0, np.float32))
        self._keep += [zt, zv, qt, qv]
        rc = self._f("add_bc")(self.s, SIDES[side], TYPES[type_], frm, to, int(is_series), z, q, len(zt),
                               _fptr(zt), _fptr(zv), len(qt), _fptr(qt), _fptr(qv))
        if rc != 0:
            raise ValueError(f"oracle rejected boundary condition ({rc})")

    def set_sampling(self, interval, points):
        n = len(points)
        arr = lambda k: (ctypes.c_int * max(n, 1))(*[p[k] for p in points])
        self._f("set_sampling")(self.s, int(interval), n, arr(0), arr(1), arr(2))

    def set_save_times(self, times):
        a = (ctypes.c_double * max(len(times), 1))(*times)
        self._f("set_save_times")(self.s, len(times), a)

    def set_threads(self, n):
        self._f("set_threads")(self.s, int(n))

    def simulate(self, n):
        return self._f("simulate")(self.s, int(n))

    def run_to(self, t):
        return self._f("run_to")(self.s, float(t))

    @property
    def duration(self):
        return self._f("duration")(self.s)

    @property
    def dt(self):
        return self._f("dt")(self.s)

    @property
    def iteration(self):
        return self._f("iteration")(self.s)

    @property
    def last_cfl(self):
        return self._f("last_cfl")(self.s)

    def volume(self):
        return self._f("volume")(self.s)

    def field(self, which):
        out = np.empty((self.H, self.W), np.float32)
        self._f("get_field")(self.s, which, _fptr(out))
        return out

    def sample_text(self):
        return self._f("sample_text")(self.s).decode()

    def dumps(self):
        res = []
        for k in range(self._f("dump_count")(self.s)):
            fs = []
            for w in range(4):
                out = np.empty((self.H, self.W), np.float32)
                self._f("dump_field")(self.s, k, w, _fptr(out))
                fs.append(out)
            res.append((self._f("dump_duration")(self.s, k), fs))
        return res

    def __del__(self):
        try:
            if getattr(self, "s", None):
                self._f("free_sim")(self.s)
                self.s = None
        except Exception:
            pass

    @classmethod
    def from_yaml(cls, path, pitch_elems, precision=64):
        """Restates SimData::loadSimData (src/simdata.cpp:238-310) for the oracle."""
        import yaml

        with open(path) as f:
            cfg = yaml.safe_load(f)
        W, H = int(cfg["W"]), int(cfg["H"])
        n = W * H

        def load(key):
            p, off = cfg[key][0], int(cfg[key][1])
            a = np.fromfile(p, dtype=np.float32, count=n, offset=off)
            if a.size != n:
                raise ValueError(f"short file {p}")
            return a.reshape(H, W)

        terr = load("terrain")
        h0 = (load("z") - terr).astype(np.float32) if "z" in cfg else None
        qx0 = load("qx") if "qx" in cfg else None
        qy0 = load("qy") if "qy" in cfg else None
        kst = load("kSt_var") if "kSt_var" in cfg else None
        vdt = cfg.get("variable_dt", True)
        o = cls(W, H, pitch_elems, float(cfg["dx"]), float(cfg["dt"]), bool(vdt),
                float(cfg.get("kSt", 30.0)), float(cfg.get("no_data", -9999.0)), terr, h0, qx0, qy0, kst,
                precision=precision)
        for bc in cfg.get("boundary_conditions") or []:
            side, typ = bc["side"], bc["type"]
            frm = int(bc.get("from", 0))
            to = int(bc.get("to", H - 1 if side in ("left", "right") else W - 1))
            is_series = isinstance(bc.get("q"), list) or isinstance(bc.get("z"), list)
            if is_series:
                zs = read_series(bc["z"][0], int(bc["z"][1]), int(bc["z"][2])) if "z" in bc else None
                qs = read_series(bc["q"][0], int(bc["q"][1]), int(bc["q"][2])) if "q" in bc else None
                o.add_bc(side, typ, frm, to, True, zs=zs, qs=qs)
            else:
                o.add_bc(side, typ, frm, to, False, z=float(bc.get("z", 0.0)), q=float(bc.get("q", 0.0)))
        if "sampling_interval" in cfg:
            pts = [(int(p["x"]), int(p["y"]), SAMPLE_TYPES[p["type"]]) for p in cfg["sampling"]]
            o.labels = [str(p["label"]) for p in cfg["sampling"]]
            o.set_sampling(int(cfg["sampling_interval"]), pts)
        if "save_state" in cfg:
            o.set_save_times([solve_simple_math(s) for s in cfg["save_state"]])
        o.target_duration = solve_simple_math(cfg["duration"])
        o.cfg = cfg
        return o
