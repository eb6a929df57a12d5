"""fip_b200: B200-native (sm_100a) slim shallow-water solver with fip's parameter files and outputs.

The product is the C ABI of include/fip.h (libfip_b200.so, built in-tree) and the `fip` command
line next to it; this package is a thin Python view of the same calls:

    from fip_b200 import Simulation
    with Simulation("scenario.yml") as sim:     # fip_init
        sim.step(100)                           # 100 x simulate()
        h = sim.field("h")                      # fip_get_field
        sim.run()                               # until target_duration, with dumps
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import _lib
from ._lib import FIELDS, FipError, FipInfo, FipOptions, bc_program, config_json, validate

__all__ = ["Simulation", "FipError", "validate", "config_json", "bc_program", "FIELDS"]


class Simulation:
    """One scenario on one GPU (a fip_handle)."""

    def __init__(self, yaml_path: str, device: int = 0, use_graphs: bool = True, all_tiles: bool = False,
                 stop_on_nonfinite: bool = False, quiet: bool = False, sample_path: str | None = None):
        L = _lib.lib()
        opt = FipOptions()
        L.fip_default_options(ctypes.byref(opt))
        opt.device = device
        opt.use_graphs = int(use_graphs)
        opt.all_tiles = int(all_tiles)
        opt.stop_on_nonfinite = int(stop_on_nonfinite)
        opt.quiet = int(quiet)
        self._sample_path = sample_path.encode() if sample_path else None
        opt.sample_path = self._sample_path
        h = ctypes.c_void_p()
        _lib.check(L.fip_init_ex(os.fspath(yaml_path).encode(), ctypes.byref(opt), ctypes.byref(h)))
        self._h = h
        inf = self.info()
        self.W, self.H, self.pitch = inf.W, inf.H, inf.pitch

    # -- simulation loop -------------------------------------------------------------------
    def step(self, n: int = 1) -> None:
        _lib.check(_lib.lib().fip_step(self._h, int(n)))

    def run(self) -> None:
        _lib.check(_lib.lib().fip_run(self._h))

    def save(self, prefix: str | None = None, current: bool = False) -> None:
        f = _lib.lib().fip_save_current if current else _lib.lib().fip_save
        _lib.check(f(self._h, prefix.encode() if prefix else None))

    def sample(self) -> None:
        _lib.check(_lib.lib().fip_sample(self._h))

    # -- state -----------------------------------------------------------------------------
    def field(self, name: str = "h", out: np.ndarray | None = None) -> np.ndarray:
        if out is None:
            out = np.empty((self.H, self.W), np.float32)
        assert out.dtype == np.float32 and out.shape == (self.H, self.W) and out.flags.c_contiguous
        _lib.check(_lib.lib().fip_get_field(self._h, FIELDS[name], out.ctypes.data_as(ctypes.POINTER(ctypes.c_float))))
        return out

    def set_field(self, name: str, values: np.ndarray) -> None:
        a = np.ascontiguousarray(values, dtype=np.float32)
        assert a.shape == (self.H, self.W)
        _lib.check(_lib.lib().fip_set_field(self._h, FIELDS[name], a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))))

    def volume(self) -> float:
        v = ctypes.c_double()
        _lib.check(_lib.lib().fip_volume(self._h, ctypes.byref(v)))
        return v.value

    def time(self):
        d, dt, it = ctypes.c_double(), ctypes.c_float(), ctypes.c_int()
        _lib.check(_lib.lib().fip_time(self._h, ctypes.byref(d), ctypes.byref(dt), ctypes.byref(it)))
        return d.value, dt.value, it.value

    @property
    def duration(self) -> float:
        return self.time()[0]

    @property
    def iteration(self) -> int:
        return self.time()[2]

    def info(self) -> FipInfo:
        inf = FipInfo()
        _lib.check(_lib.lib().fip_info(self._h, ctypes.byref(inf)))
        return inf

    def profile(self, n: int):
        """Average device ms per launch of (stencil, post) over n eager steps (advances the state)."""
        a, b = ctypes.c_float(), ctypes.c_float()
        _lib.check(_lib.lib().fip_profile_steps(self._h, int(n), ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def step_timed(self, n: int):
        """n steps in one graph, timed on the device: (total ms, stencil ms/launch, post ms/launch)."""
        t, a, b = ctypes.c_float(), ctypes.c_float(), ctypes.c_float()
        _lib.check(_lib.lib().fip_step_timed(self._h, int(n), ctypes.byref(t), ctypes.byref(a), ctypes.byref(b)))
        return t.value, a.value, b.value

    # -- lifetime --------------------------------------------------------------------------
    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            _lib.lib().fip_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
