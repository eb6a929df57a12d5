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
from ._lib import FIELDS, EnsembleInfo, EnsembleTune, FipError, FipInfo, FipOptions, bc_program, config_json, validate

__all__ = ["Simulation", "Ensemble", "FipError", "validate", "config_json", "bc_program", "FIELDS"]


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

    # -- pipelined state exchange ----------------------------------------------------------
    def stage_state(self, h: np.ndarray, qx: np.ndarray, qy: np.ndarray) -> None:
        """Queues the upload of a whole state (fip_stage_state); the arrays are kept alive until
        the step_exchange that takes them returns."""
        arrs = []
        for a in (h, qx, qy):
            assert a.dtype == np.float32 and a.shape == (self.H, self.W) and a.flags.c_contiguous
            arrs.append(a)
        fp = ctypes.POINTER(ctypes.c_float)
        _lib.check(_lib.lib().fip_stage_state(self._h, *(a.ctypes.data_as(fp) for a in arrs)))
        self._staged = getattr(self, "_staged", []) + [arrs]

    def step_exchange(self, n: int, out=None) -> None:
        """Takes the oldest staged state, runs n steps and queues the download of the state into
        `out` = (h, qx, qy) arrays (complete after the next call or exchange_wait)."""
        fp = ctypes.POINTER(ctypes.c_float)
        if out is None:
            ptrs = (None, None, None)
        else:
            for a in out:
                assert a.dtype == np.float32 and a.shape == (self.H, self.W) and a.flags.c_contiguous
            ptrs = tuple(a.ctypes.data_as(fp) for a in out)
        _lib.check(_lib.lib().fip_step_exchange(self._h, int(n), *ptrs))
        staged = getattr(self, "_staged", [])
        if staged:
            staged.pop(0)
        self._pending = getattr(self, "_pending", [])[-1:] + ([out] if out is not None else [])

    def exchange_wait(self) -> None:
        _lib.check(_lib.lib().fip_exchange_wait(self._h))
        self._pending = []

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
        """n steps in one graph, timed on the device: total ms; then n more steps with an event
        around every launch: stencil and post ms per launch. Returns the three."""
        t, a, b = ctypes.c_float(), ctypes.c_float(), ctypes.c_float()
        _lib.check(_lib.lib().fip_step_timed(self._h, int(n), ctypes.byref(t), ctypes.byref(a), ctypes.byref(b)))
        return t.value, a.value, b.value

    # -- headless colour map ----------------------------------------------------------------
    def render(self, what: str = "depth", vmax: float = 0.0, png_path: str | None = None) -> np.ndarray:
        """RGBA8 image (H, W, 4), row 0 = northern edge; optionally also written as a PNG."""
        img = np.empty((self.H, self.W, 4), np.uint8)
        _lib.check(_lib.lib().fip_render(self._h, _lib.RENDER[what], float(vmax), img.ctypes.data_as(ctypes.c_void_p),
                                         os.fspath(png_path).encode() if png_path else None))
        return img

    def inject_wait_timeout(self) -> None:
        """Test hook: the next step's bounded device waits run out (FIP_ERR_DEVICE_TIMEOUT)."""
        _lib.check(_lib.lib().fip_inject_wait_timeout(self._h))

    # -- exact resume ----------------------------------------------------------------------
    def checkpoint(self, path: str) -> None:
        """Writes both ping-pong buffers, hmax and the step state; see restore()."""
        _lib.check(_lib.lib().fip_checkpoint(self._h, os.fspath(path).encode()))

    def restore(self, path: str) -> None:
        """Loads a checkpoint of the same scenario; the run continues bit for bit."""
        _lib.check(_lib.lib().fip_restore(self._h, os.fspath(path).encode()))

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


class Ensemble:
    """Many scenarios stepped together on one GPU (a fip_ensemble): one stencil launch and one
    post-kernel launch per ensemble step over every member still short of its target duration.
    Each member computes what a Simulation of its own parameter file computes."""

    def __init__(self, yaml_paths, device: int = 0, use_graphs: bool = True, all_tiles: bool = False,
                 stop_on_nonfinite: bool = False):
        L = _lib.lib()
        opt = FipOptions()
        L.fip_default_options(ctypes.byref(opt))
        opt.device = device
        opt.use_graphs = int(use_graphs)
        opt.all_tiles = int(all_tiles)
        opt.stop_on_nonfinite = int(stop_on_nonfinite)
        opt.quiet = 1
        paths = [os.fspath(p).encode() for p in yaml_paths]
        arr = (ctypes.c_char_p * len(paths))(*paths)
        h = ctypes.c_void_p()
        _lib.check(L.fip_ensemble_init(arr, len(paths), ctypes.byref(opt), ctypes.byref(h)))
        self._h = h
        self.n = len(paths)
        self.shapes = []
        for m in range(self.n):
            cfg = config_json(os.fspath(yaml_paths[m]))
            self.shapes.append((int(cfg["H"]), int(cfg["W"])))

    def step(self, n: int = 1) -> None:
        _lib.check(_lib.lib().fip_ensemble_step(self._h, int(n)))

    def run(self) -> None:
        _lib.check(_lib.lib().fip_ensemble_run(self._h))

    def step_timed(self, n: int) -> float:
        """n ensemble steps timed on the device: total ms."""
        t = ctypes.c_float()
        _lib.check(_lib.lib().fip_ensemble_step_timed(self._h, int(n), ctypes.byref(t)))
        return t.value

    def autotune(self, steps_per_shape: int = 20):
        """Times real steps in each tile shape and keeps the fastest: list of dicts per shape."""
        res = (EnsembleTune * 16)()
        n = ctypes.c_int()
        _lib.check(_lib.lib().fip_ensemble_autotune(self._h, int(steps_per_shape), res, 16, ctypes.byref(n)))
        return [{"consumer_warps": r.consumer_warps, "cols_per_thread": r.cols_per_thread, "tile_cols": r.tile_cols,
                 "tile_rows": r.tile_rows, "steps": r.steps, "ms_per_step": r.ms_per_step} for r in res[:n.value]]

    def set_shape(self, consumer_warps: int, tile_rows: int, cols_per_thread: int = 4) -> None:
        _lib.check(_lib.lib().fip_ensemble_set_shape_nc(self._h, int(consumer_warps), int(tile_rows),
                                                         int(cols_per_thread)))

    def field(self, member: int, name: str = "h") -> np.ndarray:
        H, W = self.shapes[member]
        out = np.empty((H, W), np.float32)
        _lib.check(_lib.lib().fip_ensemble_get_field(self._h, int(member), FIELDS[name],
                                                     out.ctypes.data_as(ctypes.POINTER(ctypes.c_float))))
        return out

    def render(self, member: int, what: str = "hmax", vmax: float = 0.0, png_path: str | None = None) -> np.ndarray:
        H, W = self.shapes[member]
        img = np.empty((H, W, 4), np.uint8)
        _lib.check(_lib.lib().fip_ensemble_render(self._h, int(member), _lib.RENDER[what], float(vmax),
                                                  img.ctypes.data_as(ctypes.c_void_p),
                                                  os.fspath(png_path).encode() if png_path else None))
        return img

    def gather(self, name: str, out) -> None:
        """Every member's field, one grid after the other, into device memory `out` (a CUDA
        tensor or device pointer of sum(W * H) floats)."""
        ptr = out if isinstance(out, int) else out.data_ptr()
        _lib.check(_lib.lib().fip_ensemble_gather(self._h, FIELDS[name], ctypes.c_void_p(ptr)))

    def time(self, member: int):
        d, dt, it = ctypes.c_double(), ctypes.c_float(), ctypes.c_int()
        _lib.check(_lib.lib().fip_ensemble_time(self._h, int(member), ctypes.byref(d), ctypes.byref(dt),
                                                ctypes.byref(it)))
        return d.value, dt.value, it.value

    def info(self) -> EnsembleInfo:
        inf = EnsembleInfo()
        _lib.check(_lib.lib().fip_ensemble_info(self._h, ctypes.byref(inf)))
        return inf

    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            _lib.lib().fip_ensemble_destroy(self._h)
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
