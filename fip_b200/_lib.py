"""ctypes binding of libfip_b200.so (the C ABI in include/fip.h).

The shared library is built in-tree (fip_b200/libfip_b200.so) by ``make -C fip_b200/csrc`` or
``__graft_entry__.build()``. There is no fallback: importing the binding without the library
raises, and every simulation call runs the sm_100a kernels.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libfip_b200.so")

FIP_OK = 0
FIP_ERR_CONFIG = -1
FIP_ERR_IO = -2
FIP_ERR_CUDA = -3
FIP_ERR_NVRTC = -4
FIP_ERR_NONFINITE = -5
FIP_ERR_DEVICE_TIMEOUT = -6
FIP_ERR_ARG = -7

RENDER = {"depth": 0, "velocity": 1, "hmax": 2}

FIELDS = {"h": 0, "qx": 1, "qy": 2, "hmax": 3, "h_prev": 4, "qx_prev": 5, "qy_prev": 6, "terrain": 7, "z": 8}

# every symbol include/fip.h declares
EXPORTS = ("fip_default_options", "fip_init", "fip_init_ex", "fip_step", "fip_run", "fip_save", "fip_save_current",
           "fip_sample", "fip_volume", "fip_get_field", "fip_set_field", "fip_time", "fip_info", "fip_profile_steps", "fip_step_timed", "fip_destroy", "fip_rmg_step_noalloc",
           "fip_last_error", "fip_validate", "fip_config_json", "fip_bc_program",
           "fip_ensemble_init", "fip_ensemble_step", "fip_ensemble_run", "fip_ensemble_autotune", "fip_ensemble_set_shape",
           "fip_ensemble_set_shape_nc",
           "fip_ensemble_step_timed", "fip_ensemble_get_field", "fip_ensemble_time", "fip_ensemble_info",
           "fip_ensemble_destroy", "fip_checkpoint", "fip_restore", "fip_render", "fip_ensemble_render",
           "fip_sg_conv3x3", "fip_sg_conv3x3_wgrad", "fip_ensemble_gather", "fip_sg_pack_input", "fip_sg_target",
           "fip_sg_loss", "fip_sg_bias_grad", "fip_sg_adamw", "fip_sg_cast_weights", "fip_sg_apply",
           "fip_sg_edge_flux", "fip_sg_consistency", "fip_sg_level_bound", "fip_sg_pin", "fip_sg_edges", "fip_inject_wait_timeout",
           "fip_stage_state",
           "fip_step_exchange", "fip_exchange_wait")


class FipOptions(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("use_graphs", ctypes.c_int), ("all_tiles", ctypes.c_int),
                ("stop_on_nonfinite", ctypes.c_int), ("quiet", ctypes.c_int), ("sample_path", ctypes.c_char_p)]


class FipInfo(ctypes.Structure):
    _fields_ = [("W", ctypes.c_int), ("H", ctypes.c_int), ("pitch", ctypes.c_int), ("n_tiles", ctypes.c_int),
                ("active_tiles", ctypes.c_int), ("iteration", ctypes.c_int), ("duration", ctypes.c_double),
                ("dt", ctypes.c_float), ("last_cfl", ctypes.c_float), ("nonfinite", ctypes.c_int)]


class EnsembleTune(ctypes.Structure):
    _fields_ = [("consumer_warps", ctypes.c_int), ("tile_cols", ctypes.c_int), ("tile_rows", ctypes.c_int),
                ("steps", ctypes.c_int), ("ms_per_step", ctypes.c_float), ("cols_per_thread", ctypes.c_int)]


class EnsembleInfo(ctypes.Structure):
    _fields_ = [("n_members", ctypes.c_int), ("active_members", ctypes.c_int), ("cells", ctypes.c_longlong),
                ("packed_W", ctypes.c_int), ("packed_rows", ctypes.c_int), ("pitch", ctypes.c_int),
                ("consumer_warps", ctypes.c_int), ("tile_cols", ctypes.c_int), ("tile_rows", ctypes.c_int),
                ("n_tiles", ctypes.c_int), ("active_tiles", ctypes.c_int), ("iteration", ctypes.c_int),
                ("nonfinite", ctypes.c_int), ("cols_per_thread", ctypes.c_int)]


class FipError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"fip error {code}: {msg}")
        self.code = code


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `make -C fip_b200/csrc` "
                              "(or __graft_entry__.build()); there is no CPU fallback")
        L = ctypes.CDLL(LIB_PATH)
        vp, ip = ctypes.c_void_p, ctypes.c_int
        fp = ctypes.POINTER(ctypes.c_float)
        L.fip_default_options.argtypes = [ctypes.POINTER(FipOptions)]
        L.fip_default_options.restype = None
        L.fip_init.argtypes = [ctypes.c_char_p, ctypes.POINTER(vp)]
        L.fip_init_ex.argtypes = [ctypes.c_char_p, ctypes.POINTER(FipOptions), ctypes.POINTER(vp)]
        L.fip_step.argtypes = [vp, ip]
        L.fip_run.argtypes = [vp]
        L.fip_save.argtypes = [vp, ctypes.c_char_p]
        L.fip_save_current.argtypes = [vp, ctypes.c_char_p]
        L.fip_sample.argtypes = [vp]
        L.fip_volume.argtypes = [vp, ctypes.POINTER(ctypes.c_double)]
        L.fip_get_field.argtypes = [vp, ip, fp]
        L.fip_set_field.argtypes = [vp, ip, fp]
        L.fip_stage_state.argtypes = [vp, fp, fp, fp]
        L.fip_step_exchange.argtypes = [vp, ip, fp, fp, fp]
        L.fip_exchange_wait.argtypes = [vp]
        L.fip_time.argtypes = [vp, ctypes.POINTER(ctypes.c_double), fp, ctypes.POINTER(ctypes.c_int)]
        L.fip_info.argtypes = [vp, ctypes.POINTER(FipInfo)]
        L.fip_profile_steps.argtypes = [vp, ip, fp, fp]
        L.fip_step_timed.argtypes = [vp, ip, fp, fp, fp]
        L.fip_rmg_step_noalloc.argtypes = [vp, vp, vp, vp, vp, ctypes.c_float, vp, vp, vp, ip, ip, ip, ctypes.c_float,
                                           ctypes.c_float, ctypes.c_float, vp, vp]
        L.fip_rmg_step_noalloc.restype = ctypes.c_int
        L.fip_ensemble_init.argtypes = [ctypes.POINTER(ctypes.c_char_p), ip, ctypes.POINTER(FipOptions),
                                        ctypes.POINTER(vp)]
        L.fip_ensemble_step.argtypes = [vp, ip]
        L.fip_ensemble_run.argtypes = [vp]
        L.fip_ensemble_autotune.argtypes = [vp, ip, ctypes.POINTER(EnsembleTune), ip, ctypes.POINTER(ctypes.c_int)]
        L.fip_ensemble_set_shape.argtypes = [vp, ip, ip]
        L.fip_ensemble_set_shape_nc.argtypes = [vp, ip, ip, ip]
        L.fip_ensemble_step_timed.argtypes = [vp, ip, fp]
        L.fip_ensemble_get_field.argtypes = [vp, ip, ip, fp]
        L.fip_ensemble_time.argtypes = [vp, ip, ctypes.POINTER(ctypes.c_double), fp, ctypes.POINTER(ctypes.c_int)]
        L.fip_ensemble_info.argtypes = [vp, ctypes.POINTER(EnsembleInfo)]
        L.fip_ensemble_destroy.argtypes = [vp]
        L.fip_ensemble_destroy.restype = None
        L.fip_render.argtypes = [vp, ip, ctypes.c_float, vp, ctypes.c_char_p]
        L.fip_render.restype = ctypes.c_int
        L.fip_ensemble_render.argtypes = [vp, ip, ip, ctypes.c_float, vp, ctypes.c_char_p]
        L.fip_ensemble_render.restype = ctypes.c_int
        L.fip_ensemble_gather.argtypes = [vp, ip, vp]
        f32, ll = ctypes.c_float, ctypes.c_longlong
        L.fip_sg_conv3x3.argtypes = [vp, vp, vp, vp, vp, vp, ip, ip, ip, ip, ip, vp, vp]
        L.fip_sg_conv3x3_wgrad.argtypes = [vp, vp, vp, ip, ip, ip, ip, vp, vp]
        L.fip_sg_pack_input.argtypes = [vp, vp, vp, vp, vp, vp, ip, ip, ip, f32, vp, vp]
        L.fip_sg_target.argtypes = [vp, vp, vp, vp, vp, vp, vp, ll, f32, vp, vp]
        L.fip_sg_loss.argtypes = [vp, vp, ip, ip, ip, f32, vp, vp, vp, vp]
        L.fip_sg_bias_grad.argtypes = [vp, ll, vp, vp]
        L.fip_sg_adamw.argtypes = [vp, vp, vp, vp, ll, f32, f32, f32, f32, f32, ip, vp]
        L.fip_sg_cast_weights.argtypes = [vp, ip, vp, vp, vp]
        L.fip_sg_apply.argtypes = [vp, ip, ip, ip, f32, vp, f32, vp, vp, vp, vp, vp, vp]
        L.fip_sg_edge_flux.argtypes = [vp, vp, ip, ip, ip, vp, vp]
        L.fip_sg_consistency.argtypes = [vp, ip, ip, ip, f32, vp, f32, vp, vp, vp, vp]
        L.fip_sg_level_bound.argtypes = [vp, vp, vp, vp, vp, ip, ip, ip, f32, ip, f32, vp, vp, vp]
        L.fip_sg_pin.argtypes = [vp, vp, vp, vp, ll, vp, vp, vp, vp]
        L.fip_sg_pin.restype = ctypes.c_int
        L.fip_sg_edges.argtypes = [vp, vp, ip, ip, ip, ip, ip, ip, ip, f32, vp]
        L.fip_sg_edges.restype = ctypes.c_int
        for name in ("fip_ensemble_gather", "fip_sg_conv3x3", "fip_sg_conv3x3_wgrad", "fip_sg_pack_input",
                     "fip_sg_target", "fip_sg_loss", "fip_sg_bias_grad", "fip_sg_adamw", "fip_sg_cast_weights",
                     "fip_sg_apply", "fip_sg_edge_flux", "fip_sg_consistency", "fip_sg_level_bound"):
            getattr(L, name).restype = ctypes.c_int
        L.fip_inject_wait_timeout.argtypes = [vp]
        L.fip_inject_wait_timeout.restype = ctypes.c_int
        L.fip_checkpoint.argtypes = [vp, ctypes.c_char_p]
        L.fip_restore.argtypes = [vp, ctypes.c_char_p]
        L.fip_checkpoint.restype = ctypes.c_int
        L.fip_restore.restype = ctypes.c_int
        L.fip_destroy.argtypes = [vp]
        L.fip_destroy.restype = None
        L.fip_last_error.restype = ctypes.c_char_p
        L.fip_validate.argtypes = [ctypes.c_char_p]
        L.fip_config_json.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ip]
        L.fip_bc_program.argtypes = [ctypes.c_char_p, ip, ip, ctypes.c_char_p, ip]
        for name in ("fip_init", "fip_init_ex", "fip_step", "fip_run", "fip_save", "fip_save_current", "fip_sample",
                     "fip_volume", "fip_get_field", "fip_set_field", "fip_time", "fip_info", "fip_profile_steps", "fip_step_timed", "fip_validate",
                     "fip_config_json", "fip_bc_program", "fip_ensemble_init", "fip_ensemble_step", "fip_ensemble_run",
                     "fip_ensemble_autotune", "fip_ensemble_set_shape", "fip_ensemble_set_shape_nc",
                     "fip_ensemble_step_timed",
                     "fip_ensemble_get_field", "fip_ensemble_time", "fip_ensemble_info"):
            getattr(L, name).restype = ctypes.c_int
        _lib = L
    return _lib


def last_error() -> str:
    return lib().fip_last_error().decode(errors="replace")


def check(rc: int) -> int:
    if rc < 0:
        raise FipError(rc, last_error())
    return rc


def validate(yaml_path: str) -> None:
    check(lib().fip_validate(yaml_path.encode()))


def config_json(yaml_path: str) -> dict:
    import json

    n = check(lib().fip_config_json(yaml_path.encode(), None, 0))
    buf = ctypes.create_string_buffer(n + 1)
    check(lib().fip_config_json(yaml_path.encode(), buf, n + 1))
    return json.loads(buf.value.decode())


def bc_program(yaml_path: str, pitch: int, compile: bool = False) -> str:
    n = check(lib().fip_bc_program(yaml_path.encode(), pitch, int(compile), None, 0))
    buf = ctypes.create_string_buffer(n + 1)
    check(lib().fip_bc_program(yaml_path.encode(), pitch, 0, buf, n + 1))
    return buf.value.decode()
