"""Restarting from save_state dumps in the reference's own input format.

The reference writes `<name>_ah_<t>_<stamp>`, `_qx_`, `_qy_` dumps as two size_t (W, H) followed
by W*H float32 (src/main.cpp:154-202), and reads restart state from the YAML keys `z`, `qx`, `qy`
as raw float32 at a byte offset (src/simdata.cpp:266-274). The dump holds the water DEPTH while
the `z` key expects the water LEVEL (depth = z - terrain), so feeding the `_ah_` dump back as `z`
restarts from a wrong state. `level_file_from_dump` writes the level file that restarts the
depths (to FP32 rounding of (h + terrain) - terrain; fip_checkpoint/fip_restore resume exactly).
Note that `fip_save`/save_state dumps hold the state before the step that triggered them (the
reference dumps its ping-pong partner buffers); `fip_save_current` dumps the current state.
"""
from __future__ import annotations

import numpy as np


def read_dump(path: str) -> np.ndarray:
    """A save_state dump as an (H, W) float32 array."""
    with open(path, "rb") as f:
        hdr = np.frombuffer(f.read(16), dtype="<u8")
        W, H = int(hdr[0]), int(hdr[1])
        data = np.frombuffer(f.read(W * H * 4), dtype="<f4")
    if data.size != W * H:
        raise ValueError(f"{path}: truncated dump ({data.size} of {W * H} values)")
    return data.reshape(H, W)


def read_grid(path: str, W: int, H: int, offset: int = 0) -> np.ndarray:
    """A raw float32 input grid at a byte offset (utils::loadFileIntoArray)."""
    with open(path, "rb") as f:
        f.seek(offset)
        data = np.frombuffer(f.read(W * H * 4), dtype="<f4")
    if data.size != W * H:
        raise ValueError(f"{path}: short grid file")
    return data.reshape(H, W)


def level_file_from_dump(ah_dump: str, terrain_path: str, terrain_offset: int, out_path: str) -> None:
    """Writes z = depth + terrain behind the same 16-byte (W, H) header as the dump, so that
    `z: [out_path, 16]` in the YAML restarts from the dumped depths."""
    h = read_dump(ah_dump)
    Hh, Ww = h.shape
    terr = read_grid(terrain_path, Ww, Hh, terrain_offset)
    z = (h + terr).astype("<f4")
    with open(out_path, "wb") as f:
        f.write(np.array([Ww, Hh], dtype="<u8").tobytes())
        f.write(z.tobytes())
