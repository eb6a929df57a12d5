"""The save_state restart route on the CPU (fip_b200.restart): a depth dump (two size_t W, H and
W*H float32, src/main.cpp:154-202) turned into the level file that the `z` key expects
(src/simdata.cpp:266-270) restarts the depths to the rounding of the level; feeding the depth
dump itself as `z` does not. The loader here is the CPU oracle's (src/simdata.cpp:238-285)."""
import numpy as np
import pytest

import pyoracle
from fip_b200 import restart, synth


def _dump(path, a):
    H, W = a.shape
    with open(path, "wb") as f:
        f.write(np.array([W, H], dtype="<u8").tobytes())
        f.write(a.astype("<f4").tobytes())


def _load_depth(tmp_path, terrain_file, z_entry, W, H):
    y = tmp_path / "r.yml"
    synth.write_yaml(str(y), {"name": str(tmp_path / "r"), "terrain": [terrain_file, 0], "z": z_entry, "W": W,
                              "H": H, "dx": 2.0, "dt": 0.1, "duration": 10, "kSt": 30, "variable_dt": False})
    o = pyoracle.Oracle.from_yaml(str(y), 128 * -(-W // 128), precision=32)
    return o.field(pyoracle.F_H)


def test_level_file_restarts_the_dumped_depths(tmp_path):
    W, H = 37, 23
    rng = np.random.default_rng(3)
    terr = (50.0 + 10.0 * rng.random((H, W))).astype(np.float32)
    depth = np.where(rng.random((H, W)) < 0.6, 2.0 * rng.random((H, W)), 0.0).astype(np.float32)
    tfile = str(tmp_path / "terrain.bin")
    synth.write_grid(tfile, terr)
    ah = str(tmp_path / "r_ah_600_2024-01-01-00-00")
    _dump(ah, depth)
    assert np.array_equal(restart.read_dump(ah), depth)
    level = str(tmp_path / "level.bin")
    restart.level_file_from_dump(ah, tfile, 0, level)
    h = _load_depth(tmp_path, tfile, [level, 16], W, H)
    tol = np.spacing((depth + terr).astype(np.float32)).astype(np.float64)
    assert np.all(np.abs(h.astype(np.float64) - depth) <= tol)
    # the dump itself as `z` is read as a level below the terrain: not the dumped state
    wrong = _load_depth(tmp_path, tfile, [ah, 16], W, H)
    assert not np.allclose(wrong, depth, atol=1e-3)


def test_truncated_dump_is_rejected(tmp_path):
    p = str(tmp_path / "cut_ah_0_x")
    with open(p, "wb") as f:
        f.write(np.array([8, 8], dtype="<u8").tobytes())
        f.write(np.zeros(60, "<f4").tobytes())
    with pytest.raises(ValueError):
        restart.read_dump(p)
