"""Host-side logic of libfip_b200.so, run without a GPU: the C ABI loads and exports every entry
point include/fip.h declares, parameter files are validated and parsed like the reference's
loader (src/simdata.cpp:152-310), time series (seconds or %d.%m.%Y %H:%M:%S stamps,
src/timeseries.cpp:28-84) are read like the reference, and the boundary-condition program is
generated and compiled by NVRTC for sm_100a. No call here touches a GPU."""
import ctypes
import os
import re

import numpy as np
import pytest

import pyoracle
from fip_b200 import FipError, _lib, bc_program, config_json, synth, validate

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = []
    for hdr in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if hdr.endswith(".h"):
            with open(os.path.join(ROOT, "include", hdr)) as f:
                text = re.sub(r"/\*.*?\*/", "", f.read(), flags=re.S)
            names += re.findall(r"^[A-Za-z_][\w \*]*?\b(fip_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    names = _declared()
    assert "fip_init" in names and "fip_rmg_step_noalloc" in names and "fip_ensemble_init" in names
    L = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    assert sorted(_lib.EXPORTS) == names


def test_validate_and_parse(tmp_path):
    sc = synth.scenario1(str(tmp_path), W=64, H=48, seed=2, duration=600.0, name="v")
    validate(sc.yaml_path)
    cfg = config_json(sc.yaml_path)
    assert (cfg["W"], cfg["H"], cfg["dx"]) == (64, 48, 3.0)
    assert cfg["variable_dt"] and cfg["kst_var"] and cfg["no_data"] == -1.0
    assert [b["type"] for b in cfg["boundary_conditions"]] == ["q", "open"]
    bad = tmp_path / "bad.yml"
    bad.write_text(open(sc.yaml_path).read().replace("W: 64", "W: 65"))
    with pytest.raises(FipError):  # the terrain file is one row short for W = 65
        validate(str(bad))


def test_validation_messages_follow_the_reference(tmp_path):
    """Every check of validateSimDataConfig (src/simdata.cpp:152-236), reported on stderr as the
    reference reports it (1-based line of the offending node, the root map for missing keys),
    all of them before the load fails."""
    import subprocess
    import sys

    y = tmp_path / "v.yml"
    y.write_text("name: x\n"                           # 1
                 "terrain: [t.bin]\n"                  # 2: path without its byte offset
                 "W: 8\n"                              # 3  (H missing)
                 "dt: 0.1\n"
                 "dx: 2\n"
                 "duration: 10\n"
                 "kSt: 30\n"
                 "kSt_var: [k.bin, 0]\n"               # 8: both kSt_var and kSt
                 "boundary_conditions:\n"
                 "  - side: left\n"                    # 10: q without its q value
                 "    type: q\n"
                 "    z: [a.csv, 0]\n"                 # 12: series without its data column
                 "  - type: z\n"                       # 13: side and z missing
                 "sampling_interval: 5\n")             # no sampling points
    code = ("import sys; sys.path.insert(0, %r)\n"
            "from fip_b200 import validate, FipError\n"
            "try:\n    validate(%r)\nexcept FipError as e:\n    print(e.code)\n") % (ROOT, str(y))
    p = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=120)
    assert p.stdout.strip() == str(_lib.FIP_ERR_CONFIG), (p.stdout, p.stderr)
    got = [ln for ln in p.stderr.splitlines() if ln.strip()]
    assert got == [
        'Config error at line 1: "H" missing',
        'Config error at line 8: Both "kSt_var" and "kSt" defined',
        'Config error at line 2: file path "terrain" needs format [path, byte_offset]',
        'Config error at line 10: "q" missing',
        'Config error at line 12: timeseries "z" needs format [csv_filename, int_time_column, int_data_column]',
        'Config error at line 13: "side" missing',
        'Config error at line 13: "z" missing',
        "Configuration error: sampling interval specified but no sampling points given",
        "Warning: no save_state times given",
    ], got


def test_documented_parameter_forms(tmp_path):
    """Every form of the reference's parameter table (README.md:46-64): [path, byte offset]
    grids, a duration and save_state times as products, block and flow-style sampling points, a
    time-series condition over the whole side and a closed range of another side."""
    synth.write_grid(str(tmp_path / "t.bin"), np.zeros((12, 10), np.float32), offset=36)
    (tmp_path / "s.csv").write_text("t;z\n0;1.5\n3600;2.5\n")
    y = tmp_path / "p.yml"
    y.write_text(f"name: p\nterrain: [{tmp_path}/t.bin, 36]\nW: 10\nH: 12\ndx: 3\ndt: 0.1\n"
                 "duration: 3600*24*12\nkSt: 30.0\nvariable_dt: true\nno_data: -1\n"
                 "save_state:\n  - 3600 * 24 * 0.5\n  - 3600 * 24 * 2.5\n"
                 "sampling:\n  - x: 0\n    y: 7\n    label: sample1\n    type: z\n"
                 "  - { x: 4, y: 7, label: sample2, type: qx }\n"
                 "sampling_interval: 100\n"
                 f"boundary_conditions:\n  - side: left\n    type: z\n    z: [{tmp_path}/s.csv, 0, 1]\n"
                 "  - side: right\n    type: close\n    from: 0\n    to: 5\n")
    c = config_json(str(y))
    assert c["target_duration"] == 3600 * 24 * 12 and c["save_state"] == [43200, 216000]
    assert c["sampling"] == [{"x": 0, "y": 7, "label": "sample1", "type": "z"},
                             {"x": 4, "y": 7, "label": "sample2", "type": "qx"}]
    assert c["sampling_interval"] == 100 and c["variable_dt"] is True and c["no_data"] == -1 and c["kSt"] == 30
    bcs = [(b["side"], b["type"], b["from"], b["to"]) for b in c["boundary_conditions"]]
    assert bcs == [("left", "z", 0, 11), ("right", "close", 0, 5)]
    assert c["boundary_conditions"][0]["series"] and c["boundary_conditions"][0]["z_v"] == [1.5, 2.5]


def test_defaults_follow_the_reference(tmp_path):
    """variable_dt defaults to true, kSt to 30, no_data to -9999 (src/simdata.cpp:245-254)."""
    terr = np.zeros((8, 8), np.float32)
    synth.write_grid(str(tmp_path / "t.bin"), terr)
    y = tmp_path / "d.yml"
    y.write_text(f"name: {tmp_path}/d\nterrain: [{tmp_path}/t.bin, 0]\nW: 8\nH: 8\ndx: 2\ndt: 0.1\n"
                 f"duration: 60*2\n")
    cfg = config_json(str(y))
    assert cfg["variable_dt"] is True and cfg["kSt"] == 30.0 and cfg["no_data"] == -9999.0
    assert cfg["target_duration"] == 120.0  # solveSimpleMathExpression: products


def test_gauge_series_with_dates(tmp_path):
    """A real-gauge style record: %d.%m.%Y %H:%M:%S stamps counted from the first row, CRLF
    line ends, a header, 15-minute readings over 40 days; the library and the oracle agree."""
    n = 40 * 96
    t = np.arange(n) * 900.0
    q = 50.0 + 40.0 * np.sin(t / 86400.0 * 2 * np.pi) ** 2
    z = 1.0 + 0.01 * np.sqrt(q)
    qp, zp = tmp_path / "gauge_q.csv", tmp_path / "gauge_z.csv"
    synth.write_series(str(qp), t, q, header="date;discharge", dates=True)
    synth.write_series(str(zp), t, z, header="date;stage", dates=True)
    for p in (qp, zp):
        p.write_bytes(p.read_bytes().replace(b"\n", b"\r\n"))
    terr = np.zeros((16, 16), np.float32)
    synth.write_grid(str(tmp_path / "t.bin"), terr)
    y = tmp_path / "g.yml"
    y.write_text(f"name: {tmp_path}/g\nterrain: [{tmp_path}/t.bin, 0]\nW: 16\nH: 16\ndx: 2\ndt: 0.1\n"
                 f"duration: 100\nvariable_dt: false\nboundary_conditions:\n"
                 f"  - side: left\n    type: q\n    q: [{qp}, 0, 1]\n    z: [{zp}, 0, 1]\n    from: 2\n    to: 12\n")
    cfg = config_json(str(y))
    b = cfg["boundary_conditions"][0]
    assert b["series"] and len(b["q_t"]) == n
    assert np.array_equal(np.float32(b["q_t"]), t.astype(np.float32))
    assert np.array_equal(np.float32(b["q_v"]), q.astype(np.float32))
    ot, ov = pyoracle.read_series(str(zp), 0, 1)
    assert np.array_equal(np.float32(b["z_t"]), np.float32(ot)) and np.array_equal(np.float32(b["z_v"]), np.float32(ov))


def test_boundary_program_compiles_for_sm100a(tmp_path):
    sc = synth.scenario1(str(tmp_path), W=64, H=48, seed=2, duration=600.0, name="p")
    src = bc_program(sc.yaml_path, 128, compile=True)
    assert "fip_post" in src and "fip_interp_block" in src and "fip_sum_depths" in src


def test_surrogate_entry_points_reject_bad_arguments():
    """Argument checks of include/fip_surrogate.h run on the host before any launch."""
    L = _lib.lib()
    vp = ctypes.c_void_p
    assert L.fip_sg_conv3x3(None, None, None, None, None, None, 1, 8, 8, 1, 0, None, None) == _lib.FIP_ERR_ARG
    odd = vp(0x1008)  # not 16-byte aligned (never dereferenced: rejected first)
    al = vp(0x2000)
    assert L.fip_sg_conv3x3(al, al, None, odd, None, al, 1, 8, 8, 1, 1, None, None) == _lib.FIP_ERR_ARG
    assert L.fip_sg_conv3x3(al, al, None, None, None, al, 1, 8, 8, 9, 0, None, None) == _lib.FIP_ERR_ARG  # dilation
    assert L.fip_sg_conv3x3(al, al, None, None, None, al, 1, 8, 8, 1, 7, None, None) == _lib.FIP_ERR_ARG  # epilogue
    assert L.fip_sg_conv3x3(al, al, None, None, None, al, 1, 8, 8, 1, 1, None, None) == _lib.FIP_ERR_ARG  # needs res
    assert L.fip_sg_conv3x3_wgrad(al, al, al, 1, 8, 8, 0, None, None) == _lib.FIP_ERR_ARG
    big = (200, 3300, 3300)  # (3300 + 16)^2 * 200 pixels > 2^31
    assert L.fip_sg_conv3x3(al, al, None, None, None, al, *big, 1, 0, None, None) == _lib.FIP_ERR_ARG
    assert L.fip_sg_conv3x3_wgrad(al, al, al, *big, 1, None, None) == _lib.FIP_ERR_ARG
    assert "too many pixels" in _lib.last_error()
    assert L.fip_sg_edges(al, al, 1, 8, 8, 0, 3, 1, 1, ctypes.c_float(-1.0), None) == _lib.FIP_ERR_ARG
    assert L.fip_sg_adamw(al, al, al, al, 10, ctypes.c_float(1e-3), ctypes.c_float(0.9), ctypes.c_float(0.999),
                          ctypes.c_float(1e-8), ctypes.c_float(0.0), 0, None) == _lib.FIP_ERR_ARG  # step >= 1
