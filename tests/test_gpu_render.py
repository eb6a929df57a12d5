"""Headless colour-map export (fip_render / fip_ensemble_render) against the CPU restatement of
the reference's fragment shader (oracle/render_oracle.py, src/shaders.h:57-123): every channel
of every pixel within one 8-bit step; the PNG holds exactly the returned pixels."""
import struct
import zlib

import numpy as np
import pytest

import render_oracle
from fip_b200 import Ensemble, Simulation, synth

pytestmark = pytest.mark.gpu


def _read_png(path):
    with open(path, "rb") as f:
        data = f.read()
    assert data[:8] == b"\x89PNG\r\n\x1a\n"
    pos, idat, W = 8, b"", None
    while pos < len(data):
        (n,) = struct.unpack(">I", data[pos:pos + 4])
        typ = data[pos + 4:pos + 8]
        body = data[pos + 8:pos + 8 + n]
        (crc,) = struct.unpack(">I", data[pos + 8 + n:pos + 12 + n])
        assert crc == zlib.crc32(typ + body) & 0xFFFFFFFF
        if typ == b"IHDR":
            W, H, depth, ctype = struct.unpack(">IIBB", body[:10])
            assert (depth, ctype) == (8, 6)
        elif typ == b"IDAT":
            idat += body
        pos += 12 + n
    raw = np.frombuffer(zlib.decompress(idat), np.uint8).reshape(H, 1 + 4 * W)
    assert np.all(raw[:, 0] == 0)
    return raw[:, 1:].reshape(H, W, 4)


@pytest.mark.parametrize("what", ["depth", "velocity", "hmax"])
def test_render_matches_shader_restatement(tmp_path, what):
    sc = synth.scenario1(str(tmp_path), W=260, H=210, seed=6, duration=7200.0, name="r")
    with Simulation(sc.yaml_path, quiet=True) as s:
        s.step(700)
        png = str(tmp_path / f"{what}.png")
        img = s.render(what, vmax=3.0 if what != "velocity" else 2.0, png_path=png)
        h = s.field("hmax" if what == "hmax" else "h")
        qx, qy, terr = s.field("qx"), s.field("qy"), s.field("terrain")
    ref = render_oracle.render(h, qx, qy, terr, -1.0, what, 3.0 if what != "velocity" else 2.0)
    assert img.shape == (210, 260, 4)
    wet = (h > 0.01).sum()
    assert wet > 100  # the flood has spread: both branches of the shader are exercised
    assert np.max(np.abs(img.astype(np.int32) - ref)) <= 1
    assert np.array_equal(_read_png(png), img)


def test_ensemble_render_matches_single(tmp_path):
    paths = [synth.ensemble_member(str(tmp_path), 150, 120, seed=8, kst=30.0, q_peak=20.0, t_peak=300.0,
                                   duration=3600.0, name="a").yaml_path,
             synth.scenario1(str(tmp_path), W=200, H=170, seed=9, duration=3600.0, name="b").yaml_path]
    with Ensemble(paths) as e:
        e.step(400)
        imgs = [e.render(m, "hmax") for m in range(2)]
    for m, p in enumerate(paths):
        with Simulation(p, quiet=True) as s:
            s.step(400)
            assert np.array_equal(s.render("hmax"), imgs[m])
