"""Raster front-end (fip_b200.raster): GeoTIFF / ESRI ASCII grids to the reference's raw float32
`[path, offset]` inputs (src/simdata.cpp:143-150) and back. CPU only."""
import struct

import numpy as np
import pytest

from fip_b200 import config_json, raster, validate


def _dem(H=37, W=53, seed=0):
    rng = np.random.default_rng(seed)
    y = np.arange(H)[:, None]
    x = np.arange(W)[None, :]
    return (100.0 + 0.3 * x - 0.2 * y + rng.standard_normal((H, W))).astype(np.float32)


def test_ascii_grid_round_trip(tmp_path):
    v = _dem()
    v[3, 4] = -9999.0
    p = str(tmp_path / "dem.asc")
    raster.write_ascii_grid(p, v, cellsize=2.5, xll=1000.0, yll=2000.0, nodata=-9999.0)
    r, meta = raster.read_ascii_grid(p)
    assert np.array_equal(r, v)
    assert meta["ncols"] == 53 and meta["nrows"] == 37 and meta["cellsize"] == 2.5 and meta["nodata"] == -9999.0
    assert (meta["xll"], meta["yll"]) == (1000.0, 2000.0)


@pytest.mark.parametrize("dtype,predictor", [("f4", 1), ("f4", 3), ("f8", 3), ("f8", 1), ("i2", 2), ("u1", 1),
                                             ("i4", 2), ("u2", 1)])
@pytest.mark.parametrize("compress", [False, True])
@pytest.mark.parametrize("layout", ["strip1", "strip7", "tile16"])
@pytest.mark.parametrize("big_endian", [False, True])
def test_geotiff_round_trip(tmp_path, dtype, predictor, compress, layout, big_endian):
    v = _dem()
    if dtype[0] in "iu":
        v = np.clip(np.round(v), 0, 250).astype(dtype)
    else:
        v = v.astype(dtype)
    p = str(tmp_path / "dem.tif")
    kw = {"tile": 16} if layout == "tile16" else {"rows_per_strip": int(layout[5:])}
    raster.write_geotiff(p, v, cellsize=3.0, xll=10.0, yll=20.0, nodata=-1.0, compress=compress,
                         predictor=predictor, big_endian=big_endian, **kw)
    r, meta = raster.read_geotiff(p)
    assert np.array_equal(r, v.astype(np.float32))
    assert meta["cellsize"] == 3.0 and meta["nodata"] == -1.0
    assert abs(meta["xll"] - 10.0) < 1e-9 and abs(meta["yll"] - 20.0) < 1e-9


def test_geotiff_written_by_hand(tmp_path):
    """A 3 x 2 float32 TIFF assembled byte by byte from the TIFF 6.0 layout (independent of the
    module's writer): little endian, one uncompressed strip."""
    vals = np.array([[1.5, -2.0, 3.25], [4.0, 5.5, -6.75]], np.float32)
    data = vals.tobytes()
    entries = [(256, 3, 1, 3), (257, 3, 1, 2), (258, 3, 1, 32), (259, 3, 1, 1), (262, 3, 1, 1),
               (273, 4, 1, 0), (277, 3, 1, 1), (278, 3, 1, 2), (279, 4, 1, len(data)), (339, 3, 1, 3)]
    ifd_len = 2 + 12 * len(entries) + 4
    strip_off = 8 + ifd_len
    buf = b"II" + struct.pack("<HI", 42, 8) + struct.pack("<H", len(entries))
    for tag, typ, cnt, val in entries:
        if tag == 273:
            val = strip_off
        if typ == 3:
            buf += struct.pack("<HHIHH", tag, typ, cnt, val, 0)
        else:
            buf += struct.pack("<HHII", tag, typ, cnt, val)
    buf += struct.pack("<I", 0) + data
    p = tmp_path / "hand.tif"
    p.write_bytes(buf)
    r, meta = raster.read_geotiff(str(p))
    assert np.array_equal(r, vals) and meta["nodata"] is None


def test_convert_to_fip_inputs(tmp_path):
    """North-up rasters become fip grids with row 0 on the southern edge; no-data cells get the
    YAML no_data value; the written files load through the library's own loader."""
    dem = _dem(H=20, W=30)
    dem[0, 0] = -32768.0  # north-west corner has no data
    kst = np.full_like(dem, 35.0)
    kst[19, 29] = -1.0
    pd, pk = str(tmp_path / "dem.tif"), str(tmp_path / "kst.asc")
    raster.write_geotiff(pd, dem, cellsize=2.0, nodata=-32768.0, compress=True, predictor=3)
    raster.write_ascii_grid(pk, kst, cellsize=2.0, nodata=-1.0)
    keys = raster.convert(pd, str(tmp_path / "out" / "site"), kst_path=pk, no_data=-9999.0)
    assert keys["W"] == 30 and keys["H"] == 20 and keys["dx"] == 2.0
    g = np.fromfile(keys["terrain"][0], np.float32).reshape(20, 30)
    assert g[19, 0] == -9999.0  # the north-west corner is now in the top row (row H-1)
    assert np.array_equal(g[::-1][1:], dem[1:]) and np.array_equal(g[::-1][0, 1:], dem[0, 1:])
    k = np.fromfile(keys["kSt_var"][0], np.float32).reshape(20, 30)
    assert k[0, 29] == 30.0 and np.all(k[1:] == 35.0)
    y = tmp_path / "site.yml"
    y.write_text(f"name: {tmp_path}/site\nterrain: [{keys['terrain'][0]}, 0]\nkSt_var: [{keys['kSt_var'][0]}, 0]\n"
                 f"W: {keys['W']}\nH: {keys['H']}\ndx: {keys['dx']}\ndt: 0.1\nduration: 10\nno_data: -9999\n")
    validate(str(y))
    cfg = config_json(str(y))
    assert cfg["kst_var"] and cfg["W"] == 30
    back = raster.from_fip_grid(g)
    assert np.array_equal(back[1:], dem[1:])
