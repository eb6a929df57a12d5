"""Raster front-end: GeoTIFF and ESRI ASCII grids to and from fip's raw input grids.

The reference reads terrain, kSt, z, qx and qy only as raw float32 W*H files at a byte offset
(`terrain: [path, offset]`, src/simdata.cpp:143-150, src/utils.h:45-54) and leaves conversion
from GIS formats to the user. This module converts:

* ESRI ASCII grids (`ncols`, `nrows`, `xllcorner|xllcenter`, `yllcorner|yllcenter`, `cellsize`,
  optional `NODATA_value`, then nrows lines of values, northernmost first);
* baseline GeoTIFF: one band of uint8/int8/uint16/int16/uint32/int32/float32/float64 samples,
  strips or tiles, no compression or deflate (zlib), predictor none, horizontal differencing
  or floating point, little or big endian, GDAL_NODATA, ModelPixelScale / ModelTiepoint.

Orientation: rasters store the northernmost row first; fip's row 0 is the southern edge (row =
y, north = +1 row; the `bottom` boundary is row 0, `top` is row H-1). Conversions flip the rows
unless told not to. No-data cells get the YAML `no_data` value (cells the solver never writes).

    python -m fip_b200.raster dem.tif out/prefix [--kst landuse.asc] [--no-flip] [--no-data -9999]

writes out/prefix_terrain.bin (and _kst.bin) and prints the YAML keys to paste.
"""
from __future__ import annotations

import argparse
import json
import os
import struct
import sys
import zlib

import numpy as np

# ------------------------------------------------------------------------------------------
# ESRI ASCII grid
# ------------------------------------------------------------------------------------------


def read_ascii_grid(path: str):
    """(values, meta): values float32 (nrows, ncols), northernmost row first."""
    meta = {}
    with open(path) as f:
        text = f.read()
    tokens = text.split()
    i = 0
    keys = {"ncols", "nrows", "xllcorner", "xllcenter", "yllcorner", "yllcenter", "cellsize", "nodata_value",
            "dx", "dy"}
    while i + 1 < len(tokens) and tokens[i].lower() in keys:
        meta[tokens[i].lower()] = float(tokens[i + 1])
        i += 2
    nc, nr = int(meta["ncols"]), int(meta["nrows"])
    vals = np.array(tokens[i:i + nc * nr], dtype=np.float64)
    if vals.size != nc * nr:
        raise ValueError(f"{path}: expected {nc * nr} values, found {vals.size}")
    if "cellsize" not in meta and "dx" in meta:
        meta["cellsize"] = meta["dx"]
    out = {"ncols": nc, "nrows": nr, "cellsize": meta.get("cellsize", 1.0),
           "nodata": meta.get("nodata_value"),
           "xll": meta.get("xllcorner", meta.get("xllcenter", 0.0) - 0.5 * meta.get("cellsize", 1.0)),
           "yll": meta.get("yllcorner", meta.get("yllcenter", 0.0) - 0.5 * meta.get("cellsize", 1.0))}
    return vals.reshape(nr, nc).astype(np.float32), out


def write_ascii_grid(path: str, values: np.ndarray, cellsize: float = 1.0, xll: float = 0.0, yll: float = 0.0,
                     nodata: float | None = None) -> None:
    """values (nrows, ncols), northernmost row first."""
    v = np.asarray(values)
    nr, nc = v.shape
    with open(path, "w") as f:
        f.write(f"ncols {nc}\nnrows {nr}\nxllcorner {xll!r}\nyllcorner {yll!r}\ncellsize {cellsize!r}\n")
        if nodata is not None:
            f.write(f"NODATA_value {nodata!r}\n")
        for row in v:
            f.write(" ".join(f"{float(x):.9g}" for x in row) + "\n")


# ------------------------------------------------------------------------------------------
# GeoTIFF (baseline TIFF 6.0 + the GeoTIFF georeferencing tags GDAL writes)
# ------------------------------------------------------------------------------------------

_TYPES = {1: ("B", 1), 2: ("s", 1), 3: ("H", 2), 4: ("I", 4), 5: ("II", 8), 6: ("b", 1), 7: ("B", 1), 8: ("h", 2),
          9: ("i", 4), 10: ("ii", 8), 11: ("f", 4), 12: ("d", 8), 16: ("Q", 8), 17: ("q", 8), 18: ("Q", 8)}
_SAMPLE = {(1, 8): "u1", (1, 16): "u2", (1, 32): "u4", (2, 8): "i1", (2, 16): "i2", (2, 32): "i4", (3, 32): "f4",
           (3, 64): "f8"}


def _tags(buf: bytes, bo: str, off: int, big: bool):
    if big:
        (n,) = struct.unpack_from(bo + "Q", buf, off)
        off += 8
        entry, cnt_fmt, inline = 20, "Q", 8
    else:
        (n,) = struct.unpack_from(bo + "H", buf, off)
        off += 2
        entry, cnt_fmt, inline = 12, "I", 4
    tags = {}
    for k in range(n):
        e = off + k * entry
        tag, typ = struct.unpack_from(bo + "HH", buf, e)
        (cnt,) = struct.unpack_from(bo + cnt_fmt, buf, e + 4)
        if typ not in _TYPES:
            continue
        fmt, size = _TYPES[typ]
        total = size * cnt
        vpos = e + 4 + struct.calcsize(cnt_fmt)
        if total > inline:
            (vpos,) = struct.unpack_from(bo + cnt_fmt, buf, vpos)
        if typ == 2:
            tags[tag] = buf[vpos:vpos + cnt].split(b"\0")[0].decode(errors="replace")
        elif typ in (5, 10):
            raw = struct.unpack_from(bo + fmt[0] * (2 * cnt), buf, vpos)
            tags[tag] = [raw[2 * j] / raw[2 * j + 1] if raw[2 * j + 1] else 0.0 for j in range(cnt)]
        else:
            tags[tag] = list(struct.unpack_from(bo + fmt * cnt, buf, vpos))
    return tags


def _unpredict(block: np.ndarray, predictor: int, dtype: np.dtype, width: int) -> np.ndarray:
    """block: raw bytes of rows x width samples after decompression."""
    if predictor == 1:
        return block.view(dtype)
    if predictor == 2:  # horizontal differencing of integer samples
        a = block.view(dtype).reshape(-1, width).copy()
        np.cumsum(a, axis=1, dtype=dtype, out=a)
        return a.reshape(-1)
    if predictor == 3:  # floating point: bytes shuffled by significance, then differenced
        nb = dtype.itemsize
        b = block.reshape(-1, width * nb).astype(np.uint8)
        b = np.cumsum(b, axis=1, dtype=np.uint8)
        b = b.reshape(-1, nb, width).transpose(0, 2, 1)  # planes: most significant byte first
        if dtype.byteorder == "<" or (dtype.byteorder == "=" and sys.byteorder == "little"):
            b = b[:, :, ::-1]
        return np.ascontiguousarray(b).reshape(-1).view(dtype)
    raise ValueError(f"unsupported TIFF predictor {predictor}")


def read_geotiff(path: str):
    """(values, meta): values float32 (rows, cols), northernmost row first (TIFF row order)."""
    with open(path, "rb") as f:
        buf = f.read()
    if buf[:2] == b"II":
        bo = "<"
    elif buf[:2] == b"MM":
        bo = ">"
    else:
        raise ValueError(f"{path}: not a TIFF file")
    (magic,) = struct.unpack_from(bo + "H", buf, 2)
    big = magic == 43
    if magic not in (42, 43):
        raise ValueError(f"{path}: not a TIFF file")
    (ifd,) = struct.unpack_from(bo + ("Q" if big else "I"), buf, 8 if big else 4)
    t = _tags(buf, bo, ifd, big)
    W, H = int(t[256][0]), int(t[257][0])
    bits = int(t.get(258, [8])[0])
    comp = int(t.get(259, [1])[0])
    spp = int(t.get(277, [1])[0])
    fmt = int(t.get(339, [1])[0])
    pred = int(t.get(317, [1])[0])
    if spp != 1:
        raise ValueError(f"{path}: {spp} samples per pixel; one band expected")
    if (fmt, bits) not in _SAMPLE:
        raise ValueError(f"{path}: unsupported sample format {fmt} / {bits} bits")
    dt = np.dtype(_SAMPLE[(fmt, bits)]).newbyteorder(bo)
    if comp not in (1, 8, 32946):
        raise ValueError(f"{path}: unsupported compression {comp} (none and deflate are read)")

    def decode(off, cnt, rows, width):
        raw = buf[off:off + cnt]
        if comp != 1:
            raw = zlib.decompress(raw)
        need = rows * width * dt.itemsize
        raw = np.frombuffer(raw, dtype=np.uint8)[:need]
        if raw.size < need:
            raise ValueError(f"{path}: truncated block")
        return _unpredict(raw, pred, dt, width)

    out = np.empty((H, W), dtype=np.float64)
    if 322 in t:  # tiles
        tw, tl = int(t[322][0]), int(t[323][0])
        offs, cnts = t[324], t[325]
        across = (W + tw - 1) // tw
        for k, (o, c) in enumerate(zip(offs, cnts)):
            ty, tx = divmod(k, across)
            blk = decode(int(o), int(c), tl, tw).reshape(tl, tw)
            r0, c0 = ty * tl, tx * tw
            r1, c1 = min(r0 + tl, H), min(c0 + tw, W)
            out[r0:r1, c0:c1] = blk[:r1 - r0, :c1 - c0]
    else:
        rps = int(t.get(278, [H])[0])
        offs, cnts = t[273], t[279]
        for k, (o, c) in enumerate(zip(offs, cnts)):
            r0 = k * rps
            rows = min(rps, H - r0)
            out[r0:r0 + rows] = decode(int(o), int(c), rows, W).reshape(rows, W)
    meta = {"ncols": W, "nrows": H, "nodata": None, "cellsize": None, "xll": None, "yll": None}
    if 42113 in t:
        try:
            meta["nodata"] = float(t[42113])
        except ValueError:
            pass
    if 33550 in t:
        sx, sy = t[33550][0], t[33550][1]
        meta["cellsize"] = float(sx)
        meta["cellsize_y"] = float(sy)
        if 33922 in t:
            tp = t[33922]
            i, j, x, y = tp[0], tp[1], tp[3], tp[4]
            meta["xll"] = float(x - i * sx)
            meta["yll"] = float(y + j * sy - H * sy)
    return out.astype(np.float32), meta


def write_geotiff(path: str, values: np.ndarray, cellsize: float | None = None, xll: float = 0.0, yll: float = 0.0,
                  nodata: float | None = None, compress: bool = False, predictor: int = 1, rows_per_strip: int = 16,
                  tile: int | None = None, big_endian: bool = False) -> None:
    """Baseline GeoTIFF of one band; values (rows, cols) northernmost row first, dtype kept."""
    v = np.ascontiguousarray(values)
    H, W = v.shape
    bo = ">" if big_endian else "<"
    dt = v.dtype.newbyteorder(bo)
    v = v.astype(dt)
    kind = {"u": 1, "i": 2, "f": 3}[dt.kind]
    bits = dt.itemsize * 8

    def encode(block: np.ndarray) -> bytes:
        rows, width = block.shape
        if predictor == 2:
            d = block.copy()
            d[:, 1:] = block[:, 1:] - block[:, :-1]
            raw = d.tobytes()
        elif predictor == 3:
            nb = dt.itemsize
            b = np.frombuffer(block.tobytes(), np.uint8).reshape(rows, width, nb)
            if bo == "<":
                b = b[:, :, ::-1]
            planes = np.ascontiguousarray(b.transpose(0, 2, 1)).reshape(rows, width * nb)
            diff = planes.copy()
            diff[:, 1:] = planes[:, 1:] - planes[:, :-1]
            raw = diff.tobytes()
        else:
            raw = block.tobytes()
        return zlib.compress(raw) if compress else raw

    blocks = []
    if tile:
        across, down = (W + tile - 1) // tile, (H + tile - 1) // tile
        for ty in range(down):
            for tx in range(across):
                blk = np.zeros((tile, tile), dtype=dt)
                part = v[ty * tile:(ty + 1) * tile, tx * tile:(tx + 1) * tile]
                blk[:part.shape[0], :part.shape[1]] = part
                blocks.append(encode(blk))
    else:
        for r0 in range(0, H, rows_per_strip):
            blocks.append(encode(v[r0:r0 + rows_per_strip]))
    entries = []  # (tag, type, values)
    entries.append((256, 4, [W]))
    entries.append((257, 4, [H]))
    entries.append((258, 3, [bits]))
    entries.append((259, 3, [8 if compress else 1]))
    entries.append((262, 3, [1]))
    entries.append((277, 3, [1]))
    entries.append((284, 3, [1]))
    if predictor != 1:
        entries.append((317, 3, [predictor]))
    entries.append((339, 3, [kind]))
    if tile:
        entries += [(322, 4, [tile]), (323, 4, [tile]), (324, 4, None), (325, 4, [len(b) for b in blocks])]
    else:
        entries += [(273, 4, None), (278, 4, [rows_per_strip]), (279, 4, [len(b) for b in blocks])]
    if cellsize:
        entries.append((33550, 12, [cellsize, cellsize, 0.0]))
        entries.append((33922, 12, [0.0, 0.0, 0.0, xll, yll + H * cellsize, 0.0]))
    if nodata is not None:
        entries.append((42113, 2, repr(float(nodata)).encode() + b"\0"))
    entries.sort(key=lambda e: e[0])
    # layout: header, IFD, out-of-line values, blocks
    n = len(entries)
    ifd_off = 8
    data_off = ifd_off + 2 + 12 * n + 4
    extra = b""
    fmt_of = {3: "H", 4: "I", 12: "d"}

    def packed(typ, vals):
        if typ == 2:
            return vals
        return struct.pack(bo + fmt_of[typ] * len(vals), *vals)

    block_base = None
    # first pass: size of the out-of-line area (offset arrays are placeholders of the right size)
    sizes = []
    for tag, typ, vals in entries:
        vv = [0] * len(blocks) if vals is None else vals
        sizes.append(len(packed(typ, vv)))
    block_base = data_off + sum(s for s in sizes if s > 4)
    offsets, pos = [], block_base
    for b in blocks:
        offsets.append(pos)
        pos += len(b)
    ifd = struct.pack(bo + "H", n)
    for tag, typ, vals in entries:
        vv = offsets if vals is None else vals
        p = packed(typ, vv)
        cnt = len(vv) if typ != 2 else len(p)
        if len(p) <= 4:
            ifd += struct.pack(bo + "HHI", tag, typ, cnt) + p.ljust(4, b"\0")
        else:
            ifd += struct.pack(bo + "HHII", tag, typ, cnt, data_off + len(extra))
            extra += p
    ifd += struct.pack(bo + "I", 0)
    with open(path, "wb") as f:
        f.write((b"II" if bo == "<" else b"MM") + struct.pack(bo + "HI", 42, ifd_off))
        f.write(ifd)
        f.write(extra)
        for b in blocks:
            f.write(b)


# ------------------------------------------------------------------------------------------
# conversion to fip inputs and back
# ------------------------------------------------------------------------------------------


def read_raster(path: str):
    low = path.lower()
    if low.endswith((".tif", ".tiff", ".gtif")):
        return read_geotiff(path)
    return read_ascii_grid(path)


def to_fip_grid(values: np.ndarray, meta: dict, flip: bool = True, no_data: float = -9999.0) -> np.ndarray:
    """Raster (northernmost row first) to a fip grid (row 0 = southern edge), no-data mapped."""
    v = np.asarray(values, dtype=np.float32)
    if meta.get("nodata") is not None:
        v = np.where(v == np.float32(meta["nodata"]), np.float32(no_data), v)
    v = np.where(np.isfinite(v), v, np.float32(no_data))
    return np.ascontiguousarray(v[::-1] if flip else v, dtype=np.float32)


def from_fip_grid(grid: np.ndarray, flip: bool = True) -> np.ndarray:
    """fip grid (row 0 = south) to raster order (northernmost row first)."""
    g = np.asarray(grid, dtype=np.float32)
    return np.ascontiguousarray(g[::-1] if flip else g)


def convert(terrain_path: str, out_prefix: str, kst_path: str | None = None, flip: bool = True,
            no_data: float = -9999.0) -> dict:
    """Writes <out_prefix>_terrain.bin (and _kst.bin) and returns the YAML keys for them."""
    vals, meta = read_raster(terrain_path)
    grid = to_fip_grid(vals, meta, flip, no_data)
    H, W = grid.shape
    os.makedirs(os.path.dirname(os.path.abspath(out_prefix)), exist_ok=True)
    tpath = out_prefix + "_terrain.bin"
    grid.tofile(tpath)
    keys = {"terrain": [tpath, 0], "W": W, "H": H, "no_data": no_data}
    if meta.get("cellsize"):
        keys["dx"] = float(meta["cellsize"])
    if kst_path:
        kv, km = read_raster(kst_path)
        if kv.shape != vals.shape:
            raise ValueError(f"{kst_path}: {kv.shape} cells, the terrain has {vals.shape}")
        kg = to_fip_grid(kv, km, flip, 30.0)  # Strickler default where the land-use raster has no data
        kpath = out_prefix + "_kst.bin"
        kg.tofile(kpath)
        keys["kSt_var"] = [kpath, 0]
    return keys


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description="GeoTIFF / ASCII grid to fip raw float32 inputs")
    ap.add_argument("terrain")
    ap.add_argument("out_prefix")
    ap.add_argument("--kst", help="Strickler roughness raster of the same size")
    ap.add_argument("--no-flip", action="store_true", help="keep the raster's row order (row 0 = north)")
    ap.add_argument("--no-data", type=float, default=-9999.0)
    a = ap.parse_args(argv)
    keys = convert(a.terrain, a.out_prefix, a.kst, not a.no_flip, a.no_data)
    for k, v in keys.items():
        print(f"{k}: {json.dumps(v) if isinstance(v, list) else v}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
