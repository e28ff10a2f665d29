"""Reader for the GeoTIFF and PLY files the host library writes (test helper).

Decodes classic little-endian TIFFs with float32 samples in strips,
pixel-interleaved, uncompressed / DEFLATE / ZSTD (through libzstd.so.1), with
or without the floating-point predictor (Adobe TIFF Technical Note 3), and
returns the bands plus the GeoTIFF / GDAL tags."""
from __future__ import annotations

import ctypes
import struct
import zlib

import numpy as np

TYPES = {1: ("B", 1), 2: ("s", 1), 3: ("H", 2), 4: ("I", 4), 12: ("d", 8), 16: ("Q", 8)}


def _zstd_decompress(data: bytes, size: int) -> bytes:
    lib = ctypes.CDLL("libzstd.so.1")
    lib.ZSTD_decompress.restype = ctypes.c_size_t
    lib.ZSTD_decompress.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_size_t]
    lib.ZSTD_isError.restype = ctypes.c_uint
    out = ctypes.create_string_buffer(size)
    r = lib.ZSTD_decompress(out, size, data, len(data))
    if lib.ZSTD_isError(r):
        raise ValueError("zstd error")
    return out.raw[:r]


def _unpredict_fp(block: bytes, width_samples: int, rows: int, stride: int) -> np.ndarray:
    """Undo the floating-point predictor row by row -> float32 samples."""
    b = np.frombuffer(block, dtype=np.uint8).reshape(rows, width_samples * 4)
    out = np.empty((rows, width_samples), dtype=np.float32)
    n = width_samples
    for r in range(rows):
        row = b[r].astype(np.int64)
        # undo the byte differences at distance `stride`: a cumulative sum per residue class
        for s0 in range(stride):
            row[s0::stride] = np.cumsum(row[s0::stride]) & 0xFF
        row = row.astype(np.uint8)
        be = np.stack([row[k * n:(k + 1) * n] for k in range(4)], axis=1)  # [n, 4], most significant byte first
        out[r] = be[:, ::-1].copy().view(np.float32).reshape(n)
    return out


def read_tiff(path: str) -> dict:
    buf = open(path, "rb").read()
    assert buf[:4] == b"II*\x00", "not a little-endian classic TIFF"
    (ifd,) = struct.unpack_from("<I", buf, 4)
    (n,) = struct.unpack_from("<H", buf, ifd)
    tags = {}
    for k in range(n):
        tag, typ, cnt, val = struct.unpack_from("<HHII", buf, ifd + 2 + 12 * k)
        fmt, size = TYPES[typ]
        off = ifd + 2 + 12 * k + 8 if size * cnt <= 4 else val
        if typ == 2:
            tags[tag] = buf[off:off + cnt].rstrip(b"\x00").decode()
        else:
            tags[tag] = list(struct.unpack_from("<" + fmt * cnt, buf, off))
    nx, ny = tags[256][0], tags[257][0]
    spp = tags.get(277, [1])[0]
    comp = tags.get(259, [1])[0]
    pred = tags.get(317, [1])[0]
    planar = tags.get(284, [1])[0]
    rps = tags.get(278, [ny])[0]
    assert all(b == 32 for b in tags[258]) and all(f == 3 for f in tags.get(339, [3])), "float32 samples expected"
    assert planar == 1, "pixel-interleaved samples expected"
    offs, counts = tags[273], tags[279]
    per_row = nx * spp
    rows_out = []
    for s, (o, c) in enumerate(zip(offs, counts)):
        data = buf[o:o + c]
        rows = min(rps, ny - s * rps)
        raw_size = rows * per_row * 4
        if comp == 8:
            data = zlib.decompress(data)
        elif comp == 50000:
            data = _zstd_decompress(data, raw_size)
        elif comp != 1:
            raise ValueError(f"compression {comp}")
        if pred == 3:
            arr = _unpredict_fp(data, per_row, rows, spp)
        else:
            arr = np.frombuffer(data, dtype=np.float32).reshape(rows, per_row)
        rows_out.append(arr)
    img = np.concatenate(rows_out, axis=0)
    bands = img.reshape(ny, nx, spp).transpose(2, 0, 1)
    return {"bands": np.ascontiguousarray(bands), "nx": nx, "ny": ny, "compression": comp, "predictor": pred,
            "pixel_scale": tags.get(33550), "tiepoint": tags.get(33922), "geokeys": tags.get(34735),
            "metadata": tags.get(42112, ""), "nodata": tags.get(42113)}


def read_ply(path: str) -> dict:
    buf = open(path, "rb").read()
    end = buf.index(b"end_header\n") + len(b"end_header\n")
    head = buf[:end].decode().splitlines()
    assert head[0] == "ply" and head[1] == "format binary_little_endian 1.0"
    n = 0
    props = []
    for ln in head[2:]:
        if ln.startswith("element vertex"):
            n = int(ln.split()[2])
        elif ln.startswith("property float"):
            props.append(ln.split()[2])
    data = np.frombuffer(buf, dtype=np.float32, count=n * len(props), offset=end).reshape(n, len(props))
    return {p: data[:, k].copy() for k, p in enumerate(props)}
