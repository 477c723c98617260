"""FITS map output (lt_write_fits) and a minimal reader of the same primary images.

The writer is the library's (include/lt_b200.h); the reader parses the 80-character
header cards and the big-endian float32 data of a primary image, enough to read the maps
back (NASA/IAU FITS Standard 4.0)."""
from __future__ import annotations

import ctypes as C
import pathlib

import numpy as np


def write_fits(path, image, frame) -> None:
    """Write a 2-D float64 map (ny, nx) over frame = (xmin, xmax, ymin, ymax)."""
    from . import LensError, _Frame, load_library
    a = np.ascontiguousarray(image, np.float64)
    if a.ndim != 2:
        raise ValueError("a map is 2-D")
    L = load_library()
    fn = L.lt_write_fits
    fn.argtypes = [C.c_char_p, C.POINTER(C.c_double), C.c_int32, C.c_int32, C.POINTER(_Frame)]
    st = fn(str(path).encode(), a.ctypes.data_as(C.POINTER(C.c_double)), a.shape[1], a.shape[0],
            C.byref(_Frame(*frame)))
    if st:
        raise LensError(st, f"lt_write_fits {path}")


def read_fits(path):
    """(header dict, image float32 array (ny, nx)) of a primary image."""
    raw = pathlib.Path(path).read_bytes()
    header, order = {}, []
    pos = 0
    while True:
        block = raw[pos:pos + 2880]
        if len(block) < 2880:
            raise ValueError("truncated FITS header")
        pos += 2880
        done = False
        for k in range(36):
            c = block[80 * k:80 * (k + 1)].decode("ascii")
            key = c[:8].strip()
            if key == "END":
                done = True
                break
            if c[8:10] != "= ":
                continue
            val = c[10:]
            if val.lstrip().startswith("'"):
                s = val.lstrip()[1:]
                value = s[:s.index("'")].rstrip()
            else:
                v = val.split("/")[0].strip()
                if v in ("T", "F"):
                    value = v == "T"
                else:
                    value = float(v) if any(ch in v for ch in ".EeDd") else int(v)
            header[key] = value
            order.append(key)
        if done:
            break
    header["_order"] = order
    nx, ny = header["NAXIS1"], header["NAXIS2"]
    if header["BITPIX"] != -32:
        raise ValueError("only float32 images")
    data = np.frombuffer(raw[pos:pos + 4 * nx * ny], dtype=">f4").reshape(ny, nx)
    return header, data.astype(np.float32)
