"""PGXD: the flat container of named arrays used to move GeMSLR structures.

Layout: the 4-byte magic ``PGXD`` followed by records
``[u32 name_len][name][u8 dtype][u64 count][count elements]`` with dtype
0 = int32, 1 = float64, 2 = int64, 3 = float32, little-endian.  The same
format is written by the reference-side exporter and by this package, so structures can be handed over as files as well as through
the C ABI.
"""
from __future__ import annotations

import struct
from typing import Dict

import numpy as np

_DT = {0: np.int32, 1: np.float64, 2: np.int64, 3: np.float32}
_CODE = {np.dtype(np.int32): 0, np.dtype(np.float64): 1, np.dtype(np.int64): 2, np.dtype(np.float32): 3}


def read(path: str) -> Dict[str, np.ndarray]:
    out: Dict[str, np.ndarray] = {}
    with open(path, "rb") as f:
        data = f.read()
    if data[:4] != b"PGXD":
        raise ValueError(f"{path}: not a PGXD container")
    off = 4
    n = len(data)
    while off < n:
        (ln,) = struct.unpack_from("<I", data, off)
        off += 4
        name = data[off:off + ln].decode()
        off += ln
        code = data[off]
        off += 1
        (count,) = struct.unpack_from("<Q", data, off)
        off += 8
        dt = np.dtype(_DT[code])
        nbytes = dt.itemsize * count
        out[name] = np.frombuffer(data, dtype=dt, count=count, offset=off).copy()
        off += nbytes
    return out


def write(path: str, arrays: Dict[str, np.ndarray]) -> None:
    with open(path, "wb") as f:
        f.write(b"PGXD")
        for name, arr in arrays.items():
            a = np.ascontiguousarray(arr)
            code = _CODE[a.dtype]
            nb = name.encode()
            f.write(struct.pack("<I", len(nb)))
            f.write(nb)
            f.write(struct.pack("<BQ", code, a.size))
            f.write(a.tobytes())
