"""Reader for the oracle driver's tagged binary dumps (oracle/refdriver/refdump.h)."""
from __future__ import annotations

import struct

import numpy as np


def read_dump(path: str) -> dict[str, np.ndarray]:
    out: dict[str, np.ndarray] = {}
    with open(path, "rb") as f:
        data = f.read()
    pos = 0
    while pos < len(data):
        (nlen,) = struct.unpack_from("<i", data, pos)
        pos += 4
        name = data[pos:pos + nlen].decode()
        pos += nlen
        kind = data[pos:pos + 1].decode()
        pos += 1
        (count,) = struct.unpack_from("<q", data, pos)
        pos += 8
        dt = np.float64 if kind == "d" else np.int32
        nbytes = count * np.dtype(dt).itemsize
        out[name] = np.frombuffer(data, dtype=dt, count=count, offset=pos).copy()
        pos += nbytes
    return out
