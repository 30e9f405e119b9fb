"""Reader for the oracle harness's named-array dumps ("GDTPDMP1").

Test infrastructure: the dumps are written by ``oracle/ref_harness.cpp`` (the
unmodified reference solve path) and read here by tests only.
"""
from __future__ import annotations

import struct

import numpy as np
import scipy.sparse as sp

_DT = {1: np.int32, 2: np.float64, 3: np.float32, 4: np.int64}


def read_dump(path: str) -> dict:
    out = {}
    with open(path, "rb") as fh:
        if fh.read(8) != b"GDTPDMP1":
            raise ValueError(f"{path}: not an oracle dump")
        while True:
            head = fh.read(4)
            if len(head) < 4:
                break
            (n,) = struct.unpack("<I", head)
            name = fh.read(n).decode()
            (code,) = struct.unpack("<B", fh.read(1))
            (nd,) = struct.unpack("<I", fh.read(4))
            dims = struct.unpack(f"<{nd}q", fh.read(8 * nd))
            dt = np.dtype(_DT[code])
            count = int(np.prod(dims)) if nd else 0
            data = np.frombuffer(fh.read(count * dt.itemsize), dtype=dt).reshape(dims)
            out[name] = data.copy()
    return out


def csr(d: dict, name: str, shape=None) -> sp.csr_matrix:
    ptr, col, val = d[name + "/ptr"], d[name + "/col"], d[name + "/val"]
    n = len(ptr) - 1
    ncol = shape[1] if shape else (int(col.max()) + 1 if len(col) else 0)
    return sp.csr_matrix((val, col, ptr), shape=(n, ncol))
