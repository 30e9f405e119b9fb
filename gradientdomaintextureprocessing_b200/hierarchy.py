"""Host mirror of the reference's hierarchy interface.

``InitializeHierarchy(mesh, width, height, levels, block_info)`` returns a
``Hierarchy`` whose per-level arrays carry the reference's names and meanings
(``include/Src/Hierarchy.h``: ``GridAtlas``/``HierarchicalSystem``).  The work
is done by the native library (atlas, texel classification and indexing, line
descriptors, boundary elements); this module only moves arrays.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib

_I32 = {"cellCorners": 4, "interiorTexelToCellLines": 5, "nodeinfo": 4, "boundaryAndDeep": 1, "boundaryGlobal": 1, "deepGlobal": 1, "rasterLines": 5,
        "restrictionLines": 5, "deepLines": 5, "prolongationLines": 6, "charts": 12, "nodeType": 1, "cellType": 1,
        "textureNodes": 5, "boundaryNodes": 1}
_F64 = {"chartsd": 4, "textureBary": 2}


class Hierarchy:
    def __init__(self, handle, width: int, height: int):
        self._h = handle
        self.width = width
        self.height = height

    def __del__(self):
        h, self._h = getattr(self, "_h", None), None
        if h:
            try:
                _lib.lib().gdtp_hierarchy_free(h)
            except (TypeError, AttributeError):  # interpreter exit: module globals already cleared
                pass

    @property
    def handle(self):
        return self._h

    @property
    def levels(self) -> int:
        return _lib.lib().gdtp_hierarchy_levels(self._h)

    @property
    def charts(self) -> int:
        return _lib.lib().gdtp_hierarchy_charts(self._h)

    def counts(self, level: int = 0) -> dict:
        c = np.zeros(8, dtype=np.int64)
        _lib.check(_lib.lib().gdtp_hierarchy_counts(self._h, level, _lib.ptr(c)))
        keys = ["numTexels", "numDeepTexels", "numBoundaryTexels", "numCells", "numBoundaryCells", "numInteriorCells",
                "numInteriorTexels", "numCharts"]
        return dict(zip(keys, (int(v) for v in c)))

    def array(self, name: str, level: int = 0) -> np.ndarray:
        L = _lib.lib()
        n = C.c_int64(0)
        _lib.check(L.gdtp_hierarchy_array(self._h, name.encode(), level, None, C.byref(n)))
        base = name.split(".")[-1]
        if name in _F64 or base == "val":
            out = np.empty(n.value, dtype=np.float64)
            cols = _F64.get(name, 1)
        else:
            out = np.empty(n.value, dtype=np.int32)
            cols = _I32.get(name, 1)
        _lib.check(L.gdtp_hierarchy_array(self._h, name.encode(), level, _lib.ptr(out), C.byref(n)))
        return out.reshape(-1, cols) if cols > 1 else out

    def csr(self, name: str, level: int = 0, shape=None):
        import scipy.sparse as sp
        ptr, col, val = (self.array(f"{name}.{p}", level) for p in ("ptr", "col", "val"))
        n = len(ptr) - 1
        ncol = shape[1] if shape else (int(col.max()) + 1 if len(col) else 0)
        return sp.csr_matrix((val, col, ptr), shape=(n, ncol))


def InitializeHierarchy(mesh: dict, width: int | None = None, height: int | None = None, levels: int = 4,
                        block_info=(128, 16, 2, 0, 0)) -> Hierarchy:
    """Builds the texel hierarchy (``HierarchyConstruction.inl:799``)."""
    v = np.ascontiguousarray(mesh["vertices"], dtype=np.float64)
    t = np.ascontiguousarray(mesh["triangles"], dtype=np.int32)
    uv = np.ascontiguousarray(mesh["uv"], dtype=np.float64)
    if width is None:
        height, width = mesh["texture"].shape[:2]
    bi = np.ascontiguousarray(block_info, dtype=np.int32)
    h = C.c_void_p()
    _lib.check(_lib.lib().gdtp_hierarchy_build(_lib.ptr(v), len(v), _lib.ptr(t), len(t), _lib.ptr(uv), int(width),
                                               int(height), int(levels), _lib.ptr(bi), C.byref(h)))
    return Hierarchy(h, int(width), int(height))
