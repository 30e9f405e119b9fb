"""Host mirror of the reference's system-level interface for the solve path.

The names follow the reference so callers read the same:

* ``InitializeMassAndStiffness(hierarchy)``  -> ``System`` (FP64 assembly on the
  device; ``include/Src/MassAndStiffness.h:490``), metric from
  ``InitializeMetric`` (``include/Src/Metric.inl:448``) unless one is given.
* ``UpdateLinearSystem(stiffness, screen, system)``
  (``include/Src/UpdateCoefficients.inl:463``).
* ``MultiplyBySystemMatrix_NoReciprocals(system, x, which)``
  (``include/Src/IterativeSolvers.inl:881``).
* ``VCycle(system, x, rhs)`` (``include/Src/IterativeSolvers.inl:1211``).
* ``solve(system, b, x0, tol)``: mixed-precision solve (FP32 V-cycles inside FP64
  refinement), the device replacement for the app's loop of V-cycles.

All work runs in ``libgdtp.so``; every call raises ``GDTPError`` on failure
(no CUDA device included).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .hierarchy import Hierarchy

MASS, STIFFNESS, SYSTEM = 1, 2, 0


class System:
    def __init__(self, hierarchy: Hierarchy, device: int = 0, parameter_metric: np.ndarray | None = None,
                 vertices: np.ndarray | None = None):
        self.hierarchy = hierarchy  # keeps the hierarchy alive for the system's lifetime
        self.n = hierarchy.counts(0)["numTexels"]
        pm = None if parameter_metric is None else np.ascontiguousarray(parameter_metric, dtype=np.float64)
        vv = None if vertices is None else np.ascontiguousarray(vertices, dtype=np.float64)
        h = C.c_void_p()
        _lib.check(_lib.lib().gdtp_system_create(hierarchy.handle, int(device), 0 if pm is None else 1, _lib.ptr(pm),
                                                 _lib.ptr(vv), 0 if vv is None else len(vv), C.byref(h)))
        self._s = h

    def __del__(self):
        s, self._s = getattr(self, "_s", None), None
        if s:
            try:
                _lib.lib().gdtp_system_free(s)
            except (TypeError, AttributeError):  # interpreter exit: module globals already cleared
                pass

    @property
    def handle(self):
        return self._s

    # -- set-up -----------------------------------------------------------------
    def update(self, stiffness_weight: float, screen_weight: float = 1.0) -> None:
        _lib.check(_lib.lib().gdtp_system_update(self._s, float(stiffness_weight), float(screen_weight)))

    def set(self, knob: str, value: float) -> None:
        _lib.check(_lib.lib().gdtp_system_set(self._s, knob.encode(), float(value)))

    def get(self, knob: str) -> float:
        v = C.c_double()
        _lib.check(_lib.lib().gdtp_system_get(self._s, knob.encode(), C.byref(v)))
        return v.value

    def autotune(self, b: np.ndarray, tol: float = 1e-6) -> dict:
        """Picks the fastest converging smoother setting for solves like ``b``."""
        b, k = self._vec(b, np.float64)
        out = np.zeros(5)
        _lib.check(_lib.lib().gdtp_system_autotune(self._s, _lib.ptr(b), k, float(tol), _lib.ptr(out)))
        knobs = {name: int(self.get(name)) for name in ("pre_sweeps", "post_sweeps", "pre_boundary", "post_boundary",
                                                         "coarse_pre_sweeps", "coarse_post_sweeps", "coarse_from", "krylov",
                                                         "tile_texels", "tile_pre_sweeps", "tile_post_sweeps", "tile_rounds",
                                                         "tile_finish")}
        knobs["seconds"] = float(out[4])
        return knobs

    def device_bytes(self) -> int:
        b = C.c_int64()
        _lib.check(_lib.lib().gdtp_system_device_bytes(self._s, C.byref(b)))
        return b.value

    def array(self, name: str, level: int = 0) -> np.ndarray:
        L = _lib.lib()
        n = C.c_int64()
        _lib.check(L.gdtp_system_array(self._s, name.encode(), level, None, C.byref(n)))
        if name in ("levelsUsed",) or name.endswith((".ptr", ".col")):
            out = np.empty(n.value, dtype=np.int32)
        else:
            out = np.empty(n.value, dtype=np.float64)
        _lib.check(L.gdtp_system_array(self._s, name.encode(), level, _lib.ptr(out), C.byref(n)))
        if name in ("deepMass", "deepStiffness", "coef.deep"):
            return out.reshape(-1, 10)
        return out

    def csr(self, name: str, level: int = 0, shape=None):
        import scipy.sparse as sp
        ptr, col, val = (self.array(f"{name}.{p}", level) for p in ("ptr", "col", "val"))
        ncol = shape[1] if shape else (int(col.max()) + 1 if len(col) else 0)
        return sp.csr_matrix((val, col, ptr), shape=(len(ptr) - 1, ncol))

    @property
    def levels_used(self) -> int:
        return int(self.array("levelsUsed")[0])

    # -- operators and solves -----------------------------------------------------
    def _vec(self, a: np.ndarray, dtype) -> tuple[np.ndarray, int]:
        a = np.ascontiguousarray(a, dtype=dtype)
        if a.ndim == 1:
            a = a[:, None]
        if a.shape[0] != self.n:
            raise ValueError(f"vector has {a.shape[0]} texels, system has {self.n}")
        return a, a.shape[1]

    def apply(self, x: np.ndarray, which: int = SYSTEM) -> np.ndarray:
        x, k = self._vec(x, np.float64)
        y = np.empty_like(x)
        _lib.check(_lib.lib().gdtp_apply(self._s, int(which), _lib.ptr(x), _lib.ptr(y), k))
        return y

    def vcycle(self, x: np.ndarray, rhs: np.ndarray) -> np.ndarray:
        x, k = self._vec(x, np.float32)
        x = x.copy()
        rhs, _ = self._vec(rhs, np.float32)
        _lib.check(_lib.lib().gdtp_vcycle(self._s, _lib.ptr(x), _lib.ptr(rhs), k))
        return x

    def relax(self, x: np.ndarray, rhs: np.ndarray, sweeps: int = 1, reverse: bool = False) -> np.ndarray:
        """``Relaxation`` (IterativeSolvers.inl:174-395): level-0 Gauss-Seidel
        sweeps with the V-cycle's level-0 smoother; returns the new x."""
        x, k = self._vec(x, np.float32)
        x = x.copy()
        rhs, _ = self._vec(rhs, np.float32)
        _lib.check(_lib.lib().gdtp_relax(self._s, _lib.ptr(x), _lib.ptr(rhs), k, int(sweeps), int(bool(reverse))))
        return x

    def residual(self, b: np.ndarray, x: np.ndarray) -> np.ndarray:
        b, k = self._vec(b, np.float64)
        x, _ = self._vec(x, np.float64)
        rel = np.empty(k)
        _lib.check(_lib.lib().gdtp_residual(self._s, _lib.ptr(b), _lib.ptr(x), k, _lib.ptr(rel)))
        return rel

    def solve(self, b: np.ndarray, x0: np.ndarray | None = None, tol: float = 1e-6, max_iters: int = 60,
              precision: str = "mixed", check: bool = True):
        b, k = self._vec(b, np.float64)
        x = np.zeros_like(b) if x0 is None else self._vec(x0, np.float64)[0].copy()
        rep = _lib.Report()
        fn = _lib.lib().gdtp_solve if precision == "mixed" else _lib.lib().gdtp_solve_fp64
        code = fn(self._s, _lib.ptr(b), _lib.ptr(x), k, float(tol), int(max_iters), C.byref(rep))
        if code != 0 and (check or code != -4):
            _lib.check(code)
        return x, {"iterations": rep.iterations, "vcycles": rep.vcycles, "rel_residual_max": rep.rel_residual_max,
                   "seconds": rep.seconds, "converged": code == 0}

    def solve_stream(self, bs, xs=None, tol: float = 1e-6, max_iters: int = 60, check: bool = True):
        """Solve a sequence of problems (each from a zero guess) through
        gdtp_solve_stream: the upload of the next right-hand side and the
        download of the previous solution overlap each solve.  bs: arrays of
        the same shape (numTexels[, k]); xs: optional output arrays of that
        shape (pinned host memory, e.g. a pinned torch tensor's numpy view,
        gives the overlap).  Returns (xs, reports)."""
        vecs = [self._vec(b, np.float64) for b in bs]
        if len({(v.shape, k) for v, k in vecs}) > 1:
            raise ValueError("solve_stream: right-hand sides of different shapes")
        k = vecs[0][1] if vecs else 1
        if xs is None:
            xs = [np.zeros_like(v) for v, _ in vecs]
        if len(xs) != len(vecs) or any(x.size != v.size or x.dtype != np.float64 or not x.flags.c_contiguous
                                       for x, (v, _) in zip(xs, vecs)):
            raise ValueError("solve_stream: outputs must be C-contiguous float64 arrays sized as the right-hand sides")
        n = len(vecs)
        bp = (C.c_void_p * max(n, 1))(*[v.ctypes.data for v, _ in vecs])
        xp = (C.c_void_p * max(n, 1))(*[x.ctypes.data for x in xs])
        reps = (_lib.Report * max(n, 1))()
        code = _lib.lib().gdtp_solve_stream(self._s, bp, xp, n, k, float(tol), int(max_iters), reps)
        if code != 0 and (check or code != -4):
            _lib.check(code)
        out = [{"iterations": r.iterations, "vcycles": r.vcycles, "rel_residual_max": r.rel_residual_max, "seconds": r.seconds,
                "converged": r.rel_residual_max <= tol} for r in reps[:n]]
        return xs, out


class Brush:
    """The sharpening brush's cell-based stiffness of a signal f (numTexels x k):
    ``apply(mask)`` = sum over cells of mask[cell] S_cell f, the reference's
    CellStiffnessToTexelStiffness (IterativeSolvers.inl:1170-1208) on the
    device.  The mask has one value per cell (the hierarchy's global cell order)."""

    def __init__(self, system: System, signal: np.ndarray):
        self.system = system  # the brush reads the system's device data
        f, self.k = system._vec(signal, np.float64)
        h = C.c_void_p()
        _lib.check(_lib.lib().gdtp_brush_create(system.handle, _lib.ptr(f), self.k, C.byref(h)))
        self._b = h

    def __del__(self):
        b, self._b = getattr(self, "_b", None), None
        if b:
            try:
                _lib.lib().gdtp_brush_free(b)
            except (TypeError, AttributeError):  # interpreter exit
                pass

    def apply(self, mask: np.ndarray) -> np.ndarray:
        m = np.ascontiguousarray(mask, dtype=np.float64)
        out = np.empty((self.system.n, self.k))
        _lib.check(_lib.lib().gdtp_brush_apply(self._b, _lib.ptr(m), _lib.ptr(out)))
        return out


def CellStiffnessToTexelStiffness(brush: Brush, cell_mask: np.ndarray) -> np.ndarray:
    return brush.apply(cell_mask)


def InitializeMassAndStiffness(hierarchy: Hierarchy, device: int = 0, parameter_metric=None) -> System:
    return System(hierarchy, device=device, parameter_metric=parameter_metric)


def UpdateLinearSystem(stiffness_weight: float, screen_weight: float, system: System) -> None:
    system.update(stiffness_weight, screen_weight)


def MultiplyBySystemMatrix_NoReciprocals(system: System, x: np.ndarray, which: int = SYSTEM) -> np.ndarray:
    return system.apply(x, which)


def VCycle(system: System, x: np.ndarray, rhs: np.ndarray) -> np.ndarray:
    return system.vcycle(x, rhs)


def texture_filtering_rhs(system: System, f: np.ndarray, stiffness: float, sharpness: float) -> np.ndarray:
    """``M f + stiffness * sharpness * S f`` (TextureFiltering.cpp:693-700), formed
    on the device from one upload of ``f``."""
    x, k = system._vec(f, np.float64)
    y = np.empty_like(x)
    _lib.check(_lib.lib().gdtp_apply_mass_stiffness(system.handle, 1.0, float(stiffness) * float(sharpness), _lib.ptr(x), _lib.ptr(y), k))
    return y


def texel_signal(hierarchy: Hierarchy, texture: np.ndarray) -> np.ndarray:
    """Texture value of every active texel, in texel order (TextureFiltering.cpp:603-608)."""
    tex = texture if texture.dtype in (np.float32, np.float64) else texture.astype(np.float64)
    height, width = tex.shape[:2]
    channels = 1 if tex.ndim == 2 else int(tex.shape[2])
    strides = (tex.strides[0], tex.strides[1], tex.strides[2] if tex.ndim == 3 else 0)
    out = np.empty((hierarchy.counts(0)["numTexels"], channels), dtype=np.float64)
    _lib.check(_lib.lib().gdtp_texel_signal(hierarchy.handle, C.c_void_p(tex.ctypes.data), int(width), int(height), channels,
                                            tex.itemsize, *strides, _lib.ptr(out)))
    return out if tex.ndim == 3 else out[:, 0]
