"""Heat-method geodesic distances on the texel grid (the Geodesics app).

Mirrors ``Geodesics/Geodesics.cpp``: an impulse at each source texel is smoothed
with ``(M + t S) u = delta`` (:552-560, stiffness weight t), the unit field
``X = -grad u / |grad u|`` is integrated against the texel basis
(``IntergrateNormalizedVectorFieldFromSamples``,
``include/Src/VectorFieldIntergration.inl:453-582``) and the distance solves
``(eps M + S) d = rhs`` with ``eps = 1e-6`` (:632-650), shifted to 0 at the
source (:536-547).  Sources are right-hand sides: ``k`` sources run as one
batched solve of each system.  Everything runs in ``libgdtp.so`` on the device.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .hierarchy import Hierarchy
from .system import System


# the Geodesics app's --stiffness default (Geodesics/Geodesics.cpp:19)
DEFAULT_SMOOTHING = 1e-3


def mean_texel_area(hierarchy: Hierarchy) -> float:
    """Mean texel area of the finest level in the area-normalised metric (total area 1).

    As a smoothing time it makes the impulse response decay like exp(-d / h):
    beyond a few tens of texels it falls below what any solve to a relative
    residual of 1e-6 resolves, and the normalised field there is noise.  The
    app's default (``DEFAULT_SMOOTHING``) keeps the response resolved."""
    return 1.0 / hierarchy.counts(0)["numTexels"]


class Geodesics:
    def __init__(self, hierarchy: Hierarchy, smoothing: float = DEFAULT_SMOOTHING, epsilon: float = 1e-6, device: int = 0,
                 parameter_metric: np.ndarray | None = None):
        self.hierarchy = hierarchy
        self.t = float(smoothing)
        self.smooth = System(hierarchy, device=device, parameter_metric=parameter_metric)
        self.smooth.update(self.t, 1.0)
        self.dist = System(hierarchy, device=device, parameter_metric=parameter_metric)
        self.dist.update(1.0, float(epsilon))
        self.n = self.smooth.n
        g = C.c_void_p()
        _lib.check(_lib.lib().gdtp_geodesics_create(self.smooth.handle, C.byref(g)))
        self._g = g

    def __del__(self):
        g, self._g = getattr(self, "_g", None), None
        if g:
            try:
                _lib.lib().gdtp_geodesics_free(g)
            except (TypeError, AttributeError):  # interpreter exit: module globals already cleared
                pass

    def counts(self) -> dict:
        c = np.zeros(2, dtype=np.int64)
        _lib.check(_lib.lib().gdtp_geodesics_counts(self._g, _lib.ptr(c)))
        return {"cell_samples": int(c[0]), "boundary_samples": int(c[1])}

    def array(self, name: str) -> np.ndarray:
        n = C.c_int64()
        L = _lib.lib()
        _lib.check(L.gdtp_geodesics_array(self._g, name.encode(), None, C.byref(n)))
        out = np.empty(n.value)
        _lib.check(L.gdtp_geodesics_array(self._g, name.encode(), _lib.ptr(out), C.byref(n)))
        width = {"cellSamples": 16, "hexSamples": 20, "corners": 4, "btIdx": 6}.get(name)
        return out.reshape(-1, width) if width else out

    def rhs(self, potential: np.ndarray) -> np.ndarray:
        """Integrated normalised field of ``potential`` (n or n x k), the Poisson right-hand side."""
        u = np.ascontiguousarray(potential, dtype=np.float64)
        squeeze = u.ndim == 1
        u = u.reshape(self.n, -1)
        out = np.empty_like(u)
        _lib.check(_lib.lib().gdtp_geodesic_rhs(self._g, _lib.ptr(u), _lib.ptr(out), u.shape[1]))
        return out[:, 0] if squeeze else out

    def distance(self, sources, tol: float = 1e-6, max_iters: int = 200):
        """Distances (n x k) from k source texels, and the solve report."""
        src = np.ascontiguousarray(np.atleast_1d(sources), dtype=np.int32)
        out = np.empty((self.n, len(src)))
        rep = _lib.Report()
        code = _lib.lib().gdtp_geodesic_distance(self._g, self.smooth.handle, self.dist.handle, _lib.ptr(src), len(src), float(tol),
                                                 int(max_iters), _lib.ptr(out), C.byref(rep))
        _lib.check(code)
        return out, {"iterations": rep.iterations, "vcycles": rep.vcycles, "rel_residual_max": rep.rel_residual_max,
                     "seconds": rep.seconds}
