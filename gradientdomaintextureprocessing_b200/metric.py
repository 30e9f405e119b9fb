"""Per-triangle parameter metrics (host), the input of ``System(parameter_metric=...)``.

Names follow the reference:

* ``InitializeMetric(mesh, mode)``: embedding (``EMBEDDING_METRIC``) or uniform
  (``UNIFORM_METRIC``) metric pulled back to texture space
  (``include/Src/Metric.inl:448-466``).
* ``InitializeAnisotropicMetric(mesh, vf, across, isotropic)``: the
  line-integral-convolution metric of a tangent field
  (``include/Src/Metric.inl:468-486`` with a given field, i.e.
  ``InitializeVectorFieldMetric`` :12-67 then ``InitializeParameterMetric``
  :415-446).  ``vf`` is (nt, 2): the field on each triangle in the basis of its
  edges (p1 - p0, p2 - p0), as in the reference's ``.vf`` files
  (``meshgen.read_vf``).  The reference fixes ``across = 0.1`` and
  ``isotropic = 1e-5``; the stiffness ratio across / along the field is
  ``(across + isotropic) / isotropic``.

Both return (nt, 4) float64: g(0,0), g(0,1), g(1,0), g(1,1) per mesh triangle
(the reference's column, row indexing).  Computed by ``libgdtp.so``.
"""
from __future__ import annotations

import numpy as np

from . import _lib

EMBEDDING_METRIC, UNIFORM_METRIC = 0, 1


def _mesh_args(mesh: dict):
    v = np.ascontiguousarray(mesh["vertices"], dtype=np.float64)
    t = np.ascontiguousarray(mesh["triangles"], dtype=np.int32)
    uv = np.ascontiguousarray(mesh["uv"], dtype=np.float64)
    return v, t, uv


def InitializeMetric(mesh: dict, mode: int = EMBEDDING_METRIC) -> np.ndarray:
    v, t, uv = _mesh_args(mesh)
    out = np.empty((len(t), 4))
    _lib.check(_lib.lib().gdtp_surface_metric(_lib.ptr(v), len(v), _lib.ptr(t), len(t), _lib.ptr(uv), int(mode),
                                              _lib.ptr(out)))
    return out


def InitializeAnisotropicMetric(mesh: dict, vf: np.ndarray, across: float = 0.1, isotropic: float = 1e-5) -> np.ndarray:
    v, t, uv = _mesh_args(mesh)
    vf = np.ascontiguousarray(vf, dtype=np.float64).reshape(-1, 2)
    if len(vf) != len(t):
        raise ValueError(f"field has {len(vf)} vectors, mesh has {len(t)} triangles")
    out = np.empty((len(t), 4))
    _lib.check(_lib.lib().gdtp_anisotropic_metric(_lib.ptr(v), len(v), _lib.ptr(t), len(t), _lib.ptr(uv), _lib.ptr(vf),
                                                  float(across), float(isotropic), _lib.ptr(out)))
    return out


def across_for_ratio(ratio: float, isotropic: float = 1e-5) -> float:
    """``across`` that gives a stiffness ratio ``ratio`` between across and along the field."""
    return (ratio - 1.0) * isotropic
