"""ctypes binding of the C ABI declared in include/gdtp.h.

The shared library is built in-tree (``libgdtp.so`` next to this file) by
``gradientdomaintextureprocessing_b200.build``.  Nothing here falls back to
Python: a missing library or a failing call raises ``GDTPError``.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("GDTP_LIB", os.path.join(_HERE, "libgdtp.so"))

GDTP_OK = 0
_ERRORS = {-1: "invalid argument", -2: "setup failed", -3: "CUDA error", -4: "not converged", -5: "HBM budget exceeded",
           -6: "call out of order", -7: "numerical failure"}


class GDTPError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"gdtp error {code} ({_ERRORS.get(code, '?')}): {msg}")
        self.code = code


class Report(C.Structure):
    _fields_ = [("iterations", C.c_int), ("vcycles", C.c_int), ("rel_residual_max", C.c_double), ("seconds", C.c_double)]


_lib = None

_P = C.c_void_p
_SIGS = {
    "gdtp_last_error": (C.c_char_p, []),
    "gdtp_version": (C.c_int, []),
    "gdtp_hierarchy_build": (C.c_int, [_P, C.c_int64, _P, C.c_int64, _P, C.c_int, C.c_int, C.c_int, _P, C.POINTER(_P)]),
    "gdtp_hierarchy_free": (None, [_P]),
    "gdtp_hierarchy_levels": (C.c_int, [_P]),
    "gdtp_hierarchy_charts": (C.c_int, [_P]),
    "gdtp_hierarchy_counts": (C.c_int, [_P, C.c_int, _P]),
    "gdtp_hierarchy_array": (C.c_int, [_P, C.c_char_p, C.c_int, _P, C.POINTER(C.c_int64)]),
    "gdtp_surface_metric": (C.c_int, [_P, C.c_int64, _P, C.c_int64, _P, C.c_int, _P]),
    "gdtp_anisotropic_metric": (C.c_int, [_P, C.c_int64, _P, C.c_int64, _P, _P, C.c_double, C.c_double, _P]),
    "gdtp_system_create": (C.c_int, [_P, C.c_int, C.c_int, _P, _P, C.c_int64, C.POINTER(_P)]),
    "gdtp_system_free": (None, [_P]),
    "gdtp_system_array": (C.c_int, [_P, C.c_char_p, C.c_int, _P, C.POINTER(C.c_int64)]),
    "gdtp_apply_mass_stiffness": (C.c_int, [_P, C.c_double, C.c_double, _P, _P, C.c_int]),
    "gdtp_texel_signal": (C.c_int, [_P, _P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int64, C.c_int64, C.c_int64, _P]),
    "gdtp_system_update": (C.c_int, [_P, C.c_double, C.c_double]),
    "gdtp_apply": (C.c_int, [_P, C.c_int, _P, _P, C.c_int]),
    "gdtp_vcycle": (C.c_int, [_P, _P, _P, C.c_int]),
    "gdtp_vcycle64": (C.c_int, [_P, _P, _P, C.c_int]),
    "gdtp_brush_create": (C.c_int, [_P, _P, C.c_int, C.POINTER(_P)]),
    "gdtp_brush_free": (None, [_P]),
    "gdtp_brush_apply": (C.c_int, [_P, _P, _P]),
    "gdtp_brush_apply_device": (C.c_int, [_P, _P, _P, _P]),
    "gdtp_relax": (C.c_int, [_P, _P, _P, C.c_int, C.c_int, C.c_int]),
    "gdtp_solve": (C.c_int, [_P, _P, _P, C.c_int, C.c_double, C.c_int, C.POINTER(Report)]),
    "gdtp_solve_ex": (C.c_int, [_P, _P, _P, C.c_int, C.c_double, C.c_int, C.c_int, C.POINTER(Report)]),
    "gdtp_solve_stream": (C.c_int, [_P, _P, _P, C.c_int, C.c_int, C.c_double, C.c_int, _P]),
    "gdtp_solve_device": (C.c_int, [_P, _P, _P, C.c_int, C.c_double, C.c_int, _P, C.POINTER(Report)]),
    "gdtp_solve_fp64": (C.c_int, [_P, _P, _P, C.c_int, C.c_double, C.c_int, C.POINTER(Report)]),
    "gdtp_solve_fp64_device": (C.c_int, [_P, _P, _P, C.c_int, C.c_double, C.c_int, _P, C.POINTER(Report)]),
    "gdtp_residual": (C.c_int, [_P, _P, _P, C.c_int, _P]),
    "gdtp_system_set": (C.c_int, [_P, C.c_char_p, C.c_double]),
    "gdtp_system_get": (C.c_int, [_P, C.c_char_p, C.POINTER(C.c_double)]),
    "gdtp_system_autotune": (C.c_int, [_P, _P, C.c_int, C.c_double, _P]),
    "gdtp_residual_static": (C.c_int, [_P, _P, _P, _P, C.c_int, _P, _P]),
    "gdtp_system_device_bytes": (C.c_int, [_P, C.POINTER(C.c_int64)]),
    "gdtp_read_textured_mesh": (C.c_int, [C.c_char_p, C.POINTER(C.c_int64), C.POINTER(C.c_int64), _P, _P, _P]),
    "gdtp_textured_mesh_texture_file": (C.c_int, [C.c_char_p, C.c_char_p, C.POINTER(C.c_int64)]),
    "gdtp_write_textured_mesh": (C.c_int, [C.c_char_p, _P, C.c_int64, _P, C.c_int64, _P, C.c_char_p]),
    "gdtp_read_image": (C.c_int, [C.c_char_p, C.POINTER(C.c_int), C.POINTER(C.c_int), _P]),
    "gdtp_write_image": (C.c_int, [C.c_char_p, _P, C.c_int, C.c_int]),
    "gdtp_read_vector": (C.c_int, [C.c_char_p, C.c_int64, C.POINTER(C.c_int64), _P]),
    "gdtp_write_vector": (C.c_int, [C.c_char_p, C.c_int64, C.c_int64, _P]),
    "gdtp_compute_padding": (C.c_int, [C.c_int, C.c_int, _P, C.c_int64, _P]),
    "gdtp_pad_texture_coordinates": (C.c_int, [_P, C.c_int, C.c_int, _P, C.c_int64, C.c_int]),
    "gdtp_pad_image": (C.c_int, [_P, _P, C.c_int, C.c_int, _P, C.c_int]),
    "gdtp_server_create": (C.c_int, [C.c_int, C.c_int64, C.c_int, C.POINTER(_P)]),
    "gdtp_server_free": (None, [_P]),
    "gdtp_server_add_model": (C.c_int, [_P, _P, C.c_int64, _P, C.c_int64, _P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double,
                                        C.c_double, _P, C.POINTER(C.c_int)]),
    "gdtp_server_model_texels": (C.c_int, [_P, C.c_int, C.POINTER(C.c_int64)]),
    "gdtp_server_model_bytes": (C.c_int, [_P, C.c_int, C.POINTER(C.c_int64)]),
    "gdtp_server_warm": (C.c_int, [_P, C.c_int]),
    "gdtp_server_submit": (C.c_int, [_P, C.c_int, _P, _P, C.c_int, C.c_double, C.c_int, C.POINTER(C.c_int64)]),
    "gdtp_server_poll": (C.c_int, [_P, C.c_int64, C.POINTER(C.c_int)]),
    "gdtp_server_wait": (C.c_int, [_P, C.c_int64, _P, C.POINTER(Report), _P]),
    "gdtp_server_stats": (C.c_int, [_P, _P]),
    "gdtp_geodesics_create": (C.c_int, [_P, C.POINTER(_P)]),
    "gdtp_geodesics_free": (None, [_P]),
    "gdtp_geodesics_counts": (C.c_int, [_P, _P]),
    "gdtp_geodesics_array": (C.c_int, [_P, C.c_char_p, _P, C.POINTER(C.c_int64)]),
    "gdtp_geodesic_rhs": (C.c_int, [_P, _P, _P, C.c_int]),
    "gdtp_geodesic_rhs_device": (C.c_int, [_P, _P, _P, C.c_int, _P]),
    "gdtp_geodesic_distance": (C.c_int, [_P, _P, _P, _P, C.c_int, C.c_double, C.c_int, _P, C.POINTER(Report)]),
}


def exported_symbols() -> list[str]:
    return list(_SIGS)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise GDTPError(-3, f"{LIB_PATH} not built; run gradientdomaintextureprocessing_b200.build")
        L = C.CDLL(LIB_PATH)
        missing = []
        for name, (res, args) in _SIGS.items():
            try:
                f = getattr(L, name)
            except AttributeError:
                missing.append(name)
                continue
            f.restype = res
            f.argtypes = args
        L.gdtp_missing_symbols = missing
        _lib = L
    return _lib


def check(code: int) -> None:
    if code != GDTP_OK:
        raise GDTPError(code, lib().gdtp_last_error().decode(errors="replace"))


def ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(C.c_void_p)
