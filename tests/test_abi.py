"""The C ABI library builds, loads without a GPU and exports every entry point of include/gdtp.h."""
import os
import re

from conftest import ROOT


def header_functions():
    src = open(os.path.join(ROOT, "include", "gdtp.h")).read()
    return sorted(set(re.findall(r"\b(gdtp_[a-z0-9_]+)\s*\(", src)))


def test_header_lists_entry_points():
    fns = header_functions()
    assert "gdtp_hierarchy_build" in fns and "gdtp_solve" in fns and len(fns) >= 20


def test_library_exports_every_declared_symbol(built_lib):
    from gradientdomaintextureprocessing_b200 import _lib
    L = _lib.lib()
    assert L.gdtp_missing_symbols == []
    for name in header_functions():
        assert hasattr(L, name), name
    assert L.gdtp_version() == 1


def test_errors_are_reported_not_raised(built_lib):
    import ctypes as C
    from gradientdomaintextureprocessing_b200 import _lib
    L = _lib.lib()
    h = C.c_void_p()
    code = L.gdtp_hierarchy_build(None, 0, None, 0, None, 0, 0, 0, None, C.byref(h))
    assert code == -1 and b"invalid" in L.gdtp_last_error()
