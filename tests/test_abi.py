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


def test_solve_entry_points_reject_a_null_system(built_lib):
    """Every solve entry point checks its handle before touching the device (no GPU needed)."""
    import ctypes as C
    from gradientdomaintextureprocessing_b200 import _lib
    L = _lib.lib()
    rep = _lib.Report()
    b = (C.c_double * 4)()
    x = (C.c_double * 4)()
    bp = (C.c_void_p * 1)(C.cast(b, C.c_void_p))
    xp = (C.c_void_p * 1)(C.cast(x, C.c_void_p))
    assert L.gdtp_solve(None, b, x, 1, 1e-6, 10, C.byref(rep)) == -1
    assert L.gdtp_solve_ex(None, b, x, 1, 1e-6, 10, 1, C.byref(rep)) == -1
    assert L.gdtp_solve_stream(None, bp, xp, 1, 1, 1e-6, 10, None) == -1
    assert b"null system handle" in L.gdtp_last_error()


_NULL_CALLS = r'''
import ctypes as C, sys
sys.path.insert(0, sys.argv[1])
from gradientdomaintextureprocessing_b200 import _lib
L = _lib.lib()
for name, (res, args) in _lib._SIGS.items():
    if name in ("gdtp_last_error", "gdtp_version"):
        continue
    vals = [0 if a in (C.c_int, C.c_int64) else 1e-6 if a is C.c_double else None for a in args]
    print(name, flush=True)
    r = getattr(L, name)(*vals)
    print("=", r, flush=True)
'''


def test_every_entry_point_rejects_null_and_zero_arguments(built_lib):
    """Each entry point, called with null pointers and zero sizes, returns an
    error (or, for the free / count functions, does nothing) instead of
    crashing; run in a child process so that a crash names the entry point."""
    import subprocess
    import sys
    from conftest import ROOT
    p = subprocess.run([sys.executable, "-c", _NULL_CALLS, ROOT], capture_output=True, text=True, timeout=300)
    lines = p.stdout.split("\n")
    assert p.returncode == 0, f"crashed after: {lines[-3:]} {p.stderr[-300:]}"
    results = dict(zip(lines[0::2], lines[1::2]))
    assert len(results) >= 40
    for name, r in results.items():
        ok = {"= None", "= 0"} if name.endswith(("_free", "_levels", "_charts")) else {"= -1"}
        assert r in ok, (name, r)


def test_entry_point_exceptions_become_error_codes(built_lib):
    """guarded() (the wrapper of every C entry point's body) turns host
    allocation failures and other C++ exceptions into error codes."""
    import os
    import subprocess
    import tempfile
    from conftest import ROOT
    pkg = os.path.join(ROOT, "gradientdomaintextureprocessing_b200")
    with tempfile.TemporaryDirectory() as tmp:
        exe = os.path.join(tmp, "guard_check")
        subprocess.run(["g++", "-std=c++17", "-O2", "-I", os.path.join(pkg, "csrc"), "-I", os.path.join(ROOT, "include"),
                        os.path.join(ROOT, "tests", "native", "guard_check.cpp"), "-L", pkg, "-lgdtp", "-Wl,-rpath," + pkg,
                        "-o", exe], check=True)
        out = subprocess.run([exe], capture_output=True, text=True, timeout=60)
        assert out.returncode == 0 and out.stdout.strip() == "ok", out.stdout + out.stderr
