"""Host set-up on the reference's own meshes, from the reference's own operator.

Galerkin coarsening (csrc/setup/galerkin.cpp):
the reference's fine operator M + 1e-3 S of Julius and Bunny (256 x 256 after the
filtering app's preprocessing), from the unmodified reference (oracle/_ref/
gdtp_ref), is coarsened by the library's code (tests/native/galerkin_check.cpp)
and every level's deep stencils, BB and BD blocks are compared with the
reference's UpdateLinearSystem hierarchy (UpdateCoefficients.inl:285-399) to
1e-12 of each block's largest entry (measured ~1e-15).

Exact boundary-block solve (csrc/setup/bsolve.cpp): built from the reference's
boundary block of every level below the coarsest and applied on the host in the
kernels' sequence (tests/native/bsolve_check.cpp); the solution agrees with a
direct sparse solve to 1e-10 (measured 1e-16 to 1e-13).

Needs the reference's data directory and the built oracle (skipped otherwise);
no GPU.
"""
import os
import struct
import subprocess
import sys

import numpy as np
import pytest
import scipy.sparse as sp

from conftest import GOLDEN, ROOT, reference_data

REFERENCE_DATA = reference_data()
REF = os.path.join(ROOT, "oracle", "_ref", "gdtp_ref")
LEVELS, LAMBDA = 4, 1e-3

pytestmark = pytest.mark.skipif(not (os.path.isdir(REFERENCE_DATA) and os.path.exists(REF)),
                                reason="the reference's data files or the built oracle are not present")


def _csr(g, name):
    return sp.csr_matrix((g[name + "/val"], g[name + "/col"], g[name + "/ptr"]))


def _write_csr(f, m, cols):
    m = m.tocsr()
    m.sort_indices()
    f.write(struct.pack("<qqq", m.shape[0], cols, m.nnz))
    f.write(m.indptr.astype("<i4").tobytes() + m.indices.astype("<i4").tobytes() + m.data.astype("<f8").tobytes())


def _read_csr(b, o):
    rows, cols, nnz = struct.unpack_from("<qqq", b, o)
    o += 24
    ptr = np.frombuffer(b, "<i4", rows + 1, o)
    o += 4 * (rows + 1)
    col = np.frombuffer(b, "<i4", nnz, o)
    o += 4 * nnz
    val = np.frombuffer(b, "<f8", nnz, o)
    return sp.csr_matrix((val, col, ptr), shape=(rows, cols)), o + 8 * nnz


def _rel(a, b):
    n = max(a.shape[1], b.shape[1])
    a, b = a.copy(), b.copy()
    a.resize((a.shape[0], n))
    b.resize((b.shape[0], n))
    assert a.shape == b.shape
    return abs(a - b).max() / max(abs(b).max(), 1e-300)


def _native(tmp_path, name):
    pkg = os.path.join(ROOT, "gradientdomaintextureprocessing_b200")
    exe = str(tmp_path / name)
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", os.path.join(pkg, "csrc"), "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "native", name + ".cpp"), "-L", pkg, "-lgdtp", "-Wl,-rpath," + pkg, "-o", exe],
                   check=True)
    return exe


@pytest.fixture(scope="module", params=["Julius/julius.ply", "Bunny/bunny.ply"])
def reference_case(request, built_lib, tmp_path_factory):
    """The mesh after the app's preprocessing and the reference's dump of it."""
    import gdd
    sys.path.insert(0, GOLDEN)
    import make_real_golden as mk
    from gradientdomaintextureprocessing_b200 import meshgen
    mesh, _, w, h = mk.prepared(os.path.dirname(REFERENCE_DATA), request.param)
    mesh["texture"] = np.zeros((h, w, 3), np.float32)
    tmp = tmp_path_factory.mktemp("ref")
    gdm, dump = str(tmp / "m.gdm"), str(tmp / "m.gdd")
    meshgen.write_gdm(gdm, mesh)
    subprocess.run([REF, gdm, dump, str(LEVELS), str(LAMBDA), "2.0", "2", "dump"], check=True, capture_output=True, timeout=600)
    return gdm, gdd.read_dump(dump)


def test_galerkin_hierarchy_matches_reference(reference_case, tmp_path):
    import port
    gdm, g = reference_case
    nt, nb = int(g["L0/counts"][0]), int(g["L0/counts"][2])
    deep0 = g["fine/deepMass"].ravel() + LAMBDA * g["fine/deepStiffness"].ravel()
    fine = tmp_path / "fine.bin"
    with open(fine, "wb") as f:
        f.write(struct.pack("<q", len(deep0)) + deep0.astype("<f8").tobytes())
        _write_csr(f, _csr(g, "fine/BBmass") + LAMBDA * _csr(g, "fine/BBstiffness"), nb)
        _write_csr(f, _csr(g, "fine/BDmass") + LAMBDA * _csr(g, "fine/BDstiffness"), nt)
    exe = _native(tmp_path, "galerkin_check")
    out = tmp_path / "out.bin"
    r = subprocess.run([exe, gdm, str(LEVELS), str(fine), str(out)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    b, o = out.read_bytes(), 0
    for l in range(LEVELS):
        (m,) = struct.unpack_from("<q", b, o)
        deep = np.frombuffer(b, "<f8", m, o + 8).reshape(-1, 10)
        o += 8 + 8 * m
        bb, o = _read_csr(b, o)
        bd, o = _read_csr(b, o)
        ref = g[f"L{l}/coef/deep"]
        # the reference keeps its levels above the coarsest in reciprocal form
        mine, cols = (port.reciprocal_form(deep), 10) if l < LEVELS - 1 else (deep, 9)
        assert np.abs(mine[:, :cols] - ref[:, :cols]).max() <= 1e-12 * np.abs(ref[:, :cols]).max(), l
        assert _rel(bb, _csr(g, f"L{l}/coef/BB")) <= 1e-12, l
        assert _rel(bd, _csr(g, f"L{l}/coef/BD")) <= 1e-12, l


def test_boundary_solve_on_reference_blocks(reference_case, tmp_path):
    from scipy.sparse.linalg import spsolve
    _, g = reference_case
    exe = _native(tmp_path, "bsolve_check")
    for l in range(LEVELS - 1):
        BB = _csr(g, f"L{l}/coef/BB").tocsr()
        BB.sort_indices()
        n = BB.shape[0]
        r = np.random.default_rng(l).normal(size=n)
        inp, out = tmp_path / "in.bin", tmp_path / "out.bin"
        with open(inp, "wb") as f:
            _write_csr(f, BB, n)
            f.write(struct.pack("<q", n) + r.astype("<f8").tobytes())
        p = subprocess.run([exe, str(inp), str(out)], capture_output=True, text=True, timeout=600)
        assert p.returncode == 0, p.stdout + p.stderr
        x = np.fromfile(out, "<f8")
        xd = spsolve(BB.tocsc(), r)
        assert np.linalg.norm(x - xd) <= 1e-10 * np.linalg.norm(xd), (l, p.stdout)


def test_coarsest_level_operator_and_inverse(reference_case, tmp_path):
    """The coarsest level: the full operator that full_matrix assembles from the
    reference's coarsest coefficients equals the oracle port's assembly of them
    (oracle/port.py full_matrix), and its Jacobi-scaled dense inverse solves it
    to 1e-10 of a direct sparse solve."""
    import port
    from scipy.sparse.linalg import spsolve
    gdm, g = reference_case
    exe = _native(tmp_path, "coarse_check")
    l = LEVELS - 1
    deep = np.ascontiguousarray(g[f"L{l}/coef/deep"], np.float64)
    nb, nt = int(g[f"L{l}/counts"][2]), int(g[f"L{l}/counts"][0])
    BB, BD = _csr(g, f"L{l}/coef/BB"), _csr(g, f"L{l}/coef/BD")
    r = np.random.default_rng(5).normal(size=nt)
    inp, out = tmp_path / "in.bin", tmp_path / "out.bin"
    with open(inp, "wb") as f:
        f.write(struct.pack("<q", deep.size) + deep.astype("<f8").tobytes())
        _write_csr(f, BB, nb)
        _write_csr(f, BD, nt)
        f.write(struct.pack("<q", nt) + r.astype("<f8").tobytes())
    p = subprocess.run([exe, gdm, str(LEVELS), str(inp), str(out)], capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stdout + p.stderr
    b = out.read_bytes()
    full, o = _read_csr(b, 0)
    x = np.frombuffer(b, "<f8", nt, o)
    ref = port.full_matrix(g[f"L{l}/nodeinfo"], g[f"L{l}/deepGlobalIndex"], g[f"L{l}/boundaryGlobalIndex"], deep,
                           _csr(g, f"L{l}/coef/BB"), _csr(g, f"L{l}/coef/BD"))
    assert _rel(full, ref.tocsr()) <= 1e-15
    xd = spsolve(ref.tocsc(), r)
    assert np.linalg.norm(x - xd) <= 1e-10 * np.linalg.norm(xd)
