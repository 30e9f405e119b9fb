"""The drop-in boundary: the TextureFiltering app's solve path, written against
the reference's headers and types and compiled unchanged, runs on the device
when this repository's include/ comes first on the include path.

tests/native/dropin_replay.cpp replays TextureFilter::InitializeSystem and
UpdateSolution (TextureFiltering/TextureFiltering.cpp:581-718, 562-579) call for
call: InitializeHierarchy, InitializeBoundaryProlongationData, InitializeMetric,
InitializeMassAndStiffness, InitializeInteriorTexelToCellLines,
UpdateLinearSystem, two MultiplyBySystemMatrix_NoReciprocals for the right-hand
side, then VCycle per UpdateSolution.  oracle/Makefile builds it twice:
dropin_replay_ref (the reference alone, CPU) and dropin_replay_gdtp (the Src/
wrappers of include/ forward UpdateLinearSystem, VCycle and the operator
products to libgdtp).  Both run the same seeded fixture; checked:

* the right-hand side built through the forwarded FP64 operator equals the
  reference's to 2e-6 of its largest entry (the boundary-block difference of
  the seam-node jitter, as in test_gpu_solver);
* one forwarded V-cycle leaves at most 3x the relative residual of the
  reference's own first V-cycle (the device V-cycle's 4-colour smoother
  contracts less per cycle than the reference's lexicographic block
  Gauss-Seidel: 0.50 -> 8.3e-3 against 5.3e-3 on the torus, 0.50 -> 5.5e-4
  against 2.4e-4 on the icosphere);
* after 30 V-cycles (the app's FP32 vectors, Vec4f) the energy-norm error
  against the reference's FP64 direct solution is below 1e-5 (measured 1.5e-7
  and 8.6e-6; the reference's own 30 V-cycles: 2.5e-7 and 1.6e-6, each
  iteration stalling at its FP32 rounding).
"""
import os
import subprocess
import tempfile

import numpy as np
import pytest

from conftest import ROOT, golden_mesh, load_golden

pytestmark = pytest.mark.gpu

REF = os.path.join(ROOT, "oracle", "_ref", "dropin_replay_ref")
GDTP = os.path.join(ROOT, "oracle", "_ref", "dropin_replay_gdtp")
VCYCLES = 30


def replay(exe, gdm, g):
    lam, sharp = (float(v) for v in g["meta/weights"])
    with tempfile.TemporaryDirectory() as tmp:
        out = os.path.join(tmp, "out.bin")
        r = subprocess.run([exe, gdm, out, str(int(g["meta/size"][2])), repr(lam), repr(sharp), str(VCYCLES)], capture_output=True,
                           text=True, timeout=600)
        assert r.returncode == 0 and "replay ok" in r.stdout, r.stdout + r.stderr
        raw = open(out, "rb").read()
    n = int(np.frombuffer(raw[:8], dtype=np.int64)[0])
    a = np.frombuffer(raw[8:], dtype=np.float64).reshape(3, n, 3)
    return a[0], a[1], a[2]


@pytest.fixture(scope="module", params=["torus128", "ico256"])
def runs(request, built_lib):
    from gradientdomaintextureprocessing_b200 import meshgen
    from test_gpu_solver import ref_full
    if not (os.path.exists(REF) and os.path.exists(GDTP)):
        pytest.skip("drop-in replay binaries are not built (oracle/Makefile, needs the reference checkout)")
    g = load_golden(request.param)
    with tempfile.TemporaryDirectory() as tmp:
        gdm = os.path.join(tmp, "mesh.gdm")
        meshgen.write_gdm(gdm, golden_mesh(g))
        ref = replay(REF, gdm, g)
        dev = replay(GDTP, gdm, g)
    return g, ref_full(g), ref, dev


def test_rhs_through_forwarded_operator(runs):
    g, _, ref, dev = runs
    assert np.abs(dev[0] - ref[0]).max() <= 2e-6 * np.abs(ref[0]).max()


def test_forwarded_vcycle_contracts(runs):
    import port
    g, A, ref, dev = runs
    x0 = g["solve/f"]
    r0 = port.relative_residual(A, ref[0], x0).max()
    r_ref = port.relative_residual(A, ref[0], ref[1]).max()
    r_dev = port.relative_residual(A, dev[0], dev[1]).max()
    print(f"{g['meta/size'][:2]}: first V-cycle relative residual {r0:.2e} -> drop-in {r_dev:.2e}, reference {r_ref:.2e}")
    assert r_dev <= 3 * r_ref, (r0, r_ref, r_dev)


def test_converged_solution_matches_reference(runs):
    import port
    g, A, ref, dev = runs
    exact = g["solve/exact"]
    e_ref = port.energy_error(A, ref[2], exact).max()
    e_dev = port.energy_error(A, dev[2], exact).max()
    print(f"{g['meta/size'][:2]}: energy error after {VCYCLES} V-cycles: drop-in {e_dev:.2e}, reference {e_ref:.2e}")
    assert e_dev < 1e-5, (e_dev, e_ref)
