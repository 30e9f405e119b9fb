"""The benchmark configurations at their own sizes, solved on the device and
compared with the reference's FP64 solution of the same problem.

The ground truth is computed on the spot by the compiled reference
(oracle/_ref/gdtp_ref, the reference's solve path built from its unmodified
headers; oracle/reference_solution.py): from the seeded generator's mesh and
texture (and, for the LIC case, the parameter metric) it builds its own
hierarchy, assembles its FP64 operator and the TextureFiltering right-hand
side, and iterates its FP64 V-cycle to a relative residual of 1e-12 or its
floating-point floor.  The device then solves the reference's right-hand side
and every case checks

* operator parity at full size: ||(A - A_ref) x_ref|| / ||A_ref x_ref|| <= 2e-6
  (the device's FP64 operator against the reference's, on the reference's
  solution).  The two differ where the reference moves the seam nodes it
  inserts by a rand()-driven 1e-10 relative offset before its Delaunay step
  (BoundaryQuadraticElements.inl:433-436); the device keeps them on the seam;
  measured 4e-7 to 9e-7 (icosphere 2048^2), 1.2e-6 (genus-2 4096^2);
* the relative residual against the device's FP64 operator (<= tol) and
  against the reference's (<= tol + 1.5 x that operator difference);
* the error against the reference's solution in the reference operator's
  energy norm, ||x - x_ref||_A / ||x_ref||_A per right-hand side, below
  max(1e-5, 50 tol).  At 2048^2 the energy error of any iterate is about 20x
  its relative residual: the reference's own FP64 V-cycle iterate at residual
  2.6e-6 on icosphere 2048^2 has energy error 5.4e-5.  So the 1e-5 bar holds
  from tol 1e-8 down (measured 8e-7 on the icosphere, the operator difference
  above being its floor), and at tol 1e-6 the bar is 5e-5 (measured 2.6e-5).
  Texels whose support barely meets a chart have tiny diagonals and are not
  pinned by the residual; the energy norm weighs them by their support.

Cases:
* torus256: torus R=1, r=0.4, 64x32 quads, 4 charts, 256^2 RGB uint8 noise,
  M + 1e-3 S, rhs M f + 2e-3 S f; plain FP64 V-cycles and mixed precision,
  both to 1e-8;
* icosphere2048: icosphere(6) jittered, 16 latitude/longitude charts,
  2048^2 RGB value noise; same operator; mixed precision to 1e-6, 3
  right-hand sides (the benchmark's workload); and the plain FP64 V-cycle;
* genus2lic4096: genus-2 surface (two blended tori, 32 charts), 4096^2
  single-channel noise, anisotropic metric of stiffness ratio 1e3 along the
  90-degree-rotated gradient of 8 seeded Gaussians, M + 1e-4 S, rhs M f, one
  right-hand side, flexible CG around the FP32 V-cycle to 1e-6 and 1e-8.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _torus():
    from gradientdomaintextureprocessing_b200 import meshgen
    return meshgen.torus_atlas(256, 256), None


def _icosphere():
    from gradientdomaintextureprocessing_b200 import meshgen
    return meshgen.icosphere_atlas(2048, 2048, subdiv=6, seed=0), None


def _genus2_lic():
    from gradientdomaintextureprocessing_b200 import meshgen
    from gradientdomaintextureprocessing_b200.metric import InitializeAnisotropicMetric, across_for_ratio
    mesh = meshgen.genus2_atlas(4096, 4096)
    field = meshgen.gaussian_bump_field(mesh, bumps=8, seed=0)
    return mesh, InitializeAnisotropicMetric(mesh, field, across=across_for_ratio(1e3))


# name: (mesh and metric, levels, stiffness, sharpness, right-hand sides solved, [(precision, tol)] x 2, krylov)
CASES = {
    "torus256": (_torus, 4, 1e-3, 2.0, 3, [("fp64", 1e-8), ("mixed", 1e-8)], 0),
    "icosphere2048": (_icosphere, 4, 1e-3, 2.0, 3, [("mixed", 1e-6), ("fp64", 1e-6)], 0),
    "genus2lic4096": (_genus2_lic, 4, 1e-4, 0.0, 1, [("mixed", 1e-6), ("mixed", 1e-8)], 1),
}


@pytest.fixture(scope="module", params=sorted(CASES))
def config(request, built_lib):
    """One configuration at a time (pytest runs every test of one parameter
    before building the next; the largest hold a few GB on the host)."""
    import reference_solution as rs
    from gradientdomaintextureprocessing_b200.hierarchy import InitializeHierarchy
    from gradientdomaintextureprocessing_b200.system import System
    if not rs.available():
        pytest.skip("oracle/_ref/gdtp_ref is not built")
    name = request.param
    make, levels, stiffness, sharpness, _, _, krylov = CASES[name]
    mesh, pm = make()
    ref = rs.reference_solution(mesh, levels, stiffness, sharpness, tol=1e-12, parameter_metric=pm)
    h = InitializeHierarchy(mesh, levels=levels)
    s = System(h, parameter_metric=pm)
    s.update(stiffness, 1.0)
    s.set("krylov", krylov)
    return name, mesh, ref, h, s


def test_reference_ground_truth_converged(config):
    _, _, ref, h, _ = config
    # the reference's FP64 V-cycle reached 1e-12 or its floating-point floor (the
    # anisotropic LIC system stalls near 1.3e-11 after ~550 V-cycles)
    assert ref["history"][-1] <= 2e-11, ref["history"][-5:]
    # same texel grid on both sides (the hierarchy is bit-exact)
    assert int(ref["counts"][0]) == h.counts(0)["numTexels"]


def test_operator_matches_reference(config):
    from gradientdomaintextureprocessing_b200.system import SYSTEM
    _, _, ref, _, s = config
    xs = np.ascontiguousarray(ref["x"])
    ax_ref = ref["A"] @ xs
    floor = np.linalg.norm(s.apply(xs, SYSTEM) - ax_ref, axis=0) / np.linalg.norm(ax_ref, axis=0)
    assert floor.max() <= 2e-6, floor


def test_rhs_matches_reference(config):
    from gradientdomaintextureprocessing_b200.system import texel_signal, texture_filtering_rhs
    name, mesh, ref, h, s = config
    _, _, stiffness, sharpness, _, _, _ = CASES[name]
    f = texel_signal(h, mesh["texture"])
    if f.shape[1] == 1:  # single-channel texture: the harness replicates it into RGB
        f = np.repeat(f, 3, axis=1)
    b = texture_filtering_rhs(s, f, stiffness, sharpness)
    assert np.abs(b - ref["rhs"]).max() <= 2e-6 * np.abs(ref["rhs"]).max()


@pytest.mark.parametrize("which", [0, 1])
def test_solution_matches_reference(config, which):
    import reference_solution as rs
    name, _, ref, _, s = config
    k = CASES[name][4]
    precision, tol = CASES[name][5][which]
    b = np.ascontiguousarray(ref["rhs"][:, :k])
    from gradientdomaintextureprocessing_b200.system import SYSTEM
    x, rep = s.solve(b, tol=tol, precision=precision, max_iters=400)
    assert rep["converged"] and rep["rel_residual_max"] <= tol, rep
    assert s.residual(b, x).max() <= tol
    xs = np.ascontiguousarray(ref["x"][:, :k])
    floor = (np.linalg.norm(s.apply(xs, SYSTEM) - ref["A"] @ xs, axis=0) / np.linalg.norm(b, axis=0)).max()
    res_ref = rs.relative_residual(ref["A"], b, x).max()
    err = rs.energy_error(ref["A"], x, xs)
    print(f"{name} {precision} tol {tol:g}: energy error vs the reference's FP64 solution {err.max():.3e}, residual with the "
          f"reference's operator {res_ref:.3e} (operator difference {floor:.2e}), {rep['iterations']} steps / {rep['vcycles']} V-cycles")
    assert res_ref <= tol + 1.5 * floor
    assert err.max() < max(1e-5, 50 * tol), err
