"""The sharpening brush on the device (gdtp_brush_*) against the reference's own
CellStiffnessToTexelStiffness (IterativeSolvers.inl:1170-1208), computed by
the compiled reference (oracle/_ref/gdtp_ref, "brush" mode) from the
per-cell stiffness that its InitializeMassAndStiffness keeps with
computeCellBasedStiffness (MassAndStiffness.h:490-546), in FP64, for a seeded
cell mask m_c = ((c * 2654435761) mod 2^32 mod 1000) / 1000.

Tolerances: deep texels 1e-10 of the largest entry (the FP64 element matrices
agree to 1e-12); boundary texels 1e-6 of the largest entry (their rows hold the
quadratic boundary elements, where the reference moves its seam nodes by a
rand()-driven 1e-10 relative offset, BoundaryQuadraticElements.inl:433-436,
measured 6e-7 on the boundary stiffness block).  A uniform mask gives the
stiffness applied to the signal, S f, on both sides (1e-12 against the
device's own operator)."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

from conftest import ROOT, golden_mesh, load_golden

pytestmark = pytest.mark.gpu

HARNESS = os.path.join(ROOT, "oracle", "_ref", "gdtp_ref")


def seeded_mask(n: int) -> np.ndarray:
    c = np.arange(n, dtype=np.uint64)
    return ((c * np.uint64(2654435761)) % np.uint64(2 ** 32) % np.uint64(1000)).astype(np.float64) / 1000.0


@pytest.fixture(scope="module", params=["torus128", "ico256"])
def case(request, built_lib):
    import gdd
    from gradientdomaintextureprocessing_b200 import meshgen
    from gradientdomaintextureprocessing_b200.hierarchy import InitializeHierarchy
    from gradientdomaintextureprocessing_b200.system import Brush, System, texel_signal
    if not os.path.exists(HARNESS):
        pytest.skip("oracle/_ref/gdtp_ref is not built")
    g = load_golden(request.param)
    mesh = golden_mesh(g)
    with tempfile.TemporaryDirectory() as tmp:
        gdm, out = os.path.join(tmp, "mesh.gdm"), os.path.join(tmp, "brush.gdd")
        meshgen.write_gdm(gdm, mesh)
        subprocess.run([HARNESS, gdm, out, str(int(g["meta/size"][2])), "1e-3", "2", "0", "brush"], check=True, capture_output=True,
                       timeout=600)
        ref = gdd.read_dump(out)
    h = InitializeHierarchy(mesh, levels=int(g["meta/size"][2]))
    s = System(h)
    s.update(float(g["meta/weights"][0]), 1.0)
    f = texel_signal(h, mesh["texture"])
    return g, h, s, Brush(s, f), f, ref


def test_cell_count_and_signal(case):
    g, h, _, _, f, ref = case
    assert int(ref["L0/counts"][3]) == h.counts(0)["numCells"]
    np.testing.assert_array_equal(f, ref["solve/f"])
    # the reference's release build divides by 1000 as a multiply by its reciprocal (-ffast-math): last bit
    np.testing.assert_allclose(seeded_mask(len(ref["brush/mask"])), ref["brush/mask"], rtol=0, atol=2e-16)


def test_brush_matches_reference(case):
    _, h, _, brush, _, ref = case
    got = brush.apply(ref["brush/mask"])
    want = ref["brush/out"]
    scale = np.abs(want).max()
    deep, bnd = h.array("deepGlobal"), h.array("boundaryGlobal")
    assert np.abs(got[deep] - want[deep]).max() <= 1e-10 * scale
    assert np.abs(got[bnd] - want[bnd]).max() <= 1e-6 * scale


def test_uniform_brush_is_stiffness_of_signal(case):
    from gradientdomaintextureprocessing_b200.system import STIFFNESS
    _, _, s, brush, f, ref = case
    sf = s.apply(f, STIFFNESS)
    ones = np.ones(len(ref["brush/mask"]))
    assert np.abs(brush.apply(ones) - sf).max() <= 1e-12 * np.abs(sf).max()
    # the reference's uniform brush is its own S f as well
    assert np.abs(ref["brush/out_ones"] - ref["brush/stiffness_f"]).max() <= 1e-12 * np.abs(ref["brush/stiffness_f"]).max()


def test_brush_is_linear_in_the_mask(case):
    _, _, _, brush, _, ref = case
    m = ref["brush/mask"]
    a, b = brush.apply(m), brush.apply(1.0 - m)
    ones = brush.apply(np.ones_like(m))
    assert np.abs(a + b - ones).max() <= 1e-12 * np.abs(ones).max()
