"""Texel hierarchy (classification, indexing, lines, boundary restriction) is
bit-exact to the reference on the golden meshes (reference run by
tests/golden/make_golden.py through oracle/_ref)."""
import numpy as np
import pytest

from conftest import golden_csr, golden_mesh, load_golden

CASES = ["torus128", "torus256", "ico256", "genus2lic512"]
NAMES = {"nodeinfo": "nodeinfo", "boundaryGlobalIndex": "boundaryGlobal", "deepGlobalIndex": "deepGlobal",
         "boundaryAndDeepIndex": "boundaryAndDeep", "rasterLines": "rasterLines", "restrictionLines": "restrictionLines",
         "deepLines": "deepLines", "prolongationLines": "prolongationLines", "charts_i": "charts"}


@pytest.fixture(scope="module", params=CASES)
def case(request, built_lib):
    from gradientdomaintextureprocessing_b200.hierarchy import InitializeHierarchy
    g = load_golden(request.param)
    levels = int(g["meta/size"][2])
    return g, InitializeHierarchy(golden_mesh(g), levels=levels), levels


def test_counts_and_indices_bit_exact(case):
    g, h, levels = case
    assert h.levels >= levels
    for l in range(levels):
        c = h.counts(l)
        mine = [c[k] for k in ("numTexels", "numDeepTexels", "numBoundaryTexels", "numCells", "numBoundaryCells",
                               "numInteriorCells", "numInteriorTexels")]
        assert mine == list(g[f"L{l}/counts"]), l
        for ref, name in NAMES.items():
            key = f"L{l}/{ref}"
            if key not in g:
                continue
            a = h.array(name, l)
            assert a.shape == g[key].shape and np.array_equal(a, g[key]), (l, name)
        np.testing.assert_array_equal(h.array("chartsd", l), g[f"L{l}/charts_d"])


def test_boundary_restriction_exact(case):
    g, h, levels = case
    for l in range(levels - 1):
        R = h.csr("boundaryRestriction", l)
        Rr = golden_csr(g, f"L{l}/boundaryRestriction")
        n = max(R.shape[1], Rr.shape[1])
        R.resize((R.shape[0], n))
        Rr.resize((Rr.shape[0], n))
        assert R.shape == Rr.shape and (R != Rr).nnz == 0


def test_texture_nodes_and_boundary_nodes(case):
    g, h, _ = case
    np.testing.assert_array_equal(h.array("textureNodes"), g["fine/textureNodes"])
    np.testing.assert_array_equal(h.array("textureBary"), g["fine/textureBary"])
    np.testing.assert_array_equal(h.array("boundaryNodes"), g["fine/boundaryNodes"])


def test_extra_levels_reach_dense_coarse_size(case):
    _, h, levels = case
    assert h.counts(h.levels - 1)["numTexels"] <= 2600 or h.levels == 12


def test_texel_signal_samples_every_layout(case):
    """gdtp_texel_signal reads the texel's pixel (textureNodes' x, y) from any
    strided float32 / float64 image, equal to the gather by the reference's
    texture nodes (TextureFiltering.cpp:603-608)."""
    from gradientdomaintextureprocessing_b200.system import texel_signal
    g, h, _ = case
    tn = g["fine/textureNodes"]
    w = int(tn[:, 0].max()) + 2
    hgt = int(tn[:, 1].max()) + 3
    rng = np.random.default_rng(0)
    img = rng.random((hgt, w, 3)).astype(np.float32)
    want = img[tn[:, 1], tn[:, 0]].astype(np.float64)
    np.testing.assert_array_equal(texel_signal(h, img), want)
    np.testing.assert_array_equal(texel_signal(h, img.astype(np.float64)), want)
    # channel-planar storage seen as height x width x channels, and a single channel
    planar = np.ascontiguousarray(img.transpose(2, 0, 1)).transpose(1, 2, 0)
    assert not planar.flags["C_CONTIGUOUS"]
    np.testing.assert_array_equal(texel_signal(h, planar), want)
    np.testing.assert_array_equal(texel_signal(h, img[:, :, 1]), want[:, 1])
    with pytest.raises(Exception):
        texel_signal(h, img[: int(tn[:, 1].max()), :, :])
