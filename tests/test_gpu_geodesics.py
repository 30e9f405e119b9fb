"""Heat-method geodesics against the compiled reference (tests/golden/geo256:
icosphere 256^2, t = 1e-3, one source; the reference integrates in FP64 with
exact solves).  Tolerances:

* integrated right-hand side from the reference's own smoothed impulse: 5e-6 of
  its largest entry (interior samples and integration in FP32 as in the app's
  build, boundary elements in FP64; measured 4.9e-7);
* distances from our mixed-precision pipeline (both solves to 1e-6): 2e-4 of
  the largest distance (measured 3e-5);
* k sources batched as right-hand sides give the single-source results;
* the benchmark's smoothing time t = mean texel area (tests/golden/geo256area):
  the heat step and the integrated field where the potential is resolved
  (test_mean_texel_area_smoothing says why the distances are not compared).
"""
import numpy as np
import pytest

from conftest import golden_mesh, load_golden

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def geo(built_lib):
    from gradientdomaintextureprocessing_b200.geodesics import Geodesics
    from gradientdomaintextureprocessing_b200.hierarchy import InitializeHierarchy
    g = load_golden("geo256")
    h = InitializeHierarchy(golden_mesh(g), levels=int(g["meta/size"][2]))
    return g, Geodesics(h, smoothing=float(g["geo/weights"][0]), epsilon=float(g["geo/weights"][1]))


def test_sample_counts_cover_reference(geo):
    g, G = geo
    c = G.counts()
    # slots are (cell, triangle) / (element, triangle) pairs; the reference keeps the non-empty ones
    assert c["cell_samples"] >= int(g["geo/source"][2])
    assert c["boundary_samples"] >= int(g["geo/source"][3])


def test_rhs_matches_reference(geo):
    g, G = geo
    rhs = G.rhs(g["geo/u"])
    ref = g["geo/rhs"]
    err = np.abs(rhs - ref).max() / np.abs(ref).max()
    assert err < 5e-6, err


def test_rhs_is_batched(geo):
    g, G = geo
    u = g["geo/u"]
    U = np.stack([u, 2.0 * u, u[::-1].copy()], 1)
    R = G.rhs(U)
    for c in range(3):
        np.testing.assert_array_equal(R[:, c], G.rhs(U[:, c]))
    # the normalised field does not depend on the potential's scale
    np.testing.assert_allclose(R[:, 1], R[:, 0], rtol=0, atol=1e-6 * np.abs(R[:, 0]).max())


def test_distance_matches_reference(geo):
    g, G = geo
    src = int(g["geo/source"][0])
    d, rep = G.distance([src])
    ref = g["geo/dist"]
    assert rep["rel_residual_max"] <= 1e-6
    assert d[src, 0] == 0.0
    err = np.abs(d[:, 0] - ref).max() / np.abs(ref).max()
    assert err < 2e-4, err


def test_multi_source_batch_matches_single(geo):
    g, G = geo
    n = G.n
    srcs = [int(g["geo/source"][0]), n // 7, (5 * n) // 9]
    D, _ = G.distance(srcs)
    for c, s in enumerate(srcs):
        d, _ = G.distance([s])
        assert np.abs(D[:, c] - d[:, 0]).max() <= 1e-4 * np.abs(d).max()


@pytest.fixture(scope="module")
def geo1024(built_lib):
    from gradientdomaintextureprocessing_b200 import meshgen
    from gradientdomaintextureprocessing_b200.geodesics import Geodesics
    from gradientdomaintextureprocessing_b200.hierarchy import InitializeHierarchy
    g = load_golden("geo1024")
    h = InitializeHierarchy(meshgen.icosphere_atlas(1024, 1024, subdiv=6, seed=0), levels=4)
    assert list(h.counts(0).values())[:7] == list(g["L0/counts"])
    return g, h, Geodesics(h, smoothing=float(g["geo/weights"][0]), epsilon=float(g["geo/weights"][1]))


def test_distance_matches_reference_1024(geo1024):
    """Full-size heat-method configuration (icosphere(6), 1024^2, 356,581 texels)
    against the reference's exact FP64 pipeline."""
    g, _, G = geo1024
    src = int(g["geo/source"][0])
    d, rep = G.distance([src])
    ref = g["geo/dist"].astype(np.float64)
    assert rep["rel_residual_max"] <= 1e-6 and d[src, 0] == 0.0
    err = np.abs(d[:, 0] - ref).max() / ref.max()
    assert err < 2e-4, err


def test_geodesics_64_sources_1024(geo1024):
    """64 seeded deep-texel sources as 64 right-hand sides of one batched
    pipeline: every column converges, is 0 at its source, is not below -sqrt(t)
    (the smoothed distance's minimum sits within the smoothing length of the
    source, so values down to that scale are the method's, not the solver's)
    and is bounded by half the great circle of the unit-area sphere
    (pi r, r = 1 / sqrt(4 pi)); batched columns equal single-source runs."""
    g, h, G = geo1024
    deep = h.array("deepGlobal")
    rng = np.random.default_rng(0)
    srcs = rng.choice(deep, size=64, replace=False)
    D, rep = G.distance(srcs, tol=1e-6)
    assert rep["rel_residual_max"] <= 1e-6
    assert np.all(D[srcs, np.arange(64)] == 0.0)
    assert D.min() > -np.sqrt(G.t)
    assert D.max() < 1.1 * np.pi / np.sqrt(4 * np.pi)
    for c in (0, 37):
        d, _ = G.distance([srcs[c]], tol=1e-6)
        assert np.abs(D[:, c] - d[:, 0]).max() <= 1e-4 * np.abs(d).max()


@pytest.fixture(scope="module")
def geo_area(built_lib):
    """The benchmark's smoothing time, the mean texel area (t = 6.3e-5 on the
    icosphere 256^2 mesh of geo256), against the reference's exact FP64
    pipeline at the same t (tests/golden/geo256area.npz)."""
    from gradientdomaintextureprocessing_b200 import meshgen
    from gradientdomaintextureprocessing_b200.geodesics import Geodesics, mean_texel_area
    from gradientdomaintextureprocessing_b200.hierarchy import InitializeHierarchy
    g = load_golden("geo256area")
    h = InitializeHierarchy(meshgen.icosphere_atlas(256, 256, subdiv=5), levels=int(g["meta/size"][2]))
    assert list(h.counts(0).values())[:7] == list(g["L0/counts"])
    t = mean_texel_area(h)
    assert t == float(g["geo/weights"][0])
    return g, h, Geodesics(h, smoothing=t, epsilon=float(g["geo/weights"][1]))


def test_mean_texel_area_smoothing(geo_area):
    """At t = mean texel area the heat step (M + t S) u = delta matches the
    reference's u to 1e-5 of its largest value (measured 1.3e-7), and the
    integrated normalised field of the reference's own u matches its right-hand
    side to 5e-6 wherever |u| > 1e-20 (measured 9.3e-8 on 42 % of the texels).
    Farther out u decays to 6e-47: 8.5 % of the texels lie below FP32's
    smallest normal number (1.2e-38), where the interior samples (FP32, the
    precision of the app's Geodesics build) see a zero gradient and the
    reference's FP64 harness normalises a gradient of size 1e-46.  No solve to
    a relative residual of 1e-6 resolves those values either, so the
    distances are not compared: the reference's own exact-solve distances go
    negative there (down to -0.52 of a largest 0.88).  The pipeline still
    converges and is 0 at the source."""
    g, h, G = geo_area
    src = int(g["geo/source"][0])
    delta = np.zeros((G.n, 1))
    delta[src] = 1.0
    u, rep = G.smooth.solve(delta, tol=1e-6)
    u_ref = g["geo/u"]
    assert rep["rel_residual_max"] <= 1e-6
    assert np.abs(u[:, 0] - u_ref).max() < 1e-5 * np.abs(u_ref).max()
    resolved = np.abs(u_ref) > 1e-20
    rhs, ref = G.rhs(u_ref), g["geo/rhs"]
    assert np.abs(rhs - ref)[resolved].max() < 5e-6 * np.abs(ref).max()
    assert np.abs(u_ref).min() < np.finfo(np.float32).tiny and g["geo/dist"].min() < 0
    d, rep_d = G.distance([src])
    assert rep_d["rel_residual_max"] <= 1e-6 and d[src, 0] == 0.0
