"""Metrics and the genus-2 LIC workload (host only).

* the oracle's metric restatement is pinned to the compiled reference
  (``metric/parameter`` of the golden fixtures, embedding and anisotropic);
* ``libgdtp.so``'s metrics agree with the reference to 1e-12 relative;
* the genus-2 generator yields a closed oriented manifold of genus 2 with 32
  charts and no flipped texture triangle, and writes the reference's ``.vf``
  layout.
"""
import os
import tempfile

import numpy as np
import pytest

from conftest import golden_mesh, load_golden

CASES = ["torus128", "ico256", "genus2lic512"]


def rel(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


@pytest.mark.parametrize("name", CASES)
def test_oracle_metric_matches_reference(name):
    import port
    g = load_golden(name)
    G = port.embedding_metric(g["mesh/vertices"], g["mesh/triangles"].astype(np.int64))
    if "mesh/field" in g:
        G = port.vector_field_metric(G, g["mesh/field"])
    P = port.metric_entries(port.parameter_metric(g["mesh/uv"], G))
    assert rel(P, g["metric/parameter"]) < 1e-12


@pytest.mark.parametrize("name", CASES)
def test_library_metric_matches_reference(name, built_lib):
    from gradientdomaintextureprocessing_b200.metric import InitializeAnisotropicMetric, InitializeMetric
    g = load_golden(name)
    mesh = golden_mesh(g)
    if "mesh/field" in g:
        P = InitializeAnisotropicMetric(mesh, g["mesh/field"])
    else:
        P = InitializeMetric(mesh)
    assert rel(P, g["metric/parameter"]) < 1e-12


def test_uniform_metric_is_scaled_identity(built_lib):
    import port
    from gradientdomaintextureprocessing_b200.metric import UNIFORM_METRIC, InitializeMetric
    mesh = golden_mesh(load_golden("torus128"))
    P = InitializeMetric(mesh, UNIFORM_METRIC)
    uv = mesh["uv"]
    d1, d2 = uv[:, 1] - uv[:, 0], uv[:, 2] - uv[:, 0]
    area = (np.abs(d1[:, 0] * d2[:, 1] - d1[:, 1] * d2[:, 0]) / 2).sum()
    np.testing.assert_allclose(P[:, [0, 3]], 1.0 / area, rtol=1e-9)
    assert np.abs(P[:, [1, 2]]).max() < 1e-9 / area
    assert port is not None


def test_metric_rejects_bad_input(built_lib):
    from gradientdomaintextureprocessing_b200 import _lib
    from gradientdomaintextureprocessing_b200.metric import InitializeAnisotropicMetric
    mesh = golden_mesh(load_golden("torus128"))
    with pytest.raises(ValueError):
        InitializeAnisotropicMetric(mesh, np.zeros((3, 2)))
    with pytest.raises(_lib.GDTPError):
        InitializeAnisotropicMetric(mesh, np.zeros((len(mesh["triangles"]), 2)), isotropic=0.0)


def test_genus2_generator_topology_and_atlas():
    from gradientdomaintextureprocessing_b200 import meshgen
    m = meshgen.genus2_atlas(512, 512, nu=64, nv=32)
    t = m["triangles"].astype(np.int64)
    e = np.concatenate([t[:, [0, 1]], t[:, [1, 2]], t[:, [2, 0]]])
    key = e[:, 0] * len(m["vertices"]) + e[:, 1]
    rkey = e[:, 1] * len(m["vertices"]) + e[:, 0]
    assert len(np.unique(key)) == len(key)                 # no repeated directed edge
    assert np.isin(rkey, key).all()                        # every edge has its twin: closed, oriented
    assert len(np.unique(t)) == len(m["vertices"])         # no unreferenced vertex
    chi = len(m["vertices"]) - len(key) // 2 + len(t)
    assert chi == -2                                       # genus 2
    assert meshgen.chart_ids(m["triangles"], m["uv"]).max() + 1 == 32
    uv = m["uv"]
    area = (uv[:, 1, 0] - uv[:, 0, 0]) * (uv[:, 2, 1] - uv[:, 0, 1]) - (uv[:, 2, 0] - uv[:, 0, 0]) * (uv[:, 1, 1] - uv[:, 0, 1])
    assert (area > 0).all()
    assert uv.min() > 0 and uv.max() < 1


def test_bump_field_is_tangent_and_roundtrips():
    from gradientdomaintextureprocessing_b200 import meshgen
    m = meshgen.genus2_atlas(256, 256, nu=32, nv=16)
    vf = meshgen.gaussian_bump_field(m, seed=3)
    assert vf.shape == (len(m["triangles"]), 2) and np.isfinite(vf).all()
    with tempfile.TemporaryDirectory() as tmp:
        p = os.path.join(tmp, "f.vf")
        meshgen.write_vf(p, vf)
        assert os.path.getsize(p) == 4 + 16 * len(vf)
        np.testing.assert_array_equal(meshgen.read_vf(p), vf)
