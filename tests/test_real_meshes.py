"""The texel hierarchy on the reference's own meshes (Data/{Julius,Hand,Bunny,David},
256 x 256 after the filtering app's preprocessing) against the UNMODIFIED
reference hierarchy on the same input (tests/golden/make_real_golden.py).

* counts, every index array, cell and node types, every active cell's corners
  (the global cell order), the boundary restriction, chart corners and cell
  sizes, texture node positions / charts / interior flags, boundary nodes:
  bit-exact;
* texture node triangle ids: equal except for at most two exterior texels per
  mesh, whose nearest-triangle test is a near-tie (the reference's release
  build computes with -ffast-math, so its roundings differ in the last bit);
* texture node barycentric coordinates (seeded sample): within 1e-13, for the
  same reason;
* the embedding parameter metric (seeded sample of triangles): within 1e-12 of
  its largest entry.

Needs the reference's data directory (skipped otherwise); no GPU.
"""
import json
import os
import sys

import numpy as np
import pytest

from conftest import GOLDEN, reference_data

REAL = os.path.join(GOLDEN, "real")
REFERENCE_DATA = reference_data()
with open(os.path.join(REAL, "real_meshes.json")) as fh:
    TABLE = json.load(fh)
sys.path.insert(0, GOLDEN)  # make_real_golden: the digests and array names the fixtures use

pytestmark = pytest.mark.skipif(not os.path.isdir(REFERENCE_DATA), reason="the reference's data files are not present")


@pytest.fixture(scope="module", params=sorted(TABLE))
def case(request, built_lib):
    import make_real_golden as mk
    from gradientdomaintextureprocessing_b200 import textureio
    from gradientdomaintextureprocessing_b200.hierarchy import InitializeHierarchy
    name = request.param
    entry = TABLE[name]
    mesh = textureio.ReadTexturedMesh(os.path.join(REFERENCE_DATA, name))
    mesh, pad, w, h = textureio.prepare_filtering_mesh(mesh, mk.SIZE, mk.SIZE)
    assert [w, h] == entry["size"] and list(pad) == entry["padding"]
    hier = InitializeHierarchy(mesh, width=w, height=h, levels=entry["levels"])
    key = os.path.splitext(os.path.basename(name))[0]
    with np.load(os.path.join(REAL, f"{key}.npz")) as z:
        arrays = {k: z[k] for k in z.files}
    return entry, hier, arrays, mk


def test_counts_and_index_arrays_bit_exact(case):
    entry, h, _, mk = case
    assert h.levels == entry["levels"]  # coarsest level already below the dense-solve size
    for l in range(entry["levels"]):
        c = h.counts(l)
        mine = [c[k] for k in ("numTexels", "numDeepTexels", "numBoundaryTexels", "numCells", "numBoundaryCells",
                               "numInteriorCells", "numInteriorTexels")]
        assert mine == entry["counts"][str(l)], l
        for ref, name in mk.INDEX_ARRAYS.items():
            key = f"L{l}/{ref}"
            if key in entry["digests"]:
                assert mk.digest(h.array(name, l).astype(np.int32)) == entry["digests"][key], key


def test_boundary_restriction_bit_exact(case):
    entry, h, _, mk = case
    for l in range(entry["levels"] - 1):
        R = h.csr("boundaryRestriction", l)
        assert mk.csr_digest(R.indptr, R.indices, R.data) == entry["digests"][f"L{l}/boundaryRestriction"], l


def test_chart_corners_bit_exact(case):
    entry, h, arrays, _ = case
    for l in range(entry["levels"]):
        np.testing.assert_array_equal(h.array("chartsd", l), arrays[f"L{l}/charts_d"])


def test_texture_and_boundary_nodes(case):
    entry, h, arrays, mk = case
    tn = h.array("textureNodes").astype(np.int32)
    assert mk.digest(tn[:, [0, 1, 2, 4]]) == entry["digests"]["textureNodes_cols"]
    assert mk.digest(h.array("boundaryNodes").astype(np.int32)) == entry["digests"]["boundaryNodes"]
    differ = np.nonzero(tn[:, 3] != arrays["tId"])[0]
    assert len(differ) <= 2 and np.all(arrays["interior"][differ] == 0), differ
    rows = arrays["bary_rows"]
    same = np.isin(rows, differ, invert=True)
    bary = h.array("textureBary")[rows]
    np.testing.assert_allclose(bary[same], arrays["bary"][same], rtol=0, atol=1e-13)


def test_embedding_metric(case):
    entry, h, arrays, mk = case
    from gradientdomaintextureprocessing_b200 import textureio
    from gradientdomaintextureprocessing_b200.metric import InitializeMetric
    name = next(n for n, e in TABLE.items() if e is entry)
    mesh = textureio.ReadTexturedMesh(os.path.join(REFERENCE_DATA, name))
    mesh, _, _, _ = textureio.prepare_filtering_mesh(mesh, mk.SIZE, mk.SIZE)
    P = InitializeMetric(mesh).reshape(-1, 4)[arrays["metric_rows"]]
    assert np.abs(P - arrays["metric"]).max() <= 1e-12 * arrays["metric_scale"][0]
