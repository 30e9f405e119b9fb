"""Hierarchy fixtures on the reference's own meshes (Data/{Julius,Hand,Bunny,David}),
run in a checkout that has the reference tree and oracle/_ref built:

    python tests/golden/make_real_golden.py <reference checkout>

Each mesh goes through the filtering app's preprocessing (textureio.
prepare_filtering_mesh: unit radius, v flipped, padding) for a 256 x 256 texture,
then through the UNMODIFIED reference hierarchy (oracle/_ref/gdtp_ref, dump
mode).  Stored, per mesh (tests/golden/real/):

* real_meshes.json: padded size, per-level counts, SHA-256 digests of every
  index array, of the canonical boundary restriction (sorted CSR) and of the
  texture nodes' (ci, cj, chart, interior) columns;
* <mesh>.npz: per-level chart corners and cell sizes, every texture node's
  triangle id, the barycentric coordinates of a seeded sample of nodes, and the
  embedding metric (InitializeMetric) of a seeded sample of triangles.

The meshes themselves are not copied: the test reads them from the reference's
data directory when it is present.
"""
from __future__ import annotations

import hashlib
import json
import os
import subprocess
import sys
import tempfile

import numpy as np
import scipy.sparse as sp

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
OUT = os.path.join(HERE, "real")
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import gdd  # noqa: E402
from gradientdomaintextureprocessing_b200 import meshgen, textureio  # noqa: E402

MESHES = ["Julius/julius.ply", "Hand/hand.ply", "Bunny/bunny.ply", "David/david.ply"]
SIZE, LEVELS, SAMPLE = 256, 4, 3000
INDEX_ARRAYS = {"nodeinfo": "nodeinfo", "boundaryGlobalIndex": "boundaryGlobal", "deepGlobalIndex": "deepGlobal",
                "boundaryAndDeepIndex": "boundaryAndDeep", "rasterLines": "rasterLines",
                "restrictionLines": "restrictionLines", "deepLines": "deepLines",
                "prolongationLines": "prolongationLines", "charts_i": "charts", "cellType": "cellType",
                "nodeType": "nodeType", "cellIndices": "cellCorners",
                "interiorTexelToCellLines": "interiorTexelToCellLines"}


def digest(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def csr_digest(ptr, col, val) -> str:
    m = sp.csr_matrix((np.asarray(val, np.float64), np.asarray(col, np.int32), np.asarray(ptr, np.int32)))
    m.sum_duplicates()
    m.sort_indices()
    return digest(np.concatenate([m.indptr.astype(np.int64), m.indices.astype(np.int64)])) + digest(m.data)


def prepared(ref_tree: str, name: str):
    mesh = textureio.ReadTexturedMesh(os.path.join(ref_tree, "Data", name))
    mesh, pad, w, h = textureio.prepare_filtering_mesh(mesh, SIZE, SIZE)
    return mesh, pad, w, h


def main(ref_tree: str) -> None:
    os.makedirs(OUT, exist_ok=True)
    table = {}
    for name in MESHES:
        mesh, pad, w, h = prepared(ref_tree, name)
        mesh["texture"] = np.zeros((h, w, 3), np.float32)
        with tempfile.TemporaryDirectory() as td:
            src, out = os.path.join(td, "m.gdm"), os.path.join(td, "m.gdd")
            meshgen.write_gdm(src, mesh)
            subprocess.run([os.path.join(ROOT, "oracle", "_ref", "gdtp_ref"), src, out, str(LEVELS), "1e-3", "2.0", "2", "dump"],
                           check=True, capture_output=True)
            g = gdd.read_dump(out)
        entry = {"size": [w, h], "padding": list(pad), "levels": LEVELS, "counts": {}, "digests": {}}
        arrays = {}
        for l in range(LEVELS):
            entry["counts"][str(l)] = [int(x) for x in g[f"L{l}/counts"]]
            for ref in INDEX_ARRAYS:
                key = f"L{l}/{ref}"
                if key in g:
                    entry["digests"][key] = digest(g[key].astype(np.int32))
            arrays[f"L{l}/charts_d"] = g[f"L{l}/charts_d"]
            if l < LEVELS - 1:
                b = f"L{l}/boundaryRestriction"
                entry["digests"][b] = csr_digest(g[b + "/ptr"], g[b + "/col"], g[b + "/val"])
        tn = g["fine/textureNodes"].astype(np.int32)
        entry["digests"]["textureNodes_cols"] = digest(tn[:, [0, 1, 2, 4]])
        entry["digests"]["boundaryNodes"] = digest(g["fine/boundaryNodes"].astype(np.int32))
        rows = np.sort(np.random.default_rng(len(table)).choice(len(tn), size=min(SAMPLE, len(tn)), replace=False))
        arrays["tId"] = tn[:, 3]
        arrays["interior"] = tn[:, 4]
        arrays["bary_rows"] = rows.astype(np.int32)
        arrays["bary"] = g["fine/textureBary"][rows]
        pm = g["metric/parameter"]  # the reference's embedding metric, per mesh triangle
        mrows = np.sort(np.random.default_rng(100 + len(table)).choice(len(pm), size=min(SAMPLE, len(pm)), replace=False))
        arrays["metric_rows"] = mrows.astype(np.int32)
        arrays["metric"] = pm[mrows]
        arrays["metric_scale"] = np.array([np.abs(pm).max()])
        key = os.path.splitext(os.path.basename(name))[0]
        np.savez_compressed(os.path.join(OUT, f"{key}.npz"), **arrays)
        table[name] = entry
        print(name, entry["size"], entry["counts"]["0"][:3])
    with open(os.path.join(OUT, "real_meshes.json"), "w") as fh:
        json.dump(table, fh, indent=1, sort_keys=True)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(f"usage: python {sys.argv[0]} <reference checkout>")
    main(sys.argv[1])
