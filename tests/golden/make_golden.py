"""Regenerates the golden fixtures in this directory from the reference itself.

Runs the oracle harness (``oracle/_ref/gdtp_ref``: the reference solve path
compiled from its own sources by ``oracle/Makefile``) on seeded meshes from
``gradientdomaintextureprocessing_b200.meshgen`` and keeps the arrays the tests
compare against.  Needs the reference checkout (only this script does):

    make -C oracle && python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from gdd import read_dump  # noqa: E402
from gradientdomaintextureprocessing_b200 import meshgen  # noqa: E402

CASES = {
    # name: (mesh factory, levels, stiffness, sharpness, keep coefficients)
    "torus128": (lambda: meshgen.torus_atlas(128, 128), 4, 1e-3, 2.0, True),
    "torus256": (lambda: meshgen.torus_atlas(256, 256), 4, 1e-3, 2.0, False),
    "ico256": (lambda: meshgen.icosphere_atlas(256, 256, subdiv=5), 4, 1e-3, 2.0, True),
    # line-integral convolution: anisotropic metric of a tangent field, operator
    # M + 1e-4 S (the LIC app's default licStiffness), right-hand side M f
    "genus2lic512": (lambda: meshgen.genus2_atlas(512, 512, nu=64, nv=32), 4, 1e-4, 0.0, True),
}
# tangent fields (reference .vf files) of the anisotropic cases
FIELDS = {"genus2lic512": lambda mesh: meshgen.gaussian_bump_field(mesh, bumps=8, seed=0)}
# heat-method geodesics (the Geodesics app's pipeline): mesh, levels, smoothing weight t, source texel
GEODESIC = {"geo256": (lambda: meshgen.icosphere_atlas(256, 256, subdiv=5), 4, 1e-3, 12345),
            # the heat-method configuration at full size: only the source and the distances are kept (FP32)
            "geo1024": (lambda: meshgen.icosphere_atlas(1024, 1024, subdiv=6, seed=0), 4, 1e-3, 100000),
            # the benchmark's smoothing time, the mean texel area (None: 1 / texels of the area-normalised mesh);
            # the mesh is regenerated from its generator by the test, the reference's u, rhs and distances kept
            "geo256area": (lambda: meshgen.icosphere_atlas(256, 256, subdiv=5), 4, None, 12345)}


def make_geodesic(name: str) -> None:
    factory, levels, t, src = GEODESIC[name]
    mesh = factory()
    if t is None:
        from gradientdomaintextureprocessing_b200.geodesics import mean_texel_area
        from gradientdomaintextureprocessing_b200.hierarchy import InitializeHierarchy
        t = mean_texel_area(InitializeHierarchy(mesh, levels=levels))
    exe = os.path.join(ROOT, "oracle", "_ref", "gdtp_ref")
    with tempfile.TemporaryDirectory() as tmp:
        gdm, out = os.path.join(tmp, "m.gdm"), os.path.join(tmp, "o.gdd")
        meshgen.write_gdm(gdm, mesh)
        subprocess.run([exe, gdm, out, str(levels), repr(t), "0", "1", "geodesic", "1e-6", "", str(src)], check=True,
                       capture_output=True)
        d = read_dump(out)
    if name == "geo256area":
        keep = {"meta/size": d["meta/size"], "L0/counts": d["L0/counts"], "geo/source": d["geo/source"],
                "geo/weights": d["geo/weights"], "geo/u": d["geo/u"], "geo/rhs": d["geo/rhs"], "geo/dist": d["geo/dist"]}
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **{k.replace("/", "__"): v for k, v in keep.items()})
        print(name, sum(v.nbytes for v in keep.values()) / 1e6, "MB raw")
        return
    if name == "geo1024":  # the mesh is regenerated from its seed by the test
        keep = {"meta/size": d["meta/size"], "L0/counts": d["L0/counts"], "geo/source": d["geo/source"],
                "geo/weights": d["geo/weights"], "geo/dist": d["geo/dist"].astype(np.float32)}
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **{k.replace("/", "__"): v for k, v in keep.items()})
        print(name, sum(v.nbytes for v in keep.values()) / 1e6, "MB raw")
        return
    keep = {"mesh/vertices": mesh["vertices"], "mesh/triangles": mesh["triangles"], "mesh/uv": mesh["uv"],
            "mesh/texture": mesh["texture"][..., :1], "meta/size": d["meta/size"], "L0/counts": d["L0/counts"]}
    for k in d:
        if k.startswith("geo/"):
            keep[k] = d[k]
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **{k.replace("/", "__"): v for k, v in keep.items()})
    print(name, sum(v.nbytes for v in keep.values()) / 1e6, "MB raw")
INDEX_KEYS = ["counts", "nodeinfo", "boundaryGlobalIndex", "deepGlobalIndex", "boundaryAndDeepIndex", "rasterLines",
              "restrictionLines", "deepLines", "prolongationLines", "charts_i", "charts_d"]


def make(name: str) -> None:
    factory, levels, lam, sharp, coefs = CASES[name]
    mesh = factory()
    exe = os.path.join(ROOT, "oracle", "_ref", "gdtp_ref")
    vf = FIELDS[name](mesh) if name in FIELDS else None
    with tempfile.TemporaryDirectory() as tmp:
        gdm, out, vfp = os.path.join(tmp, "m.gdm"), os.path.join(tmp, "o.gdd"), os.path.join(tmp, "f.vf")
        meshgen.write_gdm(gdm, mesh)
        args = [exe, gdm, out, str(levels), str(lam), str(sharp), "12", "dump", "1e-6"]
        if vf is not None:
            meshgen.write_vf(vfp, vf)
            args.append(vfp)
        subprocess.run(args, check=True, capture_output=True)
        d = read_dump(out)
    keep = {"mesh/vertices": mesh["vertices"], "mesh/triangles": mesh["triangles"], "mesh/uv": mesh["uv"],
            "mesh/texture": mesh["texture"], "meta/size": d["meta/size"], "meta/weights": d["meta/weights"],
            "metric/parameter": d["metric/parameter"]}
    if vf is not None:
        keep["mesh/field"] = vf
    for k in ("solve/f", "solve/rhs", "solve/exact", "vcycle/history", "fine/textureNodes", "fine/textureBary",
              "fine/boundaryNodes"):
        keep[k] = d[k]
    for l in range(levels):
        for k in INDEX_KEYS:
            if f"L{l}/{k}" in d:
                keep[f"L{l}/{k}"] = d[f"L{l}/{k}"]
        for part in ("ptr", "col", "val"):
            if f"L{l}/boundaryRestriction/{part}" in d:
                keep[f"L{l}/boundaryRestriction/{part}"] = d[f"L{l}/boundaryRestriction/{part}"]
    if coefs:
        for k in ("fine/deepMass", "fine/deepStiffness"):
            keep[k] = d[k]
        for m in ("BBmass", "BBstiffness", "BDmass", "BDstiffness"):
            for part in ("ptr", "col", "val"):
                keep[f"fine/{m}/{part}"] = d[f"fine/{m}/{part}"]
        for l in range(levels):
            keep[f"L{l}/coef/deep"] = d[f"L{l}/coef/deep"]
            for m in ("BB", "BD"):
                for part in ("ptr", "col", "val"):
                    keep[f"L{l}/coef/{m}/{part}"] = d[f"L{l}/coef/{m}/{part}"]
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **{k.replace("/", "__"): v for k, v in keep.items()})
    print(name, sum(v.nbytes for v in keep.values()) / 1e6, "MB raw")


if __name__ == "__main__":
    for name in (sys.argv[1:] or list(CASES) + list(GEODESIC)):
        if name in GEODESIC:
            make_geodesic(name)
        else:
            make(name)
