"""Generates the texture I/O fixtures under tests/golden/io/ (run in a checkout
that has the reference tree and oracle/_ref/gdtp_ref_io built by oracle/Makefile):

    python tests/golden/make_io_golden.py <reference checkout>

* PLY files in several encodings (ASCII with float and with double columns,
  binary little and big endian, a quad face, extra properties and elements),
  each read by the reference's own ReadTexturedMesh (oracle/_ref/gdtp_ref_io):
  golden arrays in io_golden.npz;
* a file written by the reference's WriteTexturedMesh (ref_written.ply) and
  what the reference reads back from it;
* padding cases (texture coordinates near and beyond the image edge, sizes not
  multiples of 8) through the reference's ComputePadding /
  PaddTextureCoordinates / UnpaddTextureCoordinates;
* a small .vf file and the reference's ReadVector of it;
* SHA-256 digests of what the reference reads from its own shipped data
  (Data/*/*.ply, Data/Fertility/*.vf): reference_data.json.  The test compares
  the product's reader with them when that data is present.
"""
from __future__ import annotations

import hashlib
import json
import os
import struct
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
OUT = os.path.join(HERE, "io")
TOOL = os.path.join(ROOT, "oracle", "_ref", "gdtp_ref_io")
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import gdd  # noqa: E402

TYPES = {"char": "b", "uchar": "B", "short": "h", "ushort": "H", "int": "i", "uint": "I", "float": "f", "double": "d",
         "int8": "b", "uint8": "B", "int16": "h", "uint16": "H", "int32": "i", "uint32": "I", "float32": "f", "float64": "d"}


def sample_mesh(seed: int, quad: bool = False):
    rng = np.random.default_rng(seed)
    nv = 7
    v = rng.normal(size=(nv, 3)) * np.array([1.0, 10.0, 1e3])
    faces = [[0, 1, 2], [2, 1, 3], [3, 4, 5], [5, 6, 0]]
    if quad:
        faces.append([1, 3, 5, 6])
    tex = [rng.uniform(-0.05, 1.05, size=2 * len(f)) for f in faces]
    return v, faces, tex


def write_ply(path, fmt, v, faces, tex, vtype="double", ttype="double", ctype="uchar", itype="int", extra=False, comments=()):
    lines = ["ply", f"format {fmt} 1.0"] + [f"comment {c}" for c in comments]
    if extra:
        lines.append("obj_info generated for the texture I/O parity tests")
    lines += [f"element vertex {len(v)}", f"property {vtype} x", f"property {vtype} y", f"property {vtype} z"]
    if extra:
        lines += ["property uchar red", "property float nx"]
    lines += [f"element face {len(faces)}", f"property list {ctype} {itype} vertex_indices"]
    if extra:
        lines.append("property int flags")
    lines.append(f"property list {ctype} {ttype} texcoord")
    if extra:
        lines += ["element edge 2", "property int vertex1", "property int vertex2"]
    lines.append("end_header")
    head = ("\n".join(lines) + "\n").encode()
    if fmt == "ascii":
        body = []
        vf = "%.9g" if vtype in ("float", "float32") else "%.17g"
        tf = "%.9g" if ttype in ("float", "float32") else "%.17g"
        for p in v:
            body.append(" ".join(vf % x for x in p) + (" 200 -0.5" if extra else ""))
        for f, t in zip(faces, tex):
            body.append(" ".join([str(len(f))] + [str(i) for i in f] + (["7"] if extra else []) + [str(len(t))] + [tf % x for x in t]))
        if extra:
            body += ["0 1", "2 3"]
        data = ("\n".join(body) + "\n").encode()
    else:
        e = "<" if fmt == "binary_little_endian" else ">"
        data = b""
        for p in v:
            data += struct.pack(e + TYPES[vtype] * 3, *p)
            if extra:
                data += struct.pack(e + "Bf", 200, -0.5)
        for f, t in zip(faces, tex):
            data += struct.pack(e + TYPES[ctype], len(f)) + struct.pack(e + TYPES[itype] * len(f), *f)
            if extra:
                data += struct.pack(e + "i", 7)
            data += struct.pack(e + TYPES[ctype], len(t)) + struct.pack(e + TYPES[ttype] * len(t), *t)
        if extra:
            data += struct.pack(e + "iiii", 0, 1, 2, 3)
    with open(path, "wb") as fh:
        fh.write(head + data)


def ref(*args) -> dict:
    with tempfile.TemporaryDirectory() as td:
        out = os.path.join(td, "out.gdd")
        subprocess.run([TOOL, *args, out], check=True, capture_output=True)
        return gdd.read_dump(out)


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def main(ref_tree: str) -> None:
    os.makedirs(OUT, exist_ok=True)
    golden = {}
    cases = {
        "ascii_double": dict(fmt="ascii", comments=("TextureFile atlas texture.png",)),
        "ascii_float": dict(fmt="ascii", vtype="float", ttype="float", extra=True, quad=True),
        "binary_le": dict(fmt="binary_little_endian", vtype="float", ttype="float", extra=True),
        "binary_be": dict(fmt="binary_big_endian", ctype="int", itype="uint", quad=True),
    }
    for i, (name, kw) in enumerate(cases.items()):
        quad = kw.pop("quad", False)
        v, faces, tex = sample_mesh(i, quad)
        if kw.get("vtype") in ("float", "float32") and kw["fmt"] != "ascii":
            v = v.astype(np.float32).astype(np.float64)
        path = os.path.join(OUT, f"{name}.ply")
        write_ply(path, v=v, faces=faces, tex=tex, **kw)
        d = ref("ply", path)
        for k in ("vertices", "triangles", "uv"):
            golden[f"{name}/{k}"] = d[k]
    # sized type names (float64, float32, int16): the reference's PLY library
    # aborts on this file ("buffer overflow detected"), so its golden arrays are
    # the values written into it
    v, faces, tex = sample_mesh(11)
    write_ply(os.path.join(OUT, "binary_le_sized_names.ply"), "binary_little_endian", v, faces, tex, vtype="float64",
              ttype="float32", itype="int16")
    golden["sized_names/vertices"] = v
    golden["sized_names/triangles"] = np.array(faces, np.int32)
    golden["sized_names/uv"] = np.array(tex, np.float32).astype(np.float64).reshape(-1, 2)
    # a file written by the reference's WriteTexturedMesh
    written = os.path.join(OUT, "ref_written.ply")
    subprocess.run([TOOL, "writemesh", os.path.join(OUT, "ascii_double.ply"), written], check=True, capture_output=True)
    d = ref("ply", written)
    for k in ("vertices", "triangles", "uv"):
        golden[f"ref_written/{k}"] = d[k]
    # padding
    rng = np.random.default_rng(7)
    pad_cases = [(2048, 2048, rng.uniform(0.01, 0.99, (500, 2))), (1000, 700, rng.uniform(-0.02, 1.01, (500, 2))),
                 (1001, 999, rng.uniform(0.2, 0.8, (64, 2))), (640, 480, np.array([[0.0, 0.0], [1.0, 1.0]])),
                 (37, 53, rng.uniform(-0.3, 1.4, (33, 2)))]
    for i, (w, h, uv) in enumerate(pad_cases):
        with tempfile.TemporaryDirectory() as td:
            raw = os.path.join(td, "uv.f64")
            np.ascontiguousarray(uv, np.float64).tofile(raw)
            d = ref("pad", str(w), str(h), raw)
        golden[f"pad{i}/size"] = np.array([w, h], np.int32)
        golden[f"pad{i}/uv"] = uv
        for k in ("padding", "padded", "unpadded"):
            golden[f"pad{i}/{k}"] = d[k]
    # vector file
    field = rng.normal(size=(11, 2))
    vfp = os.path.join(OUT, "field.vf")
    with open(vfp, "wb") as fh:
        fh.write(struct.pack("<i", len(field)) + field.astype("<f8").tobytes())
    golden["field/field"] = ref("vf", vfp)["field"]
    np.savez_compressed(os.path.join(OUT, "io_golden.npz"), **golden)

    # the reference's own data files, read by the reference
    data = {}
    droot = os.path.join(ref_tree, "Data")
    for sub in sorted(os.listdir(droot)):
        for fn in sorted(os.listdir(os.path.join(droot, sub))):
            p = os.path.join(droot, sub, fn)
            if fn.endswith(".ply"):
                d = ref("ply", p)
                data[f"{sub}/{fn}"] = {k: [list(d[k].shape), digest(d[k].astype({"triangles": np.int32}.get(k, np.float64)))]
                                       for k in ("vertices", "triangles", "uv")}
            elif fn.endswith(".vf"):
                d = ref("vf", p)
                data[f"{sub}/{fn}"] = {"field": [list(d["field"].shape), digest(d["field"])]}
    with open(os.path.join(OUT, "reference_data.json"), "w") as fh:
        json.dump(data, fh, indent=1, sort_keys=True)
    print(f"wrote {len(golden)} arrays and {len(data)} reference data digests to {OUT}")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(f"usage: python {sys.argv[0]} <reference checkout>")
    main(sys.argv[1])
