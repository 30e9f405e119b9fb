"""Texture I/O (host, no GPU): PLY meshes, PNG / normap textures, .vf vectors and
atlas padding against the reference's own readers and helpers.

* PLY, padding and vectors: bit-exact against golden arrays that the
  reference's ReadTexturedMesh / ReadVector / Padding.h produced
  (tests/golden/make_io_golden.py with oracle/ref_io.cpp), and against digests
  of what the reference reads from its shipped data files (checked when that
  data is present).
* PNG: libpng is not in this image, so the reference's PNGReadColor cannot run
  here.  Decoding is checked against oracle/png_port.py, an independent
  restatement of the PNG format and of the reference's libpng transforms, over
  every colour type, bit depth, filter and Adam7, and against PIL.  Encoding is
  checked by decoding with PIL.
"""
import hashlib
import json
import os
import struct
import zlib

import numpy as np
import pytest

from conftest import GOLDEN, reference_data

IO = os.path.join(GOLDEN, "io")
REFERENCE_DATA = reference_data()


@pytest.fixture(scope="module")
def tio(built_lib):
    from gradientdomaintextureprocessing_b200 import textureio
    return textureio


@pytest.fixture(scope="module")
def golden():
    with np.load(os.path.join(IO, "io_golden.npz")) as z:
        return {k: z[k] for k in z.files}


# ---------------------------------------------------------------- PLY meshes

@pytest.mark.parametrize("name", ["ascii_double", "ascii_float", "binary_le", "binary_be", "ref_written"])
def test_ply_matches_reference_reader(tio, golden, name):
    m = tio.ReadTexturedMesh(os.path.join(IO, f"{name}.ply"))
    np.testing.assert_array_equal(m["vertices"], golden[f"{name}/vertices"])
    np.testing.assert_array_equal(m["triangles"], golden[f"{name}/triangles"])
    np.testing.assert_array_equal(m["uv"].reshape(-1, 2), golden[f"{name}/uv"])


def test_ply_sized_type_names(tio, golden):
    """float64 / float32 / int16 columns (the reference's PLY library aborts on
    this file): the values written into it."""
    m = tio.ReadTexturedMesh(os.path.join(IO, "binary_le_sized_names.ply"))
    np.testing.assert_array_equal(m["vertices"], golden["sized_names/vertices"])
    np.testing.assert_array_equal(m["triangles"], golden["sized_names/triangles"])
    np.testing.assert_array_equal(m["uv"].reshape(-1, 2), golden["sized_names/uv"])


def test_ply_texture_file_comment(tio):
    assert tio.ReadTexturedMesh(os.path.join(IO, "ref_written.ply"))["texture_file"] == "atlas.png"
    assert tio.ReadTexturedMesh(os.path.join(IO, "ascii_double.ply"))["texture_file"] == "atlas texture.png"
    assert tio.ReadTexturedMesh(os.path.join(IO, "binary_le.ply"))["texture_file"] == ""


def test_ply_write_read_round_trip_is_bit_exact(tio, tmp_path):
    from gradientdomaintextureprocessing_b200 import meshgen
    mesh = meshgen.torus_atlas(64, 64)
    p = tmp_path / "torus.ply"
    tio.WriteTexturedMesh(p, mesh, texture_file="torus.png")
    back = tio.ReadTexturedMesh(p)
    np.testing.assert_array_equal(back["vertices"], mesh["vertices"])
    np.testing.assert_array_equal(back["triangles"], mesh["triangles"])
    np.testing.assert_array_equal(back["uv"], mesh["uv"])
    assert back["texture_file"] == "torus.png"


def _reference_files():
    with open(os.path.join(IO, "reference_data.json")) as fh:
        return json.load(fh)


@pytest.mark.skipif(not os.path.isdir(REFERENCE_DATA), reason="the reference's data files are not present")
@pytest.mark.parametrize("name", sorted(_reference_files()))
def test_reference_data_files_read_as_the_reference_reads_them(tio, name):
    want = _reference_files()[name]
    path = os.path.join(REFERENCE_DATA, name)
    if name.endswith(".ply"):
        m = tio.ReadTexturedMesh(path)
        got = {"vertices": m["vertices"], "triangles": m["triangles"], "uv": m["uv"].reshape(-1, 2)}
    else:
        got = {"field": tio.ReadVector(path)}
    for k, (shape, digest) in want.items():
        assert list(got[k].shape) == shape, k
        assert hashlib.sha256(np.ascontiguousarray(got[k]).tobytes()).hexdigest() == digest, k


def test_ply_errors(tio, tmp_path):
    from gradientdomaintextureprocessing_b200._lib import GDTPError
    with pytest.raises(GDTPError, match="cannot open"):
        tio.ReadTexturedMesh(tmp_path / "missing.ply")
    bad = tmp_path / "notex.ply"
    bad.write_text("ply\nformat ascii 1.0\nelement vertex 3\nproperty float x\nproperty float y\nproperty float z\n"
                   "element face 1\nproperty list uchar int vertex_indices\nend_header\n0 0 0\n1 0 0\n0 1 0\n3 0 1 2\n")
    with pytest.raises(GDTPError, match="texcoord"):
        tio.ReadTexturedMesh(bad)
    out = tmp_path / "range.ply"
    out.write_text("ply\nformat ascii 1.0\nelement vertex 3\nproperty float x\nproperty float y\nproperty float z\n"
                   "element face 1\nproperty list uchar int vertex_indices\nproperty list uchar float texcoord\nend_header\n"
                   "0 0 0\n1 0 0\n0 1 0\n3 0 1 5 6 0 0 1 0 0 1\n")
    with pytest.raises(GDTPError, match="out of range"):
        tio.ReadTexturedMesh(out)
    short = tmp_path / "short.ply"
    short.write_bytes((IO and open(os.path.join(IO, "binary_le.ply"), "rb").read())[:-9])
    with pytest.raises(GDTPError, match="ends early"):
        tio.ReadTexturedMesh(short)


# ---------------------------------------------------------------- vectors

def test_vector_matches_reference_reader(tio, golden, tmp_path):
    f = tio.ReadVector(os.path.join(IO, "field.vf"))
    np.testing.assert_array_equal(f, golden["field/field"])
    tio.WriteVector(tmp_path / "f.vf", f)
    assert (tmp_path / "f.vf").read_bytes() == open(os.path.join(IO, "field.vf"), "rb").read()
    ints = np.arange(5, dtype=np.int32)
    tio.WriteVector(tmp_path / "i.bin", ints)
    np.testing.assert_array_equal(tio.ReadVector(tmp_path / "i.bin", np.int32, 1), ints)


def test_vector_agrees_with_the_generator_format(tio, tmp_path):
    from gradientdomaintextureprocessing_b200 import meshgen
    field = meshgen.gaussian_bump_field(meshgen.torus_atlas(32, 32))
    meshgen.write_vf(str(tmp_path / "g.vf"), field)
    np.testing.assert_array_equal(tio.ReadVector(tmp_path / "g.vf"), np.asarray(field).reshape(-1, 2))


def test_vector_errors(tio, tmp_path):
    from gradientdomaintextureprocessing_b200._lib import GDTPError
    p = tmp_path / "t.vf"
    p.write_bytes(struct.pack("<i", 4) + b"\0" * 40)
    with pytest.raises(GDTPError, match="shorter than its count"):
        tio.ReadVector(p)


# ---------------------------------------------------------------- padding

@pytest.mark.parametrize("case", range(5))
def test_padding_matches_reference(tio, golden, case):
    w, h = map(int, golden[f"pad{case}/size"])
    uv = golden[f"pad{case}/uv"]
    p = tio.ComputePadding(w, h, uv)
    want = golden[f"pad{case}/padding"].ravel()
    assert list(p) == list(want[:4]) and p.nonTrivial == bool(want[4])
    padded = tio.PaddTextureCoordinates(p, w, h, uv)
    np.testing.assert_array_equal(padded, golden[f"pad{case}/padded"])
    np.testing.assert_array_equal(tio.UnpaddTextureCoordinates(p, w, h, padded), golden[f"pad{case}/unpadded"])


def test_pad_and_unpad_image(tio):
    """PaddImage repeats the edge texels (Padding.h:48-60), UnpaddImage crops (:62-73)."""
    rng = np.random.default_rng(3)
    img = rng.random((5, 7, 3)).astype(np.float32)
    p = tio.Padding(left=2, bottom=1, right=3, top=4)
    padded = tio.PaddImage(p, img)
    assert padded.shape == (5 + 1 + 4, 7 + 2 + 3, 3)
    jj = np.clip(np.arange(padded.shape[0]) - p.bottom, 0, 4)
    ii = np.clip(np.arange(padded.shape[1]) - p.left, 0, 6)
    np.testing.assert_array_equal(padded, img[jj][:, ii])
    np.testing.assert_array_equal(tio.UnpaddImage(p, padded), img)


# ---------------------------------------------------------------- images

def _write(tmp_path, name, data: bytes):
    p = tmp_path / name
    p.write_bytes(data)
    return p


CASES = [(0, 1), (0, 2), (0, 4), (0, 8), (0, 16), (2, 8), (2, 16), (3, 1), (3, 2), (3, 4), (3, 8), (4, 8), (4, 16), (6, 8), (6, 16)]


@pytest.mark.parametrize("interlace", [False, True])
@pytest.mark.parametrize("ctype,depth", CASES)
def test_png_decoder_matches_the_format_port(tio, tmp_path, ctype, depth, interlace):
    import png_port
    rng = np.random.default_rng(ctype * 100 + depth)
    h, w = 13, 11  # odd sizes: partial bytes and every Adam7 pass non-empty but ragged
    ch = png_port.CHANNELS[ctype]
    palette = None
    if ctype == 3:
        palette = rng.integers(0, 256, size=(1 << depth, 3))
        samples = rng.integers(0, 1 << depth, size=(h, w, 1))
    else:
        samples = rng.integers(0, 1 << depth, size=(h, w, ch))
    data = png_port.encode(samples, ctype, depth, palette, interlace=interlace, idat_split=37)
    img = tio.read_image(_write(tmp_path, "t.png", data))
    want = png_port.expected_rgb8(samples, ctype, depth, palette).astype(np.float32) / np.float32(255)
    np.testing.assert_array_equal(img, want)


@pytest.mark.parametrize("mode", ["RGB", "RGBA", "L", "LA", "P"])
def test_png_decoder_matches_pil(tio, tmp_path, mode):
    from PIL import Image
    rng = np.random.default_rng(5)
    rgb = rng.integers(0, 256, size=(40, 57, 3), dtype=np.uint8)
    im = Image.fromarray(rgb, "RGB")
    im = im.convert(mode) if mode != "P" else im.quantize(colors=200)
    p = tmp_path / f"pil_{mode}.png"
    im.save(p, optimize=False)
    got = tio.read_image(p)
    ref = np.asarray(im.convert("RGB") if mode in ("RGB", "RGBA", "P") else im.convert("L"), np.uint8)
    if ref.ndim == 2:
        ref = np.repeat(ref[..., None], 3, axis=2)
    np.testing.assert_array_equal(got, ref.astype(np.float32) / np.float32(255))


def test_png_write_is_the_reference_conversion_and_pil_reads_it(tio, tmp_path):
    import png_port
    from PIL import Image
    rng = np.random.default_rng(9)
    img = rng.uniform(-0.2, 1.2, size=(31, 45, 3)).astype(np.float32)
    img[0, :6, 0] = [0.5 / 255, 1.5 / 255, 254.5 / 255, np.float32(0.99803925), -1e-9, 1.0]
    p = tmp_path / "out.png"
    tio.write_image(p, img)
    with Image.open(p) as im:
        assert im.mode == "RGB" and im.size == (45, 31)
        pil = np.asarray(im)
    want = png_port.to_byte(img)
    np.testing.assert_array_equal(pil, want)
    np.testing.assert_array_equal(tio.read_image(p), want.astype(np.float32) / np.float32(255))


def test_png_large_image_round_trip(tio, tmp_path):
    """Row filters over a 2048-wide photo-like image; several IDAT chunks."""
    from gradientdomaintextureprocessing_b200 import meshgen
    mesh = meshgen.icosphere_atlas(512, 512, subdiv=3, seed=1)
    img = np.ascontiguousarray(mesh["texture"][..., :3], np.float32)
    p = tmp_path / "big.png"
    tio.write_image(p, img)
    import png_port
    np.testing.assert_array_equal(tio.read_image(p), png_port.to_byte(img).astype(np.float32) / np.float32(255))


def test_normap_round_trip_and_layout(tio, tmp_path):
    rng = np.random.default_rng(2)
    img = rng.normal(size=(6, 9, 3)).astype(np.float32)
    p = tmp_path / "n.normap"
    tio.write_image(p, img)
    raw = p.read_bytes()
    assert struct.unpack("<ii", raw[:8]) == (9, 6) and len(raw) == 8 + img.nbytes
    np.testing.assert_array_equal(np.frombuffer(raw[8:], np.float32).reshape(6, 9, 3), img)
    np.testing.assert_array_equal(tio.read_image(p), img)


def test_image_errors(tio, tmp_path):
    import png_port
    from gradientdomaintextureprocessing_b200._lib import GDTPError
    good = png_port.encode(np.zeros((4, 4, 3), np.int64), 2, 8)
    with pytest.raises(GDTPError, match="extension"):
        tio.read_image(_write(tmp_path, "x.jpg", good))
    with pytest.raises(GDTPError, match="not a PNG"):
        tio.read_image(_write(tmp_path, "x.png", b"GIF89a" + good))
    corrupt = bytearray(good)
    corrupt[45] ^= 0xFF  # inside the IDAT data: its CRC no longer matches
    with pytest.raises(GDTPError, match="CRC"):
        tio.read_image(_write(tmp_path, "c.png", bytes(corrupt)))
    with pytest.raises(GDTPError, match="IEND"):
        tio.read_image(_write(tmp_path, "t.png", good[:-12]))
    pal = png_port.encode(np.full((2, 2, 1), 3, np.int64), 3, 2, palette=np.zeros((2, 3), np.int64))
    with pytest.raises(GDTPError, match="palette index"):
        tio.read_image(_write(tmp_path, "p.png", pal))
    # image data shorter than the header promises
    short = (b"\x89PNG\r\n\x1a\n" + png_port._chunk(b"IHDR", struct.pack(">IIBBBBB", 8, 8, 8, 2, 0, 0, 0)) +
             png_port._chunk(b"IDAT", zlib.compress(b"\0" * 20)) + png_port._chunk(b"IEND", b""))
    with pytest.raises(GDTPError, match="too short"):
        tio.read_image(_write(tmp_path, "s.png", short))


# ---------------------------------------------------------------- app input / output

def test_filtering_input_and_export(tio, tmp_path):
    """load_filtering_input: vertices centred and scaled to unit radius, v
    flipped, padding applied (TextureFiltering.cpp:807-837); texture_from_texels
    writes texel values at (ci, cj) and crops the padding back."""
    from gradientdomaintextureprocessing_b200 import meshgen
    from gradientdomaintextureprocessing_b200.hierarchy import InitializeHierarchy
    mesh = meshgen.torus_atlas(100, 60)
    tio.WriteTexturedMesh(tmp_path / "m.ply", mesh)
    tex = np.ascontiguousarray(mesh["texture"][..., :3] if mesh["texture"].shape[2] >= 3 else
                               np.repeat(mesh["texture"][..., :1], 3, axis=2), np.float32)
    tio.write_image(tmp_path / "m.png", tex)
    m, pad = tio.load_filtering_input(tmp_path / "m.ply", tmp_path / "m.png")
    v = mesh["vertices"]
    c = v.sum(axis=0) / v.shape[0]
    r = np.sqrt(((v - c) ** 2).sum(axis=1)).max()
    np.testing.assert_allclose(m["vertices"], (v - c) / r, rtol=0, atol=1e-15)
    assert pad == tio.ComputePadding(100, 60, np.stack([mesh["uv"][..., 0], 1.0 - mesh["uv"][..., 1]], -1))
    assert pad.nonTrivial  # 100 x 60 is not a multiple of 8 in both directions
    H, W = m["texture"].shape[:2]
    assert (W, H) == (100 + pad.left + pad.right, 60 + pad.bottom + pad.top) and W % 8 == 0 and H % 8 == 0
    flipped = np.stack([mesh["uv"][..., 0], 1.0 - mesh["uv"][..., 1]], -1)
    np.testing.assert_array_equal(m["uv"], tio.PaddTextureCoordinates(pad, 100, 60, flipped))
    h = InitializeHierarchy(m, levels=2)
    tn = h.array("textureNodes")
    x = np.random.default_rng(0).random((tn.shape[0], 3))
    out = tio.texture_from_texels(h, x, W, H, padding=pad)
    assert out.shape == (60, 100, 3)
    full = tio.texture_from_texels(h, x, W, H)
    np.testing.assert_array_equal(full[tn[:, 1], tn[:, 0]], x.astype(np.float32))
    np.testing.assert_array_equal(out, full[pad.bottom:pad.bottom + 60, pad.left:pad.left + 100])


def test_export_texture(tio, tmp_path):
    """ExportTextureCallBack: colour PNG as written; normal maps normalised and
    mapped to [0, 1] first; other extensions in the raw normap layout."""
    import png_port
    rng = np.random.default_rng(4)
    img = rng.normal(size=(12, 20, 3)).astype(np.float32)
    pad = tio.Padding(left=3, bottom=2, right=1, top=0)
    tio.export_texture(tmp_path / "c.png", img, padding=pad)
    crop = img[2:12, 3:19]
    np.testing.assert_array_equal(tio.read_image(tmp_path / "c.png"), png_port.to_byte(crop).astype(np.float32) / np.float32(255))
    tio.export_texture(tmp_path / "n.png", img, normal=True)
    n = img / np.sqrt((img * img).sum(axis=2, keepdims=True))
    want = png_port.to_byte((n * np.float32(0.5) + np.float32(0.5)).astype(np.float32))
    got = np.rint(tio.read_image(tmp_path / "n.png") * 255).astype(np.int32)
    assert np.abs(got - want.astype(np.int32)).max() <= 1  # the norm's last bit may round a byte the other way
    tio.export_texture(tmp_path / "raw.bin", img, padding=pad)
    raw = (tmp_path / "raw.bin").read_bytes()
    assert struct.unpack("<ii", raw[:8]) == (16, 10)
    np.testing.assert_array_equal(np.frombuffer(raw[8:], np.float32).reshape(10, 16, 3), crop)


def test_ply_counts_beyond_the_file_are_rejected(tio, tmp_path):
    """A header that declares more data than the file holds is an error, not an
    allocation of the declared size."""
    from gradientdomaintextureprocessing_b200._lib import GDTPError
    p = tmp_path / "huge.ply"
    p.write_bytes(b"ply\nformat binary_little_endian 1.0\nelement vertex 4000000000000\nproperty float x\n"
                  b"property float y\nproperty float z\nelement face 1\nproperty list uchar int vertex_indices\n"
                  b"property list uchar float texcoord\nend_header\n" + b"\0" * 64)
    with pytest.raises(GDTPError, match="exceed the file size"):
        tio.ReadTexturedMesh(p)



def test_sizes_that_would_overflow_are_errors(tio, tmp_path, golden):
    """Element sizes, texture coordinates and paddings whose products overflow
    are rejected (the padding of valid inputs is unchanged)."""
    import ctypes as C
    from gradientdomaintextureprocessing_b200 import _lib
    from gradientdomaintextureprocessing_b200._lib import GDTPError
    L = _lib.lib()
    n = C.c_int64(0)
    assert L.gdtp_read_vector(os.path.join(IO, "field.vf").encode(), 1 << 60, C.byref(n), None) == -1
    with pytest.raises(GDTPError, match="not finite or beyond"):
        tio.ComputePadding(256, 256, np.array([[0.5, 0.5], [np.inf, 0.5]]))
    with pytest.raises(GDTPError, match="beyond 2"):
        tio.ComputePadding(1 << 24, 256, np.array([[0.5, 0.5], [1e5, 0.5]]))
    pad = np.array([1 << 30, 0, 1 << 30, 0], np.int32)
    img = np.zeros((4, 4, 3), np.float32)
    out = np.zeros(3, np.float32)
    assert L.gdtp_pad_image(_lib.ptr(pad), _lib.ptr(img), 4, 4, _lib.ptr(out), 0) == -1
    assert "2^24" in L.gdtp_last_error().decode()
    w, h = map(int, golden["pad1/size"])
    assert list(tio.ComputePadding(w, h, golden["pad1/uv"])) == list(golden["pad1/padding"].ravel()[:4])


def test_normap_header_larger_than_the_file(tio, tmp_path):
    from gradientdomaintextureprocessing_b200._lib import GDTPError
    p = tmp_path / "big.normap"
    p.write_bytes(struct.pack("<ii", 2_000_000_000, 2_000_000_000) + b"\0" * 48)
    with pytest.raises(GDTPError, match="truncated"):
        tio.read_image(p)
