"""Texture I/O of the apps, through ``libgdtp.so`` (host only; no device needed).

Reference names and behaviour (fabianprada/GradientDomainTextureProcessing):

* ``ReadTexturedMesh`` / ``WriteTexturedMesh``  -- ``include/Src/SimpleMesh.h:93-160``
* ``read_image`` / ``write_image``              -- ``Image<Point3D<float>>::read/write``,
  ``include/Misha/Image.h:90-163`` (PNG via ``PNG.inl:10-120``; ``.normap`` via
  ``ReadBinaryImage`` / ``WriteBinaryImage``, ``include/Src/VectorIO.h:34-58``)
* ``ReadVector`` / ``WriteVector``              -- ``include/Src/VectorIO.h:9-32``
* ``ComputePadding``, ``PaddTextureCoordinates``, ``UnpaddTextureCoordinates``,
  ``PaddImage``, ``UnpaddImage``                -- ``include/Src/Padding.h:16-94``
* ``load_filtering_input``                      -- the input steps of the filtering
  app, ``TextureFiltering/TextureFiltering.cpp:807-837``
* ``texture_from_texels``                       -- ``UpdateFilteredTexture``,
  ``TextureFiltering.cpp:296-302``
* ``export_texture``                            -- ``ExportTextureCallBack``,
  ``TextureFiltering.cpp:479-499``

A mesh is the dict that :mod:`meshgen` produces and ``InitializeHierarchy``
takes: ``vertices`` (nv, 3) float64, ``triangles`` (nt, 3) int32, ``uv``
(nt, 3, 2) float64 per corner, ``texture`` (h, w, 3) float32 with texel
(ci, cj) at ``texture[cj, ci]`` (row 0 = the first PNG row).
"""
from __future__ import annotations

import ctypes as C
from typing import NamedTuple

import numpy as np

from . import _lib

__all__ = ["ReadTexturedMesh", "WriteTexturedMesh", "read_image", "write_image", "ReadVector", "WriteVector", "Padding",
           "ComputePadding", "PaddTextureCoordinates", "UnpaddTextureCoordinates", "PaddImage", "UnpaddImage",
           "prepare_filtering_mesh", "load_filtering_input", "texture_from_texels", "export_texture"]


def _path(p) -> bytes:
    return str(p).encode()


def ReadTexturedMesh(mesh_path, texture_path=None) -> dict:
    """Vertices, triangles and per-corner texture coordinates of a PLY file,
    plus the texture when ``texture_path`` is given (``.png`` or ``.normap``)."""
    L = _lib.lib()
    nv, nt = C.c_int64(0), C.c_int64(0)
    _lib.check(L.gdtp_read_textured_mesh(_path(mesh_path), C.byref(nv), C.byref(nt), None, None, None))
    v = np.empty((nv.value, 3), np.float64)
    t = np.empty((nt.value, 3), np.int32)
    uv = np.empty((nt.value, 3, 2), np.float64)
    _lib.check(L.gdtp_read_textured_mesh(_path(mesh_path), C.byref(nv), C.byref(nt), _lib.ptr(v), _lib.ptr(t), _lib.ptr(uv)))
    size = C.c_int64(0)
    _lib.check(L.gdtp_textured_mesh_texture_file(_path(mesh_path), None, C.byref(size)))
    name = C.create_string_buffer(size.value)
    _lib.check(L.gdtp_textured_mesh_texture_file(_path(mesh_path), name, C.byref(size)))
    mesh = {"vertices": v, "triangles": t, "uv": uv, "texture_file": name.value.decode()}
    if texture_path is not None:
        mesh["texture"] = read_image(texture_path)
    return mesh


def WriteTexturedMesh(path, mesh: dict, texture_file: str | None = None) -> None:
    v = np.ascontiguousarray(mesh["vertices"], np.float64).reshape(-1, 3)
    t = np.ascontiguousarray(mesh["triangles"], np.int32).reshape(-1, 3)
    uv = np.ascontiguousarray(mesh["uv"], np.float64).reshape(-1, 3, 2)
    if uv.shape[0] != t.shape[0]:
        raise ValueError("uv must hold 3 corners per triangle")
    name = None if texture_file is None else texture_file.encode()
    _lib.check(_lib.lib().gdtp_write_textured_mesh(_path(path), _lib.ptr(v), v.shape[0], _lib.ptr(t), t.shape[0], _lib.ptr(uv), name))


def read_image(path) -> np.ndarray:
    """(h, w, 3) float32: PNG bytes / 255, or a ``.normap``'s floats."""
    L = _lib.lib()
    w, h = C.c_int(0), C.c_int(0)
    _lib.check(L.gdtp_read_image(_path(path), C.byref(w), C.byref(h), None))
    img = np.empty((h.value, w.value, 3), np.float32)
    _lib.check(L.gdtp_read_image(_path(path), C.byref(w), C.byref(h), _lib.ptr(img)))
    return img


def write_image(path, img: np.ndarray) -> None:
    """(h, w, 3) values to ``.png`` (clamped, rounded to 8 bits) or ``.normap``."""
    a = np.ascontiguousarray(img, np.float32)
    if a.ndim != 3 or a.shape[2] != 3:
        raise ValueError("image must be (h, w, 3)")
    _lib.check(_lib.lib().gdtp_write_image(_path(path), _lib.ptr(a), a.shape[1], a.shape[0]))


def ReadVector(path, dtype=np.float64, width: int = 2) -> np.ndarray:
    """Elements of ``width`` values of ``dtype`` (Point2D<double> by default:
    the ``.vf`` tangent fields, one per triangle)."""
    dt = np.dtype(dtype)
    eb = dt.itemsize * width
    L = _lib.lib()
    n = C.c_int64(0)
    _lib.check(L.gdtp_read_vector(_path(path), eb, C.byref(n), None))
    out = np.empty((n.value, width), dt)
    _lib.check(L.gdtp_read_vector(_path(path), eb, C.byref(n), _lib.ptr(out)))
    return out if width > 1 else out[:, 0]


def WriteVector(path, vec: np.ndarray) -> None:
    a = np.ascontiguousarray(vec)
    n = a.shape[0] if a.ndim else 1
    eb = a.nbytes // max(n, 1) if n else a.dtype.itemsize
    _lib.check(_lib.lib().gdtp_write_vector(_path(path), eb, n, _lib.ptr(a)))


class Padding(NamedTuple):
    left: int = 0
    bottom: int = 0
    right: int = 0
    top: int = 0

    @property
    def nonTrivial(self) -> bool:
        return any(self)

    def _arr(self) -> np.ndarray:
        return np.asarray(self, dtype=np.int32)


def _uv_pairs(uv) -> np.ndarray:
    return np.ascontiguousarray(uv, np.float64).reshape(-1, 2)


def ComputePadding(width: int, height: int, uv) -> Padding:
    pairs = _uv_pairs(uv)
    p = np.zeros(4, np.int32)
    _lib.check(_lib.lib().gdtp_compute_padding(int(width), int(height), _lib.ptr(pairs), pairs.shape[0], _lib.ptr(p)))
    return Padding(*map(int, p))


def _pad_uv(padding: Padding, width: int, height: int, uv, unpad: int) -> np.ndarray:
    shape = np.shape(uv)
    pairs = _uv_pairs(uv).copy()
    pa = padding._arr()
    _lib.check(_lib.lib().gdtp_pad_texture_coordinates(_lib.ptr(pa), int(width), int(height), _lib.ptr(pairs), pairs.shape[0], unpad))
    return pairs.reshape(shape)


def PaddTextureCoordinates(padding: Padding, width: int, height: int, uv) -> np.ndarray:
    """Coordinates in the padded image; width, height: the unpadded size."""
    return _pad_uv(padding, width, height, uv, 0)


def UnpaddTextureCoordinates(padding: Padding, width: int, height: int, uv) -> np.ndarray:
    return _pad_uv(padding, width, height, uv, 1)


def _pad_img(padding: Padding, img: np.ndarray, unpad: int) -> np.ndarray:
    a = np.ascontiguousarray(img, np.float32)
    h, w = a.shape[:2]
    p = padding
    oh, ow = (h - p.bottom - p.top, w - p.left - p.right) if unpad else (h + p.bottom + p.top, w + p.left + p.right)
    if oh <= 0 or ow <= 0:
        raise ValueError("padding larger than the image")
    out = np.empty((oh, ow, 3), np.float32)
    pa = padding._arr()
    _lib.check(_lib.lib().gdtp_pad_image(_lib.ptr(pa), _lib.ptr(a), w, h, _lib.ptr(out), unpad))
    return out


def PaddImage(padding: Padding, img: np.ndarray) -> np.ndarray:
    return _pad_img(padding, img, 0)


def UnpaddImage(padding: Padding, img: np.ndarray) -> np.ndarray:
    return _pad_img(padding, img, 1)


def prepare_filtering_mesh(mesh: dict, width: int, height: int) -> tuple[dict, Padding, int, int]:
    """The apps' mesh preprocessing for a texture of width x height, the same in
    all three (TextureFiltering.cpp:814-837, Geodesics.cpp:788-809,
    LineIntegralConvolution.cpp:785-806): vertices centred and scaled to unit radius, v
    flipped, and texture coordinates (and the texture, if the mesh has one)
    padded when the atlas reaches within half a texel of the image edge or the
    size is not a multiple of 8.  The reference's optional random jitter
    (--jitter, unseeded) is not applied.  Returns the new mesh, the padding and
    the padded size."""
    m = dict(mesh)
    v = np.asarray(m["vertices"], np.float64)
    centroid = v.sum(axis=0) / v.shape[0]
    d = v - centroid
    radius = float(np.sqrt((d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1] + d[:, 2] * d[:, 2]).max())) if v.shape[0] else 1.0
    m["vertices"] = d / radius
    uv = np.array(m["uv"], np.float64)
    uv[..., 1] = 1.0 - uv[..., 1]
    padding = ComputePadding(width, height, uv)
    if padding.nonTrivial:
        uv = PaddTextureCoordinates(padding, width, height, uv)
        if m.get("texture") is not None:
            m["texture"] = PaddImage(padding, m["texture"])
    m["uv"] = uv
    return m, padding, width + padding.left + padding.right, height + padding.bottom + padding.top


def load_filtering_input(mesh_path, texture_path) -> tuple[dict, Padding]:
    """The filtering app's input steps (TextureFiltering.cpp:807-837): read the
    mesh and its texture, then prepare_filtering_mesh.  Returns the mesh
    (texture padded) and the padding to undo on export."""
    mesh = ReadTexturedMesh(mesh_path, texture_path)
    h, w = mesh["texture"].shape[:2]
    mesh, padding, _, _ = prepare_filtering_mesh(mesh, w, h)
    return mesh, padding


def texture_from_texels(hierarchy, x: np.ndarray, width: int, height: int, background: float = 0.5,
                        padding: Padding | None = None) -> np.ndarray:
    """UpdateFilteredTexture (TextureFiltering.cpp:296-302, 712-713): an image
    of the padded size filled with ``background``, each active texel's value at
    its (ci, cj); with ``padding`` the result is cropped back (UnpaddImage, as
    the export does, :479-482)."""
    tn = hierarchy.array("textureNodes")
    x = np.asarray(x, np.float32).reshape(tn.shape[0], -1)
    img = np.full((height, width, 3), background, np.float32)
    img[tn[:, 1], tn[:, 0], :] = x[:, :3] if x.shape[1] >= 3 else np.repeat(x[:, :1], 3, axis=1)
    if padding is not None and padding.nonTrivial:
        img = UnpaddImage(padding, img)
    return img


def export_texture(path, img: np.ndarray, padding: Padding | None = None, normal: bool = False) -> None:
    """ExportTextureCallBack (TextureFiltering.cpp:479-499): crop the padding
    back, then ".png" gets the 8-bit colour write; for a normal texture each
    pixel is first normalised and mapped to v * 0.5 + 0.5 (float32).  Any other
    extension gets the raw layout of WriteBinaryImage (int32 width, int32
    height, float RGB), whatever the name."""
    out = np.ascontiguousarray(img, np.float32)
    if padding is not None and padding.nonTrivial:
        out = UnpaddImage(padding, out)
    if str(path).lower().endswith(".png"):
        if normal:
            length = np.sqrt(out[..., 0] * out[..., 0] + out[..., 1] * out[..., 1] + out[..., 2] * out[..., 2])
            out = (out / length[..., None]) * np.float32(0.5) + np.float32(0.5)
        write_image(path, out)
        return
    h, w = out.shape[:2]
    with open(path, "wb") as fh:
        fh.write(np.array([w, h], "<i4").tobytes() + out.astype("<f4").tobytes())
