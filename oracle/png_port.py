"""PNG test vectors for the texture I/O path -- test infrastructure only.

The product decodes PNG natively (csrc/io/png.cpp).  This module is an
independent restatement, used only by the tests, of:

* the PNG format (ISO/IEC 15948: chunks with CRC-32, zlib stream, per-row
  filters 0-4, Adam7 interlacing) as an encoder of arbitrary sample arrays in
  every colour type and bit depth, with a chosen filter per row; and
* what the reference's ``PNGReadColor`` (include/Misha/PNG.inl:10-72) hands
  to ``Image<Point3D<float>>::read`` (include/Misha/Image.h:90-110) after its
  libpng transforms PNG_TRANSFORM_STRIP_16 (keep the high byte of 16-bit
  samples) and PNG_TRANSFORM_PACKING (1/2/4-bit samples unpacked to one byte
  each, not rescaled), palette indices looked up in PLTE, alpha ignored.  For
  grey images the reference fills only channel 0 (channels 1-2 are left
  uninitialised); the port copies grey to all three channels, the defined
  behaviour the product implements.
"""
from __future__ import annotations

import struct
import zlib

import numpy as np

CHANNELS = {0: 1, 2: 3, 3: 1, 4: 2, 6: 4}
ADAM7 = [(0, 0, 8, 8), (4, 0, 8, 8), (0, 4, 4, 8), (2, 0, 4, 4), (0, 2, 2, 4), (1, 0, 2, 2), (0, 1, 1, 2)]


def _chunk(tag: bytes, data: bytes) -> bytes:
    return struct.pack(">I", len(data)) + tag + data + struct.pack(">I", zlib.crc32(tag + data) & 0xFFFFFFFF)


def _pack_row(samples: np.ndarray, depth: int) -> bytes:
    """One row of samples (pixels x channels) at the given bit depth."""
    s = samples.reshape(-1).astype(np.int64)
    if depth == 16:
        return s.astype(">u2").tobytes()
    if depth == 8:
        return s.astype(np.uint8).tobytes()
    per = 8 // depth
    out = bytearray((len(s) + per - 1) // per)
    for i, v in enumerate(s):
        out[i // per] |= int(v) << (8 - depth * (i % per + 1))
    return bytes(out)


def _paeth(a: int, b: int, c: int) -> int:
    p = a + b - c
    pa, pb, pc = abs(p - a), abs(p - b), abs(p - c)
    return a if pa <= pb and pa <= pc else (b if pb <= pc else c)


def _filter(row: bytes, prev: bytes, ftype: int, bpp: int) -> bytes:
    out = bytearray(len(row))
    for i, x in enumerate(row):
        a = row[i - bpp] if i >= bpp else 0
        b = prev[i]
        c = prev[i - bpp] if i >= bpp else 0
        pred = (0, a, b, (a + b) >> 1, _paeth(a, b, c))[ftype]
        out[i] = (x - pred) & 0xFF
    return bytes(out)


def encode(samples: np.ndarray, colour_type: int, depth: int, palette: np.ndarray | None = None, interlace: bool = False,
           filters=(0, 1, 2, 3, 4), idat_split: int = 0) -> bytes:
    """PNG bytes for samples (h, w, channels) of the colour type; row r of each
    pass uses filter filters[r % len(filters)]."""
    h, w, ch = samples.shape
    assert ch == CHANNELS[colour_type]
    bpp = max(1, ch * depth // 8)
    raw = bytearray()
    passes = ADAM7 if interlace else [(0, 0, 1, 1)]
    for xs, ys, dx, dy in passes:
        sub = samples[ys::dy, xs::dx]
        if sub.shape[0] == 0 or sub.shape[1] == 0:
            continue
        prev = bytes(len(_pack_row(sub[0], depth)))
        for r in range(sub.shape[0]):
            row = _pack_row(sub[r], depth)
            f = filters[r % len(filters)]
            raw.append(f)
            raw += _filter(row, prev, f, bpp)
            prev = row
    z = zlib.compress(bytes(raw), 9)
    out = b"\x89PNG\r\n\x1a\n" + _chunk(b"IHDR", struct.pack(">IIBBBBB", w, h, depth, colour_type, 0, 0, 1 if interlace else 0))
    if colour_type == 3:
        out += _chunk(b"PLTE", np.asarray(palette, np.uint8).reshape(-1).tobytes())
    if idat_split:
        for o in range(0, len(z), idat_split):
            out += _chunk(b"IDAT", z[o:o + idat_split])
    else:
        out += _chunk(b"IDAT", z)
    return out + _chunk(b"IEND", b"")


def expected_rgb8(samples: np.ndarray, colour_type: int, depth: int, palette: np.ndarray | None = None) -> np.ndarray:
    """(h, w, 3) uint8 that the reference's read delivers for these samples."""
    s = samples.astype(np.int64)
    if depth == 16:
        s = s >> 8
    if colour_type == 3:
        return np.asarray(palette, np.uint8)[s[..., 0]]
    if colour_type in (0, 4):
        return np.repeat(s[..., :1], 3, axis=2).astype(np.uint8)
    return s[..., :3].astype(np.uint8)


def to_byte(v: np.ndarray) -> np.ndarray:
    """Image<Point3D<float>>::write's conversion (Image.h:152-163) in float32:
    min(255, max(0, (int)(v * 255 + 0.5)))."""
    t = (np.asarray(v, np.float32) * np.float32(255)).astype(np.float32)
    t = (t + np.float32(0.5)).astype(np.float32)
    return np.clip(np.trunc(t), 0, 255).astype(np.uint8)
