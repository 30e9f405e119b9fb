"""Deterministic synthetic textured meshes with multi-chart atlases.

The reference reads PLY meshes with per-corner texture coordinates and a PNG
texture (``Src/SimpleMesh.h:118-160``).  No data set is shipped for the solve
path, so the workloads are generated here from a seed:

* ``torus_atlas``      -- torus R=1, r=0.4, 64x32 quads (4096 triangles), four
                          rectangular charts packed into the unit square.
* ``icosphere_atlas``  -- icosphere subdivided 6 times (81,920 triangles),
                          vertex positions jittered N(0, 1e-3), 16 latitude /
                          longitude band charts (8 polar pie slices, 8
                          equatorial rectangles) packed on a 4x4 grid.
* ``genus2_atlas``     -- two tori joined by a tube (genus 2, ~200k
                          triangles), 32 charts packed on an 8x4 grid, with
                          ``gaussian_bump_field`` as its tangent field.

Every chart is separated from its neighbours and from the border of the unit
square by a gutter of at least ``gutter`` texels.  A mesh is a dict of numpy
arrays::

    vertices   (nv, 3) float64
    triangles  (nt, 3) int32      -- counter-clockwise in texture space
    uv         (nt, 3, 2) float64 -- per-corner texture coordinates in [0,1]^2
    texture    (h, w, c) float32  -- texel (ci, cj) is texture[cj, ci]

Texture coordinates are kept at least ``1e-4`` texels away from texel-centre
grid lines of the finest grid, so the reference's automatic grid-line
jitter (``Src/AtlasMesh.inl:36-55``, seeded by ``rand()``) never triggers and
the atlas is reproducible bit for bit.
"""
from __future__ import annotations

import struct

import numpy as np

__all__ = ["torus_atlas", "icosphere_atlas", "genus2_atlas", "gaussian_bump_field", "value_noise", "write_gdm",
           "read_gdm", "write_vf", "read_vf", "chart_ids"]


# ----------------------------------------------------------------------------
# texture signals
# ----------------------------------------------------------------------------

def value_noise(rng: np.random.Generator, width: int, height: int, channels: int,
                lattice: int = 32) -> np.ndarray:
    """Smooth value noise in [0,1]: random lattice values, smoothstep blended."""
    lat = rng.random((lattice + 1, lattice + 1, channels))
    xs = (np.arange(width) + 0.5) / width * lattice
    ys = (np.arange(height) + 0.5) / height * lattice
    x0 = np.minimum(np.floor(xs).astype(np.int64), lattice - 1)
    y0 = np.minimum(np.floor(ys).astype(np.int64), lattice - 1)
    fx = xs - x0
    fy = ys - y0
    sx = fx * fx * (3 - 2 * fx)
    sy = fy * fy * (3 - 2 * fy)
    a = lat[y0][:, x0]
    b = lat[y0][:, x0 + 1]
    c = lat[y0 + 1][:, x0]
    d = lat[y0 + 1][:, x0 + 1]
    sx = sx[None, :, None]
    sy = sy[:, None, None]
    top = a * (1 - sx) + b * sx
    bot = c * (1 - sx) + d * sx
    return (top * (1 - sy) + bot * sy).astype(np.float64)


# ----------------------------------------------------------------------------
# helpers
# ----------------------------------------------------------------------------

def _keep_off_texel_grid(uv: np.ndarray, width: int, height: int) -> np.ndarray:
    """Move coordinates closer than 1e-4 texel to a texel-centre line by 1e-3 texel."""
    uv = uv.copy()
    for c, dim in ((0, width), (1, height)):
        scaled = uv[..., c] * dim - 0.5
        off = scaled - np.round(scaled)
        bad = np.abs(off) < 1e-4
        if np.any(bad):
            scaled = np.where(bad, np.round(scaled) + np.where(off >= 0, 1e-3, -1e-3), scaled)
            uv[..., c] = (scaled + 0.5) / dim
    return uv


def _pack_charts(chart_uv: list[np.ndarray], grid: tuple[int, int], width: int, height: int,
                 gutter: int) -> list[np.ndarray]:
    """Place charts (arrays of local coordinates) on a gx x gy grid of cells.

    One common scale factor keeps relative chart areas; each chart is centred in
    its cell and kept ``gutter`` texels away from the cell border.
    """
    gx, gy = grid
    cw, ch = 1.0 / gx, 1.0 / gy
    inner_w = cw - 2.0 * gutter / width
    inner_h = ch - 2.0 * gutter / height
    scale = np.inf
    for p in chart_uv:
        ext = p.reshape(-1, 2).max(0) - p.reshape(-1, 2).min(0)
        scale = min(scale, inner_w / ext[0], inner_h / ext[1])
    out = []
    for k, p in enumerate(chart_uv):
        cx, cy = k % gx, k // gx
        flat = p.reshape(-1, 2)
        mid = 0.5 * (flat.max(0) + flat.min(0))
        centre = np.array([(cx + 0.5) * cw, (cy + 0.5) * ch])
        out.append((p - mid) * scale + centre)
    return out


def chart_ids(triangles: np.ndarray, uv: np.ndarray) -> np.ndarray:
    """Edge-connected components of triangles whose shared edges carry equal UVs.

    Same rule as ``Src/ChartDecomposition.h:30-73``; used to validate generators.
    """
    nt = len(triangles)
    parent = np.arange(nt)

    def find(a):
        while parent[a] != a:
            parent[a] = parent[parent[a]]
            a = parent[a]
        return a

    edge = {}
    for t in range(nt):
        for k in range(3):
            edge[(int(triangles[t, k]), int(triangles[t, (k + 1) % 3]))] = (t, k)
    for t in range(nt):
        for k in range(3):
            a, b = int(triangles[t, k]), int(triangles[t, (k + 1) % 3])
            o = edge.get((b, a))
            if o is None:
                continue
            s, m = o
            if (np.array_equal(uv[t, (k + 1) % 3], uv[s, m]) and np.array_equal(uv[t, k], uv[s, (m + 1) % 3])):
                ra, rb = find(t), find(s)
                if ra != rb:
                    parent[ra] = rb
    roots = np.array([find(t) for t in range(nt)])
    _, ids = np.unique(roots, return_inverse=True)
    return ids.astype(np.int32)


# ----------------------------------------------------------------------------
# torus, four rectangular charts
# ----------------------------------------------------------------------------

def torus_atlas(width: int = 256, height: int = 256, nu: int = 64, nv: int = 32,
                R: float = 1.0, r: float = 0.4, seed: int = 0, gutter: int = 8,
                jitter: float = 0.3, texture: str = "uniform_u8") -> dict:
    rng = np.random.default_rng(seed)
    i, j = np.meshgrid(np.arange(nu), np.arange(nv), indexing="xy")
    u = i / nu
    v = j / nv
    pos = np.stack([(R + r * np.cos(2 * np.pi * v)) * np.cos(2 * np.pi * u),
                    (R + r * np.cos(2 * np.pi * v)) * np.sin(2 * np.pi * u),
                    r * np.sin(2 * np.pi * v)], -1).reshape(-1, 3)

    def vid(a, b):
        return (b % nv) * nu + (a % nu)

    tris, corners = [], []
    for jj in range(nv):
        for ii in range(nu):
            a, b, c, d = (ii, jj), (ii + 1, jj), (ii + 1, jj + 1), (ii, jj + 1)
            for tri in ((a, b, c), (a, c, d)):
                tris.append([vid(*p) for p in tri])
                corners.append(tri)
    tris = np.array(tris, dtype=np.int32)
    corners = np.array(corners, dtype=np.float64)          # (nt,3,2) integer grid coords
    hu, hv = nu // 2, nv // 2
    cell = np.stack([np.minimum(corners[:, :, 0].min(1) // hu, 1),
                     np.minimum(corners[:, :, 1].min(1) // hv, 1)], -1).astype(np.int64)
    chart = cell[:, 1] * 2 + cell[:, 0]
    local = np.empty_like(corners)
    local[..., 0] = (corners[..., 0] - hu * cell[:, None, 0]) / hu
    local[..., 1] = (corners[..., 1] - hv * cell[:, None, 1]) / hv
    # place the four charts on a 2x2 grid, keep the torus aspect (u spans 2*pi*R, v 2*pi*r)
    inner_w = 0.5 - 2.0 * gutter / width
    inner_h = 0.5 - 2.0 * gutter / height
    uv = np.empty_like(local)
    uv[..., 0] = cell[:, None, 0] * 0.5 + gutter / width + local[..., 0] * inner_w
    uv[..., 1] = cell[:, None, 1] * 0.5 + gutter / height + local[..., 1] * inner_h
    # jitter every chart vertex (same jitter for all corners of one chart vertex)
    key = (chart[:, None] * (nu + 1) * (nv + 1) + corners[..., 1].astype(np.int64) * (nu + 1)
           + corners[..., 0].astype(np.int64))
    ukeys, inv = np.unique(key.reshape(-1), return_inverse=True)
    jit = rng.uniform(-jitter, jitter, size=(len(ukeys), 2)) / np.array([width, height])
    uv = uv + jit[inv].reshape(uv.shape)
    uv = _keep_off_texel_grid(uv, width, height)
    if texture == "uniform_u8":
        tex = (rng.integers(0, 256, size=(height, width, 3)).astype(np.float32) / 255.0)
    else:
        tex = value_noise(rng, width, height, 3).astype(np.float32)
    return {"vertices": pos.astype(np.float64), "triangles": tris, "uv": uv,
            "texture": tex, "name": f"torus{nu}x{nv}_{width}x{height}"}


# ----------------------------------------------------------------------------
# icosphere, 16 latitude / longitude charts
# ----------------------------------------------------------------------------

def _icosphere(subdiv: int):
    t = (1.0 + 5 ** 0.5) / 2.0
    v = np.array([[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0],
                  [0, -1, t], [0, 1, t], [0, -1, -t], [0, 1, -t],
                  [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]], dtype=np.float64)
    f = np.array([[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11],
                  [1, 5, 9], [5, 11, 4], [11, 10, 2], [10, 7, 6], [7, 1, 8],
                  [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9],
                  [4, 9, 5], [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1]], dtype=np.int64)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    for _ in range(subdiv):
        e = np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]], 0)
        es = np.sort(e, 1)
        uniq, inv = np.unique(es, axis=0, return_inverse=True)
        mid = v[uniq[:, 0]] + v[uniq[:, 1]]
        mid /= np.linalg.norm(mid, axis=1, keepdims=True)
        m = inv.reshape(3, -1).T + len(v)
        v = np.concatenate([v, mid], 0)
        a, b, c = f[:, 0], f[:, 1], f[:, 2]
        ab, bc, ca = m[:, 0], m[:, 1], m[:, 2]
        f = np.concatenate([np.stack([a, ab, ca], 1), np.stack([b, bc, ab], 1),
                            np.stack([c, ca, bc], 1), np.stack([ab, bc, ca], 1)], 0)
    return v, f


def _triangle_adjacency(f: np.ndarray) -> np.ndarray:
    """(nt,3) neighbour across edge k (k -> k+1), -1 if none."""
    nt = len(f)
    e = np.stack([f, np.roll(f, -1, 1)], -1).reshape(-1, 2)
    key = e[:, 0] * (f.max() + 1) + e[:, 1]
    rkey = e[:, 1] * (f.max() + 1) + e[:, 0]
    order = np.argsort(key)
    pos = np.searchsorted(key[order], rkey)
    pos = np.minimum(pos, len(key) - 1)
    hit = key[order][pos] == rkey
    nb = np.where(hit, order[pos] // 3, -1)
    return nb.reshape(nt, 3)


def icosphere_atlas(width: int = 2048, height: int = 2048, subdiv: int = 6, seed: int = 0,
                    sigma: float = 1e-3, gutter: int = 8, channels: int = 3) -> dict:
    rng = np.random.default_rng(seed)
    v, f = _icosphere(subdiv)
    v = v + rng.normal(0.0, sigma, size=v.shape)
    dirs = v / np.linalg.norm(v, axis=1, keepdims=True)
    cen = dirs[f].mean(1)
    cen /= np.linalg.norm(cen, axis=1, keepdims=True)
    lat = np.arcsin(np.clip(cen[:, 2], -1, 1))
    lon = np.arctan2(cen[:, 1], cen[:, 0])
    lat_bin = np.clip(((lat + np.pi / 2) // (np.pi / 4)).astype(np.int64), 0, 3)
    lon_bin = np.clip(((lon + np.pi) // (np.pi / 2)).astype(np.int64), 0, 3)
    chart = lat_bin * 4 + lon_bin
    nb = _triangle_adjacency(f)
    # smooth jagged borders: adopt a chart shared by two or more edge neighbours
    for _ in range(50):
        nc = np.where(nb >= 0, chart[np.maximum(nb, 0)], -1)
        maj = np.where((nc[:, 0] == nc[:, 1]) | (nc[:, 0] == nc[:, 2]), nc[:, 0],
                       np.where(nc[:, 1] == nc[:, 2], nc[:, 1], chart))
        change = (maj != chart) & (maj >= 0) & (((nc == maj[:, None]).sum(1)) >= 2)
        if not change.any():
            break
        chart = np.where(change, maj, chart)
    # per-vertex spherical coordinates
    vlat = np.arcsin(np.clip(dirs[:, 2], -1, 1))
    vlon = np.arctan2(dirs[:, 1], dirs[:, 0])
    chart_uv = []
    order_tris = []
    for c in range(16):
        tids = np.nonzero(chart == c)[0]
        lb, ob = divmod(c, 4)
        lon_c = -np.pi + (ob + 0.5) * np.pi / 2
        corner = f[tids]
        la = vlat[corner]
        lo = vlon[corner]
        lo = np.mod(lo - lon_c + np.pi, 2 * np.pi) - np.pi       # unwrap around sector centre
        if lb in (0, 3):
            rho = np.pi / 2 - np.abs(la)                          # azimuthal equidistant
            sgn = 1.0 if lb == 3 else -1.0
            p = np.stack([rho * np.sin(lo), -sgn * rho * np.cos(lo)], -1)
        else:
            lat_mid = -np.pi / 8 if lb == 1 else np.pi / 8
            p = np.stack([lo * np.cos(lat_mid), la], -1)
        area = ((p[:, 1, 0] - p[:, 0, 0]) * (p[:, 2, 1] - p[:, 0, 1]) -
                (p[:, 2, 0] - p[:, 0, 0]) * (p[:, 1, 1] - p[:, 0, 1]))
        if np.median(area) < 0:
            p[..., 0] *= -1
        chart_uv.append(p)
        order_tris.append(tids)
    placed = _pack_charts(chart_uv, (4, 4), width, height, gutter)
    uv = np.empty((len(f), 3, 2))
    for tids, p in zip(order_tris, placed):
        uv[tids] = p
    area = ((uv[:, 1, 0] - uv[:, 0, 0]) * (uv[:, 2, 1] - uv[:, 0, 1]) -
            (uv[:, 2, 0] - uv[:, 0, 0]) * (uv[:, 1, 1] - uv[:, 0, 1]))
    if np.any(area <= 0):
        raise RuntimeError(f"icosphere atlas has {int((area <= 0).sum())} flipped triangles")
    uv = _keep_off_texel_grid(uv, width, height)
    tex = value_noise(rng, width, height, channels) + rng.uniform(-0.1, 0.1, size=(height, width, channels))
    return {"vertices": v, "triangles": f.astype(np.int32), "uv": uv,
            "texture": tex.astype(np.float32), "name": f"icosphere{subdiv}_{width}x{height}"}


# ----------------------------------------------------------------------------
# genus 2: two tori joined by a straight tube, 32 charts
# ----------------------------------------------------------------------------

def _signed_uv_area(uv: np.ndarray) -> np.ndarray:
    return ((uv[:, 1, 0] - uv[:, 0, 0]) * (uv[:, 2, 1] - uv[:, 0, 1]) -
            (uv[:, 2, 0] - uv[:, 0, 0]) * (uv[:, 1, 1] - uv[:, 0, 1]))


def genus2_atlas(width: int = 4096, height: int = 4096, nu: int = 352, nv: int = 144, R: float = 1.0,
                 r: float = 0.4, gap: float = 0.3, seed: int = 0, gutter: int = 8, jitter: float = 0.3,
                 channels: int = 1) -> dict:
    """Genus-2 surface: two tori side by side, each opened by one block of its
    (u, v) grid where it faces the other, the two openings joined by a straight
    tube (a surface of genus 2).

    Torus A is centred at x = -(R + r + gap), torus B is its mirror image.  The
    grid of each torus is cut into 4 x 4 blocks of 90 x 90 degrees, block (0, 0)
    (facing the other torus, outer equator) is removed, and each remaining block
    is one chart (rectangle in (u (R + r cos v_mid), v r)).  The tube is the
    extrusion along x of the opening's rim and is split into 2 charts
    (developed: rim arc length x extrusion length).  32 charts, about
    4 nu nv triangles; vertices of the removed blocks are dropped.  Texture: ``channels`` of uniform noise in [0, 1)."""
    if nu % 4 or nv % 4:
        raise ValueError("nu and nv must be multiples of 4")
    rng = np.random.default_rng(seed)
    cx = R + r + gap
    bu, bv = nu // 4, nv // 4
    ii, jj = np.meshgrid(np.arange(nu), np.arange(nv), indexing="xy")
    u = 2 * np.pi * ii / nu - np.pi / 4
    v = 2 * np.pi * jj / nv - np.pi / 4
    rad = R + r * np.cos(v)
    posA = np.stack([-cx + rad * np.cos(u), rad * np.sin(u), r * np.sin(v)], -1).reshape(-1, 3)
    nA = nu * nv

    def vid(i, j):
        return (j % nv) * nu + (i % nu)

    # torus quads outside the removed block, two triangles each, grouped by block
    tA, cA, blk = [], [], []
    for j in range(nv):
        for i in range(nu):
            b = (i // bu, j // bv)
            if b == (0, 0):
                continue
            a_, b_, c_, d_ = (i, j), (i + 1, j), (i + 1, j + 1), (i, j + 1)
            for tri in ((a_, b_, c_), (a_, c_, d_)):
                tA.append([vid(*q) for q in tri])
                cA.append(tri)
                blk.append(b[1] * 4 + b[0])
    tA = np.array(tA, dtype=np.int64)
    cA = np.array(cA, dtype=np.float64)
    blk = np.array(blk, dtype=np.int64)
    # rim of the opening, counter-clockwise in (i, j)
    rim = ([(i, 0) for i in range(0, bu)] + [(bu, j) for j in range(0, bv)] +
           [(i, bv) for i in range(bu, 0, -1)] + [(0, j) for j in range(bv, 0, -1)])
    rim_ids = np.array([vid(i, j) for i, j in rim], dtype=np.int64)
    nr = len(rim_ids)
    # tube rings between rim A (x < 0) and its mirror: x runs from x_A to -x_A
    rimA = posA[rim_ids]
    h = 2 * np.pi * r / nv
    m = max(2, int(np.ceil(2 * np.abs(rimA[:, 0]).max() / h)))
    s = np.arange(1, m) / m
    rings = np.empty((m - 1, nr, 3))
    rings[:, :, 0] = rimA[None, :, 0] * (1 - 2 * s[:, None])
    rings[:, :, 1:] = rimA[None, :, 1:]
    nRing = (m - 1) * nr
    # vertex array: torus A, torus B (mirror), tube rings
    posB = posA * np.array([-1.0, 1.0, 1.0])
    verts = np.concatenate([posA, posB, rings.reshape(-1, 3)], 0)
    ring_vid = np.empty((m + 1, nr), dtype=np.int64)
    ring_vid[0] = rim_ids
    ring_vid[m] = nA + rim_ids
    ring_vid[1:m] = 2 * nA + np.arange(nRing).reshape(m - 1, nr)
    tB = nA + tA[:, ::-1]            # mirror image: reversed winding
    cB = cA[:, ::-1]
    # tube quads (k, q) -> (k+1, q) ... oriented below
    tT, cT, qT = [], [], []
    for k in range(m):
        for q in range(nr):
            a_, b_ = ring_vid[k, q], ring_vid[k, (q + 1) % nr]
            c_, d_ = ring_vid[k + 1, (q + 1) % nr], ring_vid[k + 1, q]
            for tri, cc in (((a_, b_, c_), ((q, k), (q + 1, k), (q + 1, k + 1))),
                            ((a_, c_, d_), ((q, k), (q + 1, k + 1), (q, k + 1)))):
                tT.append(tri)
                cT.append(cc)
                qT.append(q)
    tT = np.array(tT, dtype=np.int64)
    cT = np.array(cT, dtype=np.float64)
    qT = np.array(qT, dtype=np.int64)
    # orient the tube outwards (away from the rim's centroid axis, parallel to x)
    axis = rimA[:, 1:].mean(0)
    p0, p1, p2 = verts[tT[:, 0]], verts[tT[:, 1]], verts[tT[:, 2]]
    nrm = np.cross(p1 - p0, p2 - p0)
    out = (p0 + p1 + p2)[:, 1:] / 3 - axis
    if np.median((nrm[:, 1:] * out).sum(1)) < 0:
        tT = tT[:, [0, 2, 1]]
        cT = cT[:, [0, 2, 1]]
    tris = np.concatenate([tA, tB, tT], 0)
    used = np.zeros(len(verts), dtype=bool)
    used[tris.reshape(-1)] = True
    remap = np.cumsum(used) - 1
    verts = verts[used]
    tris = remap[tris]
    # charts: 15 blocks per torus, 2 tube halves
    chart = np.concatenate([blk, 16 + blk, 32 + (qT * 2) // nr], 0)
    corners = np.concatenate([cA, cB, cT], 0)
    kind = np.concatenate([np.zeros(len(tA)), np.ones(len(tB)), 2 * np.ones(len(tT))]).astype(np.int64)
    # rim arc length (tube development)
    seg = np.linalg.norm(np.roll(rimA[:, 1:], -1, 0) - rimA[:, 1:], axis=1)
    arc = np.concatenate([[0.0], np.cumsum(seg)])
    chart_uv, groups = [], []
    for c in np.unique(chart):
        tids = np.nonzero(chart == c)[0]
        cc = corners[tids]
        if kind[tids[0]] < 2:       # torus block: (u * (R + r cos v_mid), v * r)
            uu = 2 * np.pi * cc[..., 0] / nu
            vv = 2 * np.pi * cc[..., 1] / nv
            vmid = 2 * np.pi * ((c % 16) // 4 + 0.5) / 4 - np.pi / 4
            p = np.stack([uu * (R + r * np.cos(vmid)), vv * r], -1)
        else:                       # tube half: (arc length along the rim, x)
            q = cc[..., 0].astype(np.int64)
            k = cc[..., 1]
            xA = np.abs(rimA[q % nr, 0])
            p = np.stack([arc[q], -xA + 2 * xA * k / m], -1)
        if np.median(_signed_uv_area(p)) < 0:
            p[..., 0] *= -1
        chart_uv.append(p)
        groups.append(tids)
    placed = _pack_charts(chart_uv, (8, 4), width, height, gutter)
    uv = np.empty((len(tris), 3, 2))
    for tids, p in zip(groups, placed):
        uv[tids] = p
    # per chart-vertex texture jitter (same for every corner of one chart vertex),
    # at most a tenth of the shortest texture-space edge
    scale = np.array([width, height])
    edge = np.linalg.norm((np.roll(uv, -1, 1) - uv) * scale, axis=-1).min()
    amp = min(jitter, 0.1 * edge)
    ckey = chart[:, None] * (len(verts) + 1) + tris
    ukeys, inv = np.unique(ckey.reshape(-1), return_inverse=True)
    jit = rng.uniform(-amp, amp, size=(len(ukeys), 2)) / scale
    uv = uv + jit[inv].reshape(uv.shape)
    bad = int((_signed_uv_area(uv) <= 0).sum())
    if bad:
        raise RuntimeError(f"genus-2 atlas has {bad} flipped triangles")
    uv = _keep_off_texel_grid(uv, width, height)
    tex = rng.uniform(0.0, 1.0, size=(height, width, channels))
    return {"vertices": verts.astype(np.float64), "triangles": tris.astype(np.int32), "uv": uv,
            "texture": tex.astype(np.float32), "name": f"genus2_{nu}x{nv}_{width}x{height}"}


def gaussian_bump_field(mesh: dict, bumps: int = 8, seed: int = 0, sigma: float = 0.5) -> np.ndarray:
    """Tangent field per triangle: the surface gradient of a seeded sum of
    Gaussians, rotated by 90 degrees about the normal.  Returned in each
    triangle's edge basis (coefficients of p1 - p0 and p2 - p0), the layout of
    the reference's vector-field files."""
    rng = np.random.default_rng(seed)
    v = mesh["vertices"]
    t = mesh["triangles"].astype(np.int64)
    centres = v[rng.choice(len(v), size=bumps, replace=False)]
    amp = rng.uniform(0.5, 1.5, size=bumps) * rng.choice([-1.0, 1.0], size=bumps)
    d2 = ((v[:, None, :] - centres[None]) ** 2).sum(-1)
    phi = (amp * np.exp(-d2 / (2 * sigma * sigma))).sum(1)
    e1 = v[t[:, 1]] - v[t[:, 0]]
    e2 = v[t[:, 2]] - v[t[:, 0]]
    n = np.cross(e1, e2)
    n /= np.linalg.norm(n, axis=1, keepdims=True)
    # gradient of the linear interpolant: G [e1 e2] = [phi1 - phi0, phi2 - phi0], G in the plane
    E = np.stack([e1, e2], 1)                          # (nt, 2, 3)
    gram = np.einsum("tai,tbi->tab", E, E)
    dphi = np.stack([phi[t[:, 1]] - phi[t[:, 0]], phi[t[:, 2]] - phi[t[:, 0]]], -1)
    coef = np.linalg.solve(gram, dphi[..., None])[..., 0]
    grad = np.einsum("ta,tai->ti", coef, E)
    rot = np.cross(n, grad)
    # rotated vector in the edge basis
    rhs = np.einsum("tai,ti->ta", E, rot)
    return np.linalg.solve(gram, rhs[..., None])[..., 0]


def write_vf(path: str, vf: np.ndarray) -> None:
    """Reference vector file: int32 count, then count Point2D<double> (Src/VectorIO.h:9-32)."""
    vf = np.ascontiguousarray(vf, dtype=np.float64).reshape(-1, 2)
    with open(path, "wb") as fh:
        fh.write(struct.pack("<i", len(vf)))
        fh.write(vf.tobytes())


def read_vf(path: str) -> np.ndarray:
    with open(path, "rb") as fh:
        (n,) = struct.unpack("<i", fh.read(4))
        return np.frombuffer(fh.read(16 * n), dtype=np.float64).reshape(n, 2).copy()


# ----------------------------------------------------------------------------
# binary mesh container shared with the reference harness
# ----------------------------------------------------------------------------

_MAGIC = b"GDTPMSH1"


def write_gdm(path: str, mesh: dict) -> None:
    v = np.ascontiguousarray(mesh["vertices"], dtype=np.float64)
    t = np.ascontiguousarray(mesh["triangles"], dtype=np.int32)
    uv = np.ascontiguousarray(mesh["uv"], dtype=np.float64)
    tex = np.ascontiguousarray(mesh["texture"], dtype=np.float32)
    h, w, c = tex.shape
    with open(path, "wb") as fh:
        fh.write(_MAGIC)
        fh.write(struct.pack("<qqqqq", len(v), len(t), w, h, c))
        fh.write(v.tobytes())
        fh.write(t.tobytes())
        fh.write(uv.tobytes())
        fh.write(tex.tobytes())


def read_gdm(path: str) -> dict:
    with open(path, "rb") as fh:
        if fh.read(8) != _MAGIC:
            raise ValueError("not a GDTP mesh file")
        nv, nt, w, h, c = struct.unpack("<qqqqq", fh.read(40))
        v = np.frombuffer(fh.read(nv * 24), dtype=np.float64).reshape(nv, 3)
        t = np.frombuffer(fh.read(nt * 12), dtype=np.int32).reshape(nt, 3)
        uv = np.frombuffer(fh.read(nt * 48), dtype=np.float64).reshape(nt, 3, 2)
        tex = np.frombuffer(fh.read(w * h * c * 4), dtype=np.float32).reshape(h, w, c)
    return {"vertices": v.copy(), "triangles": t.copy(), "uv": uv.copy(), "texture": tex.copy()}
