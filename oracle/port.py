"""Oracle port: numpy/scipy restatement of the reference's solve-path operators.

TEST INFRASTRUCTURE ONLY.  Nothing in the product imports this module; tests
use it as the checker.  It is pinned against the compiled reference
(``oracle/_ref``, fixtures in ``tests/golden``) by ``tests/test_oracle_port.py``.

Every function restates one reference operator on the reference's data layout
(texel order, 10-slot deep coefficients, boundary CSR blocks):

* ``full_matrix``             FullMatrixConstruction   include/Src/UpdateCoefficients.inl:137-219
* ``multiply_no_reciprocals`` MultiplyBySystemMatrix_NoReciprocals include/Src/IterativeSolvers.inl:881-950
* ``prolongation``            InitializeProlongationMatrix include/Src/ProlongationAndRestriction.inl:218-263
* ``reciprocal_form``         UpdateMultigridCoefficients include/Src/UpdateCoefficients.inl:374-397
* ``relax``                   Relaxation's per-texel update include/Src/IterativeSolvers.inl:449-463, in the
                              device's 4-colour order (one colour per chart-local parity), optionally tile
                              by tile (32 x 32 blocks of a chart, four block colours in turn)
* ``direct_solve``            the --useDirectSolver FP64 solve (TextureFiltering.cpp:651-655, 704-707;
                              Eigen SimplicialLDLT in include/Src/Solver.h:144-203, here scipy's LU)
* ``embedding_metric``        InitializeEmbeddingMetric include/Src/Metric.inl:248-275
* ``vector_field_metric``     InitializeVectorFieldMetric include/Src/Metric.inl:12-67
* ``parameter_metric``        InitializeParameterMetric include/Src/Metric.inl:415-446

Metrics are (nt, 2, 2) arrays in ordinary row/column order (m[t, i, j]); the
reference's SquareMatrix g(c, r) is column c, row r, so g(c, r) = m[t, r, c].
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla


def full_matrix(nodeinfo: np.ndarray, deep_global: np.ndarray, boundary_global: np.ndarray, deep: np.ndarray,
                bb: sp.csr_matrix, bd: sp.csr_matrix) -> sp.csr_matrix:
    """Global operator from deep 9-point rows and the BB / BD boundary blocks."""
    n = len(nodeinfo)
    key = {(int(c), int(i), int(j)): g for g, (c, i, j, _) in enumerate(nodeinfo)}
    rows, cols, vals = [], [], []
    for d, g in enumerate(deep_global):
        c, i, j, _ = nodeinfo[g]
        for oy in (-1, 0, 1):
            for ox in (-1, 0, 1):
                rows.append(g)
                cols.append(key[(int(c), int(i) + ox, int(j) + oy)])
                vals.append(deep[d, (oy + 1) * 3 + ox + 1])
    bbc, bdc = bb.tocoo(), bd.tocoo()
    rows += list(boundary_global[bbc.row]) + list(boundary_global[bdc.row])
    cols += list(boundary_global[bbc.col]) + list(bdc.col)
    vals += list(bbc.data) + list(bdc.data)
    return sp.csr_matrix((vals, (rows, cols)), shape=(n, n))


def multiply_no_reciprocals(A: sp.csr_matrix, x: np.ndarray) -> np.ndarray:
    """y = A x with the raw (non-reciprocal) operator."""
    return A @ x


def prolongation(fine_nodeinfo: np.ndarray, fine_charts: np.ndarray, coarse_nodeinfo: np.ndarray,
                 coarse_charts: np.ndarray) -> sp.csr_matrix:
    """Bilinear per-chart prolongation: even offsets from the chart centre sit on a
    coarse texel (weight 1), odd ones between two (1/2 per axis)."""
    key = {(int(c), int(i), int(j)): g for g, (c, i, j, _) in enumerate(coarse_nodeinfo)}
    rows, cols, vals = [], [], []
    for g, (c, i, j, _) in enumerate(fine_nodeinfo):
        ri, rj = int(i) - fine_charts[c, 2], int(j) - fine_charts[c, 3]
        for a in ((0,) if ri % 2 == 0 else (0, 1)):
            for b in ((0,) if rj % 2 == 0 else (0, 1)):
                rows.append(g)
                cols.append(key[(int(c), ri // 2 + a + coarse_charts[c, 2], rj // 2 + b + coarse_charts[c, 3])])
                vals.append((1.0 if ri % 2 == 0 else 0.5) * (1.0 if rj % 2 == 0 else 0.5))
    return sp.csr_matrix((vals, (rows, cols)), shape=(len(fine_nodeinfo), len(coarse_nodeinfo)))


def deep_rows(A: sp.csr_matrix, nodeinfo: np.ndarray, deep_global: np.ndarray) -> np.ndarray:
    """10-slot deep coefficients (slot (dj+1)*3+(di+1)) read back from a global operator."""
    key = {(int(c), int(i), int(j)): g for g, (c, i, j, _) in enumerate(nodeinfo)}
    out = np.zeros((len(deep_global), 10))
    A = A.tocsr()
    for d, g in enumerate(deep_global):
        c, i, j, _ = nodeinfo[g]
        for oy in (-1, 0, 1):
            for ox in (-1, 0, 1):
                out[d, (oy + 1) * 3 + ox + 1] = A[g, key[(int(c), int(i) + ox, int(j) + oy)]]
    return out


def reciprocal_form(deep: np.ndarray) -> np.ndarray:
    """c_k /= c4 (k != 4), c4 = 1/c4, c9 = c4 (the smoother's stored form)."""
    out = deep.copy()
    c4 = deep[:, 4].copy()
    out[:, :9] = deep[:, :9] / c4[:, None]
    out[:, 4] = 1.0 / c4
    out[:, 9] = c4
    return out


def relax(nodeinfo: np.ndarray, deep_global: np.ndarray, recip: np.ndarray, x: np.ndarray, rhs: np.ndarray, sweeps: int,
          reverse: bool = False, tile: int = 0) -> np.ndarray:
    """Gauss-Seidel sweeps over the deep texels in FP32: x_i = rhs_i c4 - sum_{k != 4} c_k x_k
    with the reciprocal-form coefficients ``recip`` (n_deep x 10, stencil slot 3 (dj + 1) + di + 1),
    colour (ci & 1) | (cj & 1) << 1 of the chart-local coordinates, colours 0..3 (3..0 if reverse).
    tile > 0: texels are grouped in tile x tile blocks of their chart's grid, coloured by block parity
    (bi & 1) | (bj & 1) << 1; the blocks of one colour run all sweeps in turn (colours of blocks
    0..3, 3..0 if reverse), each seeing the current values of every neighbour.
    x, rhs: n x k; returns the new x (float32)."""
    ni = np.asarray(nodeinfo)
    chart, ci, cj = ni[:, 0], ni[:, 1], ni[:, 2]
    w, h = ci.max() + 3, cj.max() + 3
    look = -np.ones((chart.max() + 1, w, h), dtype=np.int64)
    look[chart, ci + 1, cj + 1] = np.arange(len(ni))
    g = np.asarray(deep_global, dtype=np.int64)
    gc, gi, gj = chart[g], ci[g], cj[g]
    nb = np.empty((len(g), 9), dtype=np.int64)
    for k in range(9):
        di, dj = k % 3 - 1, k // 3 - 1
        nb[:, k] = look[gc, gi + di + 1, gj + dj + 1]
    assert (nb >= 0).all(), "a deep texel has an inactive neighbour"
    c = np.asarray(recip, dtype=np.float32)
    out = np.asarray(x, dtype=np.float32).reshape(len(ni), -1).copy()
    b = np.asarray(rhs, dtype=np.float32).reshape(len(ni), -1)
    colour = (gi & 1) | ((gj & 1) << 1)
    block = ((gi // tile) & 1) | (((gj // tile) & 1) << 1) if tile else np.zeros_like(gi)
    order = [3, 2, 1, 0] if reverse else [0, 1, 2, 3]
    for blk in (order if tile else [0]):
        for _ in range(sweeps):
            for col in order:
                sel = np.nonzero((colour == col) & (block == blk))[0]
                t = [c[sel, k][:, None] * out[nb[sel, k]] for k in range(9)]
                acc = ((t[0] + t[1] + t[2]) + (t[6] + t[7] + t[8])) + (t[3] + t[5])
                out[g[sel]] = b[g[sel]] * c[sel, 4][:, None] - acc
    return out


def direct_solve(A: sp.csr_matrix, b: np.ndarray) -> np.ndarray:
    return spla.splu(A.tocsc()).solve(np.asarray(b, dtype=np.float64))


def relative_residual(A: sp.csr_matrix, b: np.ndarray, x: np.ndarray) -> np.ndarray:
    return np.linalg.norm(b - A @ x, axis=0) / np.linalg.norm(b, axis=0)


def energy_error(A: sp.csr_matrix, x: np.ndarray, x_ref: np.ndarray) -> np.ndarray:
    """Relative error in the operator's energy norm, per right-hand side.  Texels
    whose support barely meets a chart have tiny diagonals and are not pinned by
    the residual; the energy norm weighs every texel by its support."""
    e = x - x_ref
    return np.sqrt(np.einsum("ik,ik->k", e, A @ e) / np.einsum("ik,ik->k", x_ref, A @ x_ref))


# ----------------------------------------------------------------------------
# metrics (per mesh triangle, in the basis of the triangle's edges)
# ----------------------------------------------------------------------------

def embedding_metric(vertices: np.ndarray, triangles: np.ndarray, normalize: bool = True) -> np.ndarray:
    """g_kl = e_k . e_l with e_0 = p1 - p0, e_1 = p2 - p0, divided by the total area."""
    p = vertices[triangles]
    e = np.stack([p[:, 1] - p[:, 0], p[:, 2] - p[:, 0]], 1)
    g = np.einsum("tki,tli->tkl", e, e)
    if normalize:
        g = g / (np.sqrt(np.linalg.det(g)) / 2).sum()
    return g


def vector_field_metric(g: np.ndarray, vf: np.ndarray, across: float = 0.1, isotropic: float = 1e-5,
                        normalize: bool = True) -> np.ndarray:
    """g B diag(0, across) B^-1 + isotropic g, B = g-orthonormal {vf, rotated g vf}."""
    out = np.empty_like(g)
    for t in range(len(g)):
        G = g[t]
        v0 = vf[t]
        u = np.zeros((2, 2))
        if v0 @ G @ v0 > 0:
            gv = G @ v0
            e = [v0.copy(), np.array([-gv[1], gv[0]])]
            e = [x / np.sqrt(x @ G @ x) for x in e]
            B = np.stack(e, 1)
            u = G @ B @ np.diag([0.0, across]) @ np.linalg.inv(B)
        out[t] = u + G * isotropic
    if normalize:
        out = out / (np.sqrt(np.linalg.det(out)) / 2).sum()
    return out


def parameter_metric(uv: np.ndarray, g: np.ndarray) -> np.ndarray:
    """Pull-back to texture coordinates: J^-T g J^-1, J = [q1 - q0, q2 - q0] as columns."""
    J = np.stack([uv[:, 1] - uv[:, 0], uv[:, 2] - uv[:, 0]], 2)
    Ji = np.linalg.inv(J)
    return np.einsum("tki,tkl,tlj->tij", Ji, g, Ji)


def metric_entries(m: np.ndarray) -> np.ndarray:
    """(nt, 4) entries g(0,0), g(0,1), g(1,0), g(1,1) in the reference's (column, row) indexing."""
    return np.stack([m[:, 0, 0], m[:, 1, 0], m[:, 0, 1], m[:, 1, 1]], 1)
