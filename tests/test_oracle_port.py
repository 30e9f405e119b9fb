"""Pins the numpy oracle port (oracle/port.py) to the compiled reference's
outputs stored in tests/golden, so tests can use the port as a checker."""
import numpy as np
import pytest

from conftest import golden_csr, load_golden


@pytest.fixture(scope="module", params=["torus128", "ico256"])
def g(request):
    return load_golden(request.param)


def full(g, which):
    import port
    n = len(g["L0/nodeinfo"])
    nb = len(g["L0/boundaryGlobalIndex"])
    BB = golden_csr(g, f"fine/BB{which}", (nb, nb))
    BD = golden_csr(g, f"fine/BD{which}", (nb, n))
    return port.full_matrix(g["L0/nodeinfo"], g["L0/deepGlobalIndex"], g["L0/boundaryGlobalIndex"], g[f"fine/deep{which.capitalize()}"], BB, BD)


def test_port_rhs_matches_reference(g):
    import port
    lam, sharp = g["meta/weights"]
    M, S = full(g, "mass"), full(g, "stiffness")
    f = g["solve/f"]
    rhs = port.multiply_no_reciprocals(M, f) + lam * sharp * port.multiply_no_reciprocals(S, f)
    assert np.abs(rhs - g["solve/rhs"]).max() <= 1e-12 * np.abs(g["solve/rhs"]).max()


def test_port_direct_solve_matches_reference_in_energy(g):
    import port
    lam = g["meta/weights"][0]
    A = full(g, "mass") + lam * full(g, "stiffness")
    x = port.direct_solve(A, g["solve/rhs"])
    assert port.relative_residual(A, g["solve/rhs"], g["solve/exact"]).max() < 1e-12
    assert port.energy_error(A, x, g["solve/exact"]).max() < 1e-9


def test_port_galerkin_matches_reference_hierarchy(g):
    import port
    lam = g["meta/weights"][0]
    A = full(g, "mass") + lam * full(g, "stiffness")
    levels = int(g["meta/size"][2])
    for l in range(1, levels):
        P = port.prolongation(g[f"L{l-1}/nodeinfo"], g[f"L{l-1}/charts_i"], g[f"L{l}/nodeinfo"], g[f"L{l}/charts_i"])
        A = (P.T @ A @ P).tocsr()
        deep = port.deep_rows(A, g[f"L{l}/nodeinfo"], g[f"L{l}/deepGlobalIndex"])
        ref = g[f"L{l}/coef/deep"]
        mine = port.reciprocal_form(deep) if l < levels - 1 else deep
        cols = 10 if l < levels - 1 else 9
        assert np.abs(mine[:, :cols] - ref[:, :cols]).max() <= 1e-10 * np.abs(ref[:, :cols]).max(), l


@pytest.mark.parametrize("tile", [0, 32])
@pytest.mark.parametrize("reverse", [False, True])
def test_port_relax_update_rule(g, tile, reverse):
    """The smoother restatement applies the reference's per-texel update
    (IterativeSolvers.inl:449-463, reciprocal-form coefficients of the
    reference's own level 0): after one sweep the texels updated last (the last
    colour; with tiles, in the tiles of the last tile colour) satisfy
    x_i = rhs_i c4 - sum_k c_k x_k with the final values of all neighbours;
    boundary texels are unchanged; tiles of the first tile colour see the
    starting values of their ring in the other tiles."""
    import port
    ni, dg = g["L0/nodeinfo"], g["L0/deepGlobalIndex"]
    recip = g["L0/coef/deep"]  # the reference stores level 0 in reciprocal form
    rng = np.random.default_rng(3)
    n = len(ni)
    x0 = rng.uniform(-1, 1, (n, 3)).astype(np.float32)
    rhs = rng.uniform(-1, 1, (n, 3)).astype(np.float32)
    x1 = port.relax(ni, dg, recip, x0, rhs, 1, reverse=reverse, tile=tile)
    bnd = g["L0/boundaryGlobalIndex"]
    np.testing.assert_array_equal(x1[bnd], x0[bnd])
    look = {(int(c), int(i), int(j)): t for t, (c, i, j, _) in enumerate(ni)}
    last = 0 if reverse else 3

    def block(i, j):
        return ((i // tile) & 1) | (((j // tile) & 1) << 1) if tile else 0

    order = [3, 2, 1, 0] if reverse else [0, 1, 2, 3]
    present = {block(int(ni[t, 1]), int(ni[t, 2])) for t in dg}
    last_block = [b for b in order if b in present][-1]  # narrow charts may have one row of tiles
    checked = 0
    for d, t in enumerate(dg):
        c, i, j = (int(v) for v in ni[t, :3])
        if ((i & 1) | ((j & 1) << 1)) != last or (tile and block(i, j) != last_block):
            continue
        acc = np.zeros(3)
        for k in (0, 1, 2, 3, 5, 6, 7, 8):
            di, dj = k % 3 - 1, k // 3 - 1
            acc += recip[d, k] * x1[look[(c, i + di, j + dj)]].astype(np.float64)
        want = rhs[t].astype(np.float64) * recip[d, 4] - acc
        assert np.abs(x1[t] - want).max() <= 1e-5 * max(1.0, np.abs(want).max())
        checked += 1
    assert checked > 100
    if tile:  # one tile-colour group alone equals a plain sweep of those texels with the rest frozen
        first = [b for b in order if b in present][0]
        rows = [t for t in dg if block(int(ni[t, 1]), int(ni[t, 2])) == first]
        x_first = port.relax(ni, np.array(rows), recip[[list(dg).index(t) for t in rows]], x0, rhs, 1, reverse=reverse)
        np.testing.assert_allclose(x1[rows], x_first[rows], rtol=0, atol=1e-5)
