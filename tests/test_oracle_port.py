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
