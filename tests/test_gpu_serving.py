"""Solve server on the device: resident models of three kinds, continuous
batching, HBM admission.

* every request's result is the same alone and in the mix: converged
  right-hand sides are frozen inside a batch, so the bound is 1e-12 of the
  result's largest entry (measured: bitwise equal);
* requests arriving together for one model are batched;
* a budget that holds one model at a time evicts and rebuilds without changing
  results; a model larger than the budget fails with GDTP_ERR_BUDGET.
"""
import numpy as np
import pytest

from conftest import golden_mesh, load_golden

pytestmark = pytest.mark.gpu


def models_for(server):
    from gradientdomaintextureprocessing_b200.metric import InitializeAnisotropicMetric
    from gradientdomaintextureprocessing_b200.serving import KIND_FILTER, KIND_GEODESIC, KIND_LIC
    t = golden_mesh(load_golden("torus128"))
    g = golden_mesh(load_golden("ico256"))
    lg = load_golden("genus2lic512")
    lm = golden_mesh(lg)
    return {
        "filter": server.add_model(t, KIND_FILTER, 1e-3, 2.0),
        "geodesic": server.add_model(g, KIND_GEODESIC, 1e-3, 1e-6),
        "lic": server.add_model(lm, KIND_LIC, 1e-4, 0.0, parameter_metric=InitializeAnisotropicMetric(lm, lg["mesh/field"])),
    }


def requests(server, m, rng):
    reqs = []
    for i in range(12):
        kind = ["filter", "geodesic", "lic"][i % 3]
        n = server.texels[m[kind]]
        if kind == "geodesic":
            reqs.append((m[kind], None, np.array([rng.integers(n)], dtype=np.int32), 1))
        else:
            k = 3 if kind == "filter" else 1
            reqs.append((m[kind], rng.uniform(0, 1, size=(n, k)), None, k))
    return reqs


def submit(server, r):
    mid, sig, src, _ = r
    return server.submit(mid, signal=sig, sources=src, tol=1e-6, max_iters=400)


@pytest.fixture(scope="module")
def served(built_lib):
    from gradientdomaintextureprocessing_b200.serving import Server
    server = Server(budget_bytes=16 << 30, slots=3)
    m = models_for(server)
    rng = np.random.default_rng(0)
    reqs = requests(server, m, rng)
    alone = []
    for r in reqs:
        x, rep = server.wait(submit(server, r), server.texels[r[0]], r[3])
        assert rep["rel_residual_max"] <= 1e-6 and rep["batch"] == 1
        alone.append(x)
    ids = [submit(server, r) for r in reqs]  # all at once: batched per model, models in parallel
    mix = [server.wait(i, server.texels[r[0]], r[3]) for i, r in zip(ids, reqs)]
    return server, m, reqs, alone, mix


def test_results_same_alone_and_in_mix(served):
    _, _, reqs, alone, mix = served
    for a, (x, rep) in zip(alone, mix):
        assert rep["rel_residual_max"] <= 1e-6
        assert np.abs(x - a).max() <= 1e-12 * np.abs(a).max()


def test_requests_are_batched(served):
    server, _, reqs, _, mix = served
    assert max(rep["batch"] for _, rep in mix) > 1
    st = server.stats()
    assert st["completed"] == 2 * len(reqs) and st["failed"] == 0
    assert st["batched_requests"] > st["batches"]
    assert 0 < st["p50_ms"] <= st["p99_ms"]
    assert st["peak_bytes"] <= st["budget"]


def test_small_budget_evicts_and_keeps_results(served):
    from gradientdomaintextureprocessing_b200 import _lib
    from gradientdomaintextureprocessing_b200.serving import Server
    big, m, reqs, alone, _ = served
    # room for the largest single model (by its estimate), not for two of them
    probe = Server(budget_bytes=1 << 40, slots=1)
    pm = models_for(probe)
    est = {k: probe.model_bytes(v) for k, v in pm.items()}
    assert all(est[k] >= big.model_bytes(m[k]) for k in m)
    budget = int(1.05 * max(est.values()))
    big_kind = max(est, key=est.get)
    assert all(est[big_kind] + est[k] > budget for k in est if k != big_kind)  # the largest model lives alone
    server = Server(budget_bytes=budget, slots=2)
    m2 = models_for(server)
    assert m2 == m
    for r, a in zip(reqs[:6], alone[:6]):  # alternating kinds: every request needs another model
        x, rep = server.wait(submit(server, r), server.texels[r[0]], r[3])
        assert np.abs(x - a).max() <= 1e-12 * np.abs(a).max()
    st = server.stats()
    assert st["evictions"] >= 2 and st["peak_bytes"] <= st["budget"]
    tiny = Server(budget_bytes=8 << 20, slots=1)  # below any model's size
    mt = models_for(tiny)
    with pytest.raises(_lib.GDTPError) as e:
        r = reqs[0]
        tiny.wait(tiny.submit(mt["filter"], signal=r[1], tol=1e-6), tiny.texels[mt["filter"]], r[3])
    assert e.value.code == -5
