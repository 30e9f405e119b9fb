"""Solve server: resident models, HBM admission, continuous batching.

``Server`` wraps ``gdtp_server_*`` (``include/gdtp.h``): models (mesh,
resolution, kind) are added once (host hierarchy), made resident on the device
under an HBM budget, and requests are batched per model by the server's worker
threads.  ``request_stream`` / ``run_stream`` build and replay the serving
workload: Poisson arrivals, meshes {torus, icosphere, genus-2}, texture sizes
log-uniform between two bounds (snapped to multiples of 8 on a sqrt(2) ladder so
that requests share resident models), kinds 60 % filtering (k = 3), 30 %
geodesic (k = 1), 10 % line-integral convolution (k = 1).
"""
from __future__ import annotations

import ctypes as C
import time

import numpy as np

from . import _lib
from . import meshgen
from .metric import InitializeAnisotropicMetric, across_for_ratio

KIND_FILTER, KIND_GEODESIC, KIND_LIC = 0, 1, 2
KIND_NAMES = {KIND_FILTER: "filtering", KIND_GEODESIC: "geodesic", KIND_LIC: "lic"}


class Server:
    def __init__(self, budget_bytes: int = 80 << 30, slots: int = 4, device: int = 0):
        s = C.c_void_p()
        _lib.check(_lib.lib().gdtp_server_create(int(device), int(budget_bytes), int(slots), C.byref(s)))
        self._s = s
        self.texels = {}
        self.kinds = {}

    def __del__(self):
        s, self._s = getattr(self, "_s", None), None
        if s:
            try:
                _lib.lib().gdtp_server_free(s)
            except (TypeError, AttributeError):  # interpreter exit: module globals already cleared
                pass

    def add_model(self, mesh: dict, kind: int, weight: float, second: float = 0.0, levels: int = 4,
                  parameter_metric: np.ndarray | None = None) -> int:
        v = np.ascontiguousarray(mesh["vertices"], dtype=np.float64)
        t = np.ascontiguousarray(mesh["triangles"], dtype=np.int32)
        uv = np.ascontiguousarray(mesh["uv"], dtype=np.float64)
        h, w = mesh["texture"].shape[:2]
        pm = None if parameter_metric is None else np.ascontiguousarray(parameter_metric, dtype=np.float64)
        mid = C.c_int()
        _lib.check(_lib.lib().gdtp_server_add_model(self._s, _lib.ptr(v), len(v), _lib.ptr(t), len(t), _lib.ptr(uv), w, h, levels,
                                                    int(kind), float(weight), float(second), _lib.ptr(pm), C.byref(mid)))
        n = C.c_int64()
        _lib.check(_lib.lib().gdtp_server_model_texels(self._s, mid.value, C.byref(n)))
        self.texels[mid.value] = n.value
        self.kinds[mid.value] = kind
        return mid.value

    def model_bytes(self, model: int) -> int:
        """Measured device bytes when resident, else the admission estimate."""
        b = C.c_int64()
        _lib.check(_lib.lib().gdtp_server_model_bytes(self._s, int(model), C.byref(b)))
        return b.value

    def warm(self, model: int) -> None:
        _lib.check(_lib.lib().gdtp_server_warm(self._s, int(model)))

    def submit(self, model: int, signal: np.ndarray | None = None, sources=None, tol: float = 1e-6, max_iters: int = 200) -> int:
        L = _lib.lib()
        rid = C.c_int64()
        if sources is not None:
            src = np.ascontiguousarray(np.atleast_1d(sources), dtype=np.int32)
            _lib.check(L.gdtp_server_submit(self._s, int(model), None, _lib.ptr(src), len(src), float(tol), int(max_iters), C.byref(rid)))
        else:
            f = np.ascontiguousarray(signal, dtype=np.float64).reshape(self.texels[model], -1)
            _lib.check(L.gdtp_server_submit(self._s, int(model), _lib.ptr(f), None, f.shape[1], float(tol), int(max_iters), C.byref(rid)))
        return rid.value

    def wait(self, request: int, n: int, k: int):
        out = np.empty((n, k))
        rep = _lib.Report()
        timing = np.zeros(3)
        _lib.check(_lib.lib().gdtp_server_wait(self._s, int(request), _lib.ptr(out), C.byref(rep), _lib.ptr(timing)))
        return out, {"iterations": rep.iterations, "rel_residual_max": rep.rel_residual_max, "latency_ms": float(timing[0]),
                     "queued_ms": float(timing[1]), "batch": int(timing[2])}

    def stats(self) -> dict:
        v = np.zeros(14)
        _lib.check(_lib.lib().gdtp_server_stats(self._s, _lib.ptr(v)))
        keys = ["completed", "failed", "p50_ms", "p99_ms", "mean_ms", "texel_rhs_per_s", "batches", "batched_requests",
                "evictions", "builds", "resident_bytes", "peak_bytes", "budget"]
        return {k: float(v[i]) for i, k in enumerate(keys)}


SIZE_LADDER = [256, 360, 512, 720, 1024, 1448, 2048, 2896, 4096]


def request_stream(n_requests: int = 256, rate_per_s: float = 200.0, min_size: int = 256, max_size: int = 4096, seed: int = 0):
    """(arrival s, mesh name, size, kind) tuples: Poisson arrivals, sizes
    log-uniform in [min_size, max_size] snapped to the ladder, kinds 60/30/10 %."""
    rng = np.random.default_rng(seed)
    ladder = [s for s in SIZE_LADDER if min_size <= s <= max_size]
    arrivals = np.cumsum(rng.exponential(1.0 / rate_per_s, size=n_requests))
    out = []
    for a in arrivals:
        mesh = ["torus", "icosphere", "genus2"][rng.integers(3)]
        size = float(np.exp(rng.uniform(np.log(min_size), np.log(max_size))))
        size = min(ladder, key=lambda s: abs(np.log(s / size)))
        kind = rng.choice([KIND_FILTER, KIND_GEODESIC, KIND_LIC], p=[0.6, 0.3, 0.1])
        out.append((float(a), mesh, int(size), int(kind)))
    return out


def make_mesh(name: str, size: int) -> dict:
    if name == "torus":
        return meshgen.torus_atlas(size, size, texture="value_noise")
    if name == "icosphere":
        return meshgen.icosphere_atlas(size, size, subdiv=6 if size >= 1024 else 5)
    return meshgen.genus2_atlas(size, size, nu=352 if size >= 2048 else 176, nv=144 if size >= 2048 else 72)


def build_models(server: Server, stream, lic_ratio: float = 1e3, warm: bool = True) -> dict:
    """One model per (mesh, size, kind) the stream uses; returns {(mesh, size, kind): (model, mesh dict)}."""
    models = {}
    for _, name, size, kind in stream:
        key = (name, size, kind)
        if key in models:
            continue
        mesh = make_mesh(name, size)
        if kind == KIND_FILTER:
            mid = server.add_model(mesh, KIND_FILTER, 1e-3, 2.0)
        elif kind == KIND_GEODESIC:
            mid = server.add_model(mesh, KIND_GEODESIC, 1e-3, 1e-6)
        else:
            vf = meshgen.gaussian_bump_field(mesh, bumps=8, seed=0)
            pm = InitializeAnisotropicMetric(mesh, vf, across=across_for_ratio(lic_ratio))
            mid = server.add_model(mesh, KIND_LIC, 1e-4, 0.0, parameter_metric=pm)
        if warm:
            server.warm(mid)
        models[key] = (mid, mesh)
    return models


def run_stream(server: Server, stream, models: dict, tol: float = 1e-6, seed: int = 1, max_iters: int = 1000):
    """Submits every request at its arrival time (wall clock), waits for all;
    returns per-request results and the server's statistics."""
    rng = np.random.default_rng(seed)
    payload = []
    for _, name, size, kind in stream:
        mid, mesh = models[(name, size, kind)]
        n = server.texels[mid]
        if kind == KIND_GEODESIC:
            payload.append(("sources", np.array([rng.integers(n)], dtype=np.int32), 1))
        else:
            k = 3 if kind == KIND_FILTER else 1
            payload.append(("signal", rng.uniform(0.0, 1.0, size=(n, k)), k))
    t0 = time.perf_counter()
    ids = []
    for (arrival, name, size, kind), (what, data, k) in zip(stream, payload):
        delay = arrival - (time.perf_counter() - t0)
        if delay > 0:
            time.sleep(delay)
        mid = models[(name, size, kind)][0]
        rid = (server.submit(mid, sources=data, tol=tol, max_iters=max_iters) if what == "sources"
               else server.submit(mid, signal=data, tol=tol, max_iters=max_iters))
        ids.append((rid, mid, k))
    results = []
    for (rid, mid, k), (_, name, size, kind) in zip(ids, stream):
        try:
            x, rep = server.wait(rid, server.texels[mid], k)
            rep["ok"] = True
        except _lib.GDTPError as e:  # reported, not fatal: a request that misses its tolerance
            x, rep = None, {"ok": False, "error": str(e), "latency_ms": float("nan"), "rel_residual_max": float("nan")}
        rep.update({"mesh": name, "size": size, "kind": KIND_NAMES[kind]})
        results.append((x, rep))
    wall = time.perf_counter() - t0
    return results, server.stats(), wall
