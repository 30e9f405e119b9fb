"""The reference's own FP64 solution of a whole configuration (test infrastructure).

Runs the compiled reference (``oracle/_ref/gdtp_ref``: the reference's solve
path built from its unmodified headers by ``oracle/Makefile``) in its
``vsolve`` mode on a mesh from the seeded generators: the reference builds its
hierarchy, assembles its own FP64 mass and stiffness
(``MassAndStiffness.h:490``), forms the TextureFiltering right-hand side
``M f + stiffness * sharpness * S f`` (``TextureFiltering.cpp:693-700``) and
iterates its FP64 V-cycle (``IterativeSolvers.inl:1211``, ``Vec4d``) until its
relative residual reaches ``tol``.  At 1e-12 that iterate is the FP64 ground
truth for meshes where the ``--useDirectSolver`` path (``TextureFiltering.cpp:
651-655``) is too slow for a test.  The dump also holds the reference's FP64
operator ``A = M + stiffness S``, so errors are measured in the reference's own
energy norm.

Only ``tests/`` and ``bench.py``'s checker leg use this module.
"""
from __future__ import annotations

import os
import subprocess
import tempfile

import numpy as np

from gdd import csr, read_dump

HERE = os.path.dirname(os.path.abspath(__file__))
HARNESS = os.path.join(HERE, "_ref", "gdtp_ref")


def available() -> bool:
    return os.path.exists(HARNESS)


def reference_solution(mesh: dict, levels: int, stiffness: float, sharpness: float, tol: float = 1e-12,
                       max_vcycles: int = 600, parameter_metric: np.ndarray | None = None, threads: int | None = None,
                       timeout: float = 1800.0) -> dict:
    """The reference's solve of ``(M + stiffness S) x = M f + stiffness sharpness S f``.

    mesh: a generator mesh (vertices, triangles, per-corner uv, texture);
    parameter_metric: optional per-triangle metric (nt x 4) used instead of the
    embedding metric (the anisotropic LIC operator).  Returns ``rhs`` and ``x``
    (n x 3: the texture's channels, a single-channel texture replicated),
    ``A`` (scipy CSR), the residual ``history`` and the level-0 ``counts``."""
    from gradientdomaintextureprocessing_b200 import meshgen
    if not available():
        raise FileNotFoundError(f"{HARNESS} is not built (oracle/Makefile)")
    env = dict(os.environ, OMP_NUM_THREADS=str(threads or os.cpu_count() or 1))
    with tempfile.TemporaryDirectory() as tmp:
        gdm, out = os.path.join(tmp, "mesh.gdm"), os.path.join(tmp, "out.gdd")
        meshgen.write_gdm(gdm, mesh)
        cmd = [HARNESS, gdm, out, str(levels), repr(float(stiffness)), repr(float(sharpness)), str(max_vcycles), "vsolve",
               repr(float(tol))]
        if parameter_metric is not None:
            pm = os.path.join(tmp, "metric.pm")
            np.ascontiguousarray(parameter_metric, dtype=np.float64).tofile(pm)
            cmd.append(pm)
        subprocess.run(cmd, check=True, capture_output=True, env=env, timeout=timeout)
        d = read_dump(out)
    n = int(d["L0/counts"][0])
    return {"rhs": d["solve/rhs"], "x": d["solve/vcycle_x"], "A": csr(d, "fine/A", (n, n)),
            "history": d["vcycle/history"], "counts": d["L0/counts"], "vcycle_times": d["time/vcycle"],
            "threads": int(env["OMP_NUM_THREADS"])}


def energy_error(A, x: np.ndarray, x_ref: np.ndarray) -> np.ndarray:
    """||x - x_ref||_A / ||x_ref||_A per right-hand side."""
    x = np.asarray(x, dtype=np.float64).reshape(x_ref.shape[0], -1)
    x_ref = np.asarray(x_ref, dtype=np.float64).reshape(x_ref.shape[0], -1)
    e = x - x_ref
    return np.sqrt(np.einsum("ik,ik->k", e, A @ e) / np.einsum("ik,ik->k", x_ref, A @ x_ref))


def relative_residual(A, b: np.ndarray, x: np.ndarray) -> np.ndarray:
    b = np.asarray(b, dtype=np.float64).reshape(A.shape[0], -1)
    x = np.asarray(x, dtype=np.float64).reshape(A.shape[0], -1)
    return np.linalg.norm(b - A @ x, axis=0) / np.linalg.norm(b, axis=0)
