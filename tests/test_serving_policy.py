"""Host logic of the solve server: HBM admission (LRU eviction of idle models,
busy models never evicted, budget bound) and the serving workload generator."""
import os
import subprocess
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_admission_policy_native():
    with tempfile.TemporaryDirectory() as tmp:
        exe = os.path.join(tmp, "policy_check")
        subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "gradientdomaintextureprocessing_b200", "csrc"),
                        os.path.join(ROOT, "tests", "native", "policy_check.cpp"), "-o", exe], check=True)
        out = subprocess.run([exe], capture_output=True, text=True)
        assert out.returncode == 0, out.stdout + out.stderr
        assert out.stdout.strip() == "ok"


def test_request_stream_shape():
    from gradientdomaintextureprocessing_b200.serving import KIND_FILTER, KIND_GEODESIC, KIND_LIC, SIZE_LADDER, request_stream
    s = request_stream(2000, rate_per_s=100.0, seed=3)
    arr = np.array([a for a, *_ in s])
    assert np.all(np.diff(arr) > 0)
    assert abs(np.mean(np.diff(arr)) - 0.01) < 0.002                    # Poisson, rate 100/s
    kinds = np.array([k for *_, k in s])
    for kind, p in ((KIND_FILTER, 0.6), (KIND_GEODESIC, 0.3), (KIND_LIC, 0.1)):
        assert abs(np.mean(kinds == kind) - p) < 0.04
    sizes = {sz for _, _, sz, _ in s}
    assert sizes <= set(SIZE_LADDER) and all(sz % 8 == 0 for sz in sizes) and len(sizes) >= 8
    assert {m for _, m, _, _ in s} == {"torus", "icosphere", "genus2"}
