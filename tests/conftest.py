import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def load_golden(name: str) -> dict:
    with np.load(os.path.join(GOLDEN, f"{name}.npz")) as z:
        return {k.replace("__", "/"): z[k] for k in z.files}


def golden_mesh(g: dict) -> dict:
    return {"vertices": g["mesh/vertices"], "triangles": g["mesh/triangles"], "uv": g["mesh/uv"], "texture": g["mesh/texture"]}


def golden_csr(g: dict, name: str, shape=None):
    import scipy.sparse as sp
    ptr, col, val = g[name + "/ptr"], g[name + "/col"], g[name + "/val"]
    ncol = shape[1] if shape else (int(col.max()) + 1 if len(col) else 0)
    return sp.csr_matrix((val, col, ptr), shape=(len(ptr) - 1, ncol))


@pytest.fixture(scope="session")
def built_lib():
    from gradientdomaintextureprocessing_b200 import build
    return build.build()
