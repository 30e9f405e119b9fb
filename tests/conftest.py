import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def reference_checkout():
    """The reference checkout: $GDTP_REFERENCE, else the one oracle/Makefile
    compiled the oracle from (recorded in oracle/_ref/REFERENCE); None when
    neither names an existing directory (tests that read its data then skip)."""
    path = os.environ.get("GDTP_REFERENCE")
    if not path:
        try:
            with open(os.path.join(ROOT, "oracle", "_ref", "REFERENCE")) as fh:
                path = fh.read().strip()
        except OSError:
            return None
    return path if path and os.path.isdir(path) else None


def reference_data():
    """The reference's Data/ directory (its shipped meshes and fields), or a path
    that does not exist."""
    ref = reference_checkout()
    return os.path.join(ref, "Data") if ref else os.path.join(ROOT, "oracle", "_ref", "no-reference-checkout")


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
