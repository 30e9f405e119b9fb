"""The allocation-free residual entry point (gdtp_residual_static) agrees with
the allocating one (gdtp_residual) on two calls in a row.

Callers that cannot allocate device memory when they check a solve (loops with
pre-planned memory, pools that must not grow, hosts where cudaMalloc would
stall their own work) pass their own device buffers; the norm reduction's
scratch is a static device array inside the library.  This file is collected
last so that a failure here leaves every other test already run."""
import ctypes as C

import numpy as np
import pytest

from conftest import golden_mesh, load_golden

pytestmark = pytest.mark.gpu


def test_static_residual_matches_allocating_residual(built_lib):
    import torch
    from gradientdomaintextureprocessing_b200 import _lib
    from gradientdomaintextureprocessing_b200.hierarchy import InitializeHierarchy
    from gradientdomaintextureprocessing_b200.system import System, SYSTEM
    g = load_golden("torus128")
    h = InitializeHierarchy(golden_mesh(g), levels=4)
    s = System(h)
    s.update(float(g["meta/weights"][0]), 1.0)
    b = np.ascontiguousarray(g["solve/rhs"])
    x = np.ascontiguousarray(g["solve/exact"] * 0.999 + 0.001)  # a non-trivial residual
    k = b.shape[1]
    ref = s.residual(b, x)  # allocating entry point
    r_ref = b - s.apply(x, SYSTEM)
    b_dev = torch.from_numpy(b).cuda()
    x_dev = torch.from_numpy(x).cuda()
    r_dev = torch.empty_like(b_dev)
    stream = torch.cuda.current_stream()
    torch.cuda.synchronize()
    device_before = torch.cuda.current_device()
    for _ in range(2):
        r_dev.fill_(float("nan"))
        rel = np.zeros(k)
        code = _lib.lib().gdtp_residual_static(s.handle, C.c_void_p(b_dev.data_ptr()), C.c_void_p(x_dev.data_ptr()),
                                               C.c_void_p(r_dev.data_ptr()), k, rel.ctypes.data_as(C.c_void_p),
                                               C.c_void_p(stream.cuda_stream))
        _lib.check(code)
        assert torch.cuda.current_device() == device_before  # the caller's device is left as it was
        np.testing.assert_allclose(rel, ref, rtol=1e-12)
        r = r_dev.cpu().numpy()
        assert np.abs(r - r_ref).max() <= 1e-12 * np.abs(r_ref).max()


def test_static_residual_rejects_oversized_batches(built_lib):
    import torch
    from gradientdomaintextureprocessing_b200 import _lib
    from gradientdomaintextureprocessing_b200.hierarchy import InitializeHierarchy
    from gradientdomaintextureprocessing_b200.system import System
    g = load_golden("torus128")
    h = InitializeHierarchy(golden_mesh(g), levels=4)
    s = System(h)
    s.update(float(g["meta/weights"][0]), 1.0)
    n = h.counts(0)["numTexels"]
    buf = torch.zeros(n * 65, dtype=torch.float64, device="cuda")
    rel = np.zeros(65)
    code = _lib.lib().gdtp_residual_static(s.handle, C.c_void_p(buf.data_ptr()), C.c_void_p(buf.data_ptr()),
                                           C.c_void_p(buf.data_ptr()), 65, rel.ctypes.data_as(C.c_void_p), None)
    assert code == -1 and b"static scratch limit" in _lib.lib().gdtp_last_error()
