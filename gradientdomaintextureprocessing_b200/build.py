"""Builds the native library ``libgdtp.so`` in-tree with nvcc for sm_100a.

    python -m gradientdomaintextureprocessing_b200.build

Host set-up code (C++17 + OpenMP) and the CUDA kernels are compiled by nvcc
with the system g++ as host compiler; objects go to ``_build/`` and are
compiled in parallel.  No CUDA device is needed to build.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libgdtp.so")
BUILD = os.path.join(ROOT, "_build")

SOURCES = [
    "setup/atlas.cpp", "setup/grid.cpp", "setup/csr.cpp", "setup/boundary.cpp", "setup/assembly.cpp",
    "setup/galerkin.cpp", "setup/bsolve.cpp", "setup/metric.cpp", "io/png.cpp", "io/ply.cpp", "io/texture_io.cpp", "capi_io.cpp",
    "capi_hierarchy.cpp", "capi_system.cpp", "capi_metric.cpp", "capi_geodesics.cpp", "geodesics.cu", "capi_server.cpp", "server.cpp", "system.cu", "numeric.cu", "brush.cu", "noalloc.cu",
    "kernels/vcycle_kernels.cu", "kernels/tile_smoother.cu", "kernels/dense_kernels.cu", "kernels/coarse_cycle.cu", "kernels/geodesic_kernels.cu", "kernels/assembly_kernels.cu",
]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _host_cxx() -> str:
    return "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else (shutil.which("g++") or "g++")


def _flags() -> list[str]:
    return ["-O3", "-std=c++17", "-lineinfo", "-ccbin", _host_cxx(), "-Xcompiler", "-fPIC,-fopenmp,-O3",
            "--expt-relaxed-constexpr", "-I" + CSRC, "-I" + os.path.join(ROOT, "include")] + ARCH


def _compile(src: str) -> str:
    obj = os.path.join(BUILD, src.replace("/", "_") + ".o")
    path = os.path.join(CSRC, src)
    lang = ["-x", "cu"] if src.endswith(".cu") else ["-x", "c++"]
    deps = [path] + [os.path.join(dp, f) for dp, _, fs in os.walk(CSRC) for f in fs if f.endswith((".h", ".cuh"))]
    if os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(d) for d in deps):
        return obj
    cmd = [_nvcc()] + _flags() + lang + ["-c", path, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return obj


def build(verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        objs = list(ex.map(_compile, SOURCES))
    if not os.path.exists(OUT) or os.path.getmtime(OUT) < max(os.path.getmtime(o) for o in objs):
        cmd = [_nvcc(), "-shared", "-ccbin", _host_cxx()] + ARCH + ["-o", OUT] + objs + ["-lgomp", "-lcudart", "-ldl"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    if verbose:
        print(OUT)
    return OUT


if __name__ == "__main__":
    build(verbose=True)
    sys.exit(0)
