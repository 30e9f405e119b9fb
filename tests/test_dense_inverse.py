"""Host dense SPD inverse (coarsest level, boundary blocks, Schur complement)
and the parallel CSR builders of the set-up: compiled with the library's host
sources and checked natively."""
import os
import subprocess
import tempfile

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "gradientdomaintextureprocessing_b200", "csrc")


def test_dense_spd_inverse_native():
    with tempfile.TemporaryDirectory() as tmp:
        exe = os.path.join(tmp, "dense_inverse_check")
        subprocess.run(["g++", "-std=c++17", "-O2", "-fopenmp", "-I", CSRC, os.path.join(ROOT, "tests", "native", "dense_inverse_check.cpp"),
                        os.path.join(CSRC, "setup", "bsolve.cpp"), os.path.join(CSRC, "setup", "csr.cpp"), "-o", exe], check=True)
        out = subprocess.run([exe], capture_output=True, text=True, timeout=300)
        assert out.returncode == 0, out.stdout + out.stderr
        assert out.stdout.strip() == "ok"


def test_parallel_csr_builders_native():
    with tempfile.TemporaryDirectory() as tmp:
        exe = os.path.join(tmp, "csr_check")
        subprocess.run(["g++", "-std=c++17", "-O2", "-fopenmp", "-I", CSRC, os.path.join(ROOT, "tests", "native", "csr_check.cpp"),
                        os.path.join(CSRC, "setup", "csr.cpp"), "-o", exe], check=True)
        out = subprocess.run([exe], capture_output=True, text=True, timeout=300)
        assert out.returncode == 0, out.stdout + out.stderr
        assert out.stdout.strip() == "ok"
