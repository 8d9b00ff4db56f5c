"""The closed-form partials of the WENO face flux that the scalar-advection tangent
linear and adjoint use (csrc/weno_partials.cuh) equal the face flux evaluated on dual
numbers, on every branch (upwind side, u = 0, nonlinear weights, positivity limiter,
reduced weights).  A host program compiled by nvcc; no GPU is needed."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_closed_form_partials_match_dual_numbers(tmp_path):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not found")
    exe = str(tmp_path / "weno_partials_check")
    src = os.path.join(ROOT, "tests", "weno_partials_check.cu")
    r = subprocess.run([nvcc, "-O2", "-std=c++17", "-fmad=false", "-I", os.path.join(ROOT, "fdd3260_b200", "csrc"),
                        "-I", os.path.join(ROOT, "include"), src, "-o", exe], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
