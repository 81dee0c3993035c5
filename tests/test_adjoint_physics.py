"""Reverse-mode Euler adjoints (volume flux and HLLC) against forward-mode differentiation of
the same device functors, on the host: ``tests/native/euler_adjoint_check.cu`` is compiled
by nvcc as host code (the functors are ``__host__ __device__``) and checks 20,000 random
states, requiring every HLLC branch (upwind side x star region, pStar clamp, shock factors)
to be hit and all gradients to agree to 1e-11 relative."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.skipif(shutil.which("nvcc") is None, reason="nvcc not available")
def test_euler_adjoint_matches_forward_mode(tmp_path):
    exe = str(tmp_path / "euler_adjoint_check")
    subprocess.run(["nvcc", "-std=c++17", "--expt-relaxed-constexpr", "-O2", "-Wno-deprecated-gpu-targets", "-x",
                    "cu", os.path.join(HERE, "native", "euler_adjoint_check.cu"), "-o", exe], check=True,
                   capture_output=True)
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
