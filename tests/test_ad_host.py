"""Derivative building blocks of the adjoint, checked on the host (no GPU):
the dual-number Jacobian of the face flux against long-double central
differences, and the hand-written HLLC adjoint against the transposed dual
Jacobian (tests/ad_host_check.cu, compiled with nvcc as host code)."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


@pytest.fixture(scope="module")
def result(tmp_path_factory):
    nvcc = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
    if not os.path.exists(nvcc) and not shutil.which("nvcc"):
        pytest.skip("nvcc not available")
    exe = str(tmp_path_factory.mktemp("adhost") / "ad_host_check")
    subprocess.check_call([nvcc, "-std=c++17", "-O2", "-gencode", "arch=compute_100a,code=sm_100a",
                           "-I", os.path.join(ROOT, "include"), os.path.join(HERE, "ad_host_check.cu"), "-o", exe])
    out = subprocess.check_output([exe], text=True).split()
    return dict(fd=float(out[1]), adj=float(out[3]))


def test_dual_flux_jacobian_matches_long_double_fd(result):
    assert result["fd"] < 1e-7


def test_hllc_adjoint_matches_dual_jacobian(result):
    assert result["adj"] < 1e-12
