"""Host-side helpers of the kernels, compiled by nvcc as host code (CPU only):
the invariant-divisor arithmetic of the index kernels (FastDiv,
tnbp_b200/csrc/kernels.cuh: Granlund-Montgomery multiply-high and shift)
against exact division on every divisor up to 70000, powers of two and their
neighbours, 20000 random divisors, and edge and random dividends below 2^31
(tests/cpp/fastdiv_check.cu); and which sites the site-resident sweep kernel
takes (tests/cpp/site_sweep_limits.cu)."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")


def _build_and_run(tmp_path, name):
    if not (os.path.exists(NVCC) or shutil.which("nvcc")):
        pytest.skip("nvcc not available")
    exe = str(tmp_path / name)
    subprocess.check_call([NVCC, "-std=c++17", "-O2", "-I", os.path.join(ROOT, "tnbp_b200", "csrc"),
                           os.path.join(HERE, "cpp", name + ".cu"), "-o", exe])
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "mismatches 0" in r.stdout


def test_fast_division_equals_exact_division(tmp_path):
    _build_and_run(tmp_path, "fastdiv_check")


def test_site_sweep_takes_the_documented_sites(tmp_path):
    _build_and_run(tmp_path, "site_sweep_limits")
