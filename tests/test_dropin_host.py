"""The drop-in tensor backend that tnbp's apps compile against
(include/tnbp_dropin/gqten/gqten.h): contraction, SVD, truncated SVD, QR,
transpose/reshape, trace and linear combination checked on the CPU by their
defining identities (tests/cpp/dropin_gqten_checks.cc), under AddressSanitizer
and UndefinedBehaviorSanitizer."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(shutil.which("g++") is None, reason="no C++ compiler")
def test_dropin_tensor_backend(tmp_path):
    exe = str(tmp_path / "dropin_gqten_checks")
    subprocess.run(["g++", "-std=c++17", "-O1", "-g", "-fsanitize=address,undefined", "-fno-sanitize-recover=all",
                    "-I", os.path.join(ROOT, "include", "tnbp_dropin"),
                    os.path.join(ROOT, "tests", "cpp", "dropin_gqten_checks.cc"), "-o", exe], check=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300,
                       env=dict(os.environ, ASAN_OPTIONS="detect_leaks=1"))
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.count("ok ") >= 20, r.stdout
