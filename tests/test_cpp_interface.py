"""The C++ interface (include/tnbp_b200.hpp) compiled with g++ against the
built library: host-side names, argument meanings and the exceptions the
reference throws (tests/cpp/hpp_host_checks.cc).  Runs on the CPU."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "tnbp_b200", "libtnbp_b200.so")


@pytest.mark.skipif(shutil.which("g++") is None, reason="no C++ compiler")
def test_cpp_interface_host_checks(tmp_path):
    if not os.path.exists(LIB):
        pytest.fail(f"{LIB} is not built: run `python tnbp_b200/build.py`")
    exe = str(tmp_path / "hpp_host_checks")
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "hpp_host_checks.cc"), "-L", os.path.dirname(LIB),
                    "-ltnbp_b200", f"-Wl,-rpath,{os.path.dirname(LIB)}", "-o", exe], check=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.count("ok ") >= 13, r.stdout
