"""The C++ interface (include/tnbp_b200.hpp) on the device: the estimator
loop through State and the same program served through Server agree
(1e-10, complex128); SaveTPS / LoadTPS by their C++ names reproduce the
state exactly; a cancelled request throws (tests/cpp/hpp_device_checks.cc)."""
import os
import shutil
import subprocess

import pytest

from records import load_probe

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "tnbp_b200", "libtnbp_b200.so")
G = os.path.join(ROOT, "tests", "golden")


@pytest.mark.skipif(shutil.which("g++") is None, reason="no C++ compiler")
@pytest.mark.parametrize("name", ["ki3x3", "rc3x3"])
def test_cpp_interface_on_the_device(name, tmp_path):
    exe = str(tmp_path / "hpp_device_checks")
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "hpp_device_checks.cc"), "-L", os.path.dirname(LIB),
                    "-ltnbp_b200", f"-Wl,-rpath,{os.path.dirname(LIB)}", "-o", exe], check=True)
    _, meta = load_probe(os.path.join(G, f"probe_{name}.npz"))
    r = subprocess.run([exe, os.path.join(G, "inputs", f"{name}.qasm"), os.path.join(G, "inputs", f"{name}.txt"),
                        str(meta["chi"]), repr(meta["tol"]), str(meta["maxit"]), repr(meta["sv_min"]),
                        str(tmp_path / "ck.dat")], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
