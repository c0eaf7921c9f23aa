"""Host code under AddressSanitizer / UndefinedBehaviorSanitizer: the QASM,
Pauli and TPO builders (including OptTPObySVD) and the checkpoint reader on
every golden input plus seeded truncations and mutations of them
(tests/cpp/host_sanitize.cc).  Malformed input must be refused with a status,
never crash.  Runs on the CPU."""
import glob
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "tnbp_b200", "csrc")
G = os.path.join(ROOT, "tests", "golden")


@pytest.mark.skipif(shutil.which("g++") is None, reason="no C++ compiler")
def test_host_code_under_asan_ubsan(tmp_path):
    exe = str(tmp_path / "host_sanitize")
    subprocess.run(["g++", "-std=c++17", "-O1", "-g", "-fsanitize=address,undefined", "-fno-sanitize-recover=all",
                    "-fno-omit-frame-pointer", "-I", CSRC, os.path.join(ROOT, "tests", "cpp", "host_sanitize.cc"),
                    os.path.join(CSRC, "host_setup.cpp"),
                    os.path.join(CSRC, "qasm_text.cpp"), os.path.join(CSRC, "tps_io.cpp"), "-o", exe], check=True)
    qasm = sorted(glob.glob(os.path.join(G, "inputs", "*.qasm")))
    pauli = sorted(glob.glob(os.path.join(G, "inputs", "*.txt")))
    ckpt = [os.path.join(G, "ckpt_ki3x3r000000.dat"), os.path.join(G, "inputs", "ki3x3r.qasm")]
    env = dict(os.environ, ASAN_OPTIONS="detect_leaks=0:abort_on_error=0", UBSAN_OPTIONS="print_stacktrace=1")
    r = subprocess.run([exe, *qasm, "--", *pauli, "--", *ckpt], capture_output=True, text=True, timeout=900,
                       cwd=str(tmp_path), env=env)
    assert r.returncode == 0, (r.stdout + r.stderr)[-4000:]
    ok, refused = (int(x) for x in r.stdout.split()[1::2])
    assert ok > 10 and refused > 100, r.stdout
