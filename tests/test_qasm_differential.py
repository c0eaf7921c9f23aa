"""The engine's QASM reader against the reference's own parser
(qasm::parse_any, run by oracle/_ref/ref_qasmdump) on every golden program and
on seeded mutations of them: truncations, single-byte replacements (with
characters the grammar uses), duplicated spans and deleted spans.  Whenever
the reference accepts a text the engine must accept it with the same
instructions (op, qubits, parameters as identical doubles); whenever the
reference refuses it the engine must refuse it with TNBP_EPARSE.  Texts on
which the reference's behaviour is undefined (a signed register size or
index, which it converts from a negative double to size_t) or would allocate
without bound (a size of more than six digits) are left out, and so are
indices and sizes written as a bare exponent marker ("q[e]", "q[.E]"): the
reference's number scanner reads those as 0, the engine refuses them as
malformed (its one deliberate difference).  Runs on the CPU."""
import math
import os
import random
import re
import subprocess

import pytest

import tnbp_b200 as tb

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DUMP = os.path.join(ROOT, "oracle", "_ref", "ref_qasmdump")
INPUTS = os.path.join(ROOT, "tests", "golden", "inputs")
ALPHABET = "qQ[]();,:-+>*/. \n0123456789e\"'_abcxyzpiuOPENQASM3"
UNDEFINED = re.compile(r"\[\s*[-+]|\[[^\]]*:\s*[-+]|\d{7,}")
BARE_EXPONENT = re.compile(r"[\[:]\s*\.?[eE]")


def mutations(src, rng, n):
    out = []
    for i in range(n):
        v = src
        k = i % 4
        if k == 0:
            v = v[: rng.randrange(len(v))]
        elif k == 1:
            p = rng.randrange(len(v))
            v = v[:p] + rng.choice(ALPHABET) + v[p + 1:]
        elif k == 2:
            a = rng.randrange(len(v))
            b = min(len(v), a + 1 + rng.randrange(12))
            v = v[:a] + v[a:b] + v[a:]
        else:
            a = rng.randrange(len(v))
            b = min(len(v), a + 1 + rng.randrange(6))
            v = v[:a] + v[b:]
        out.append(v)
    return out


def ours(src):
    try:
        ins = tb.qasm_instructions(src)
    except tb.TnbpError as e:
        assert e.code == tb.EPARSE, str(e)
        return None
    return ins


def theirs(line):
    if line == "ERR":
        return None
    out = []
    for rec in line.split(";")[1:]:
        f = rec.split(",")
        op, nq = int(f[0]), int(f[1])
        qs = [int(x) for x in f[2:2 + nq]]
        npar = int(f[2 + nq])
        ps = [float.fromhex(x) for x in f[3 + nq:3 + nq + npar]]
        out.append((op, qs, ps))
    return out


def same_double(a, b):
    return (math.isnan(a) and math.isnan(b)) or a == b


@pytest.mark.skipif(not os.path.exists(DUMP), reason="oracle/_ref/ref_qasmdump is not built (needs the reference tree)")
def test_qasm_reader_matches_reference_parser(tmp_path):
    rng = random.Random(20261204)
    texts = []
    for name in sorted(os.listdir(INPUTS)):
        if not name.endswith(".qasm"):
            continue
        src = open(os.path.join(INPUTS, name)).read()
        src = src[:6000]
        texts.append(src)
        texts.extend(mutations(src, rng, 150))
    # hand-written cases around the grammar's corners
    texts += [
        "OPENQASM 2.0;\nqreg q[3];\nU3(pi/2, -pi/4, 2*tau - 1e-3) q[0];\ncx q[0],q[1];\n",
        "OPENQASM 2.0;\nqreg q[2];\nrx(1/0) q[0];\n",
        "OPENQASM 2.0;\nqreg q[2];\nRX(--1.5e2) q;\nbarrier q[1], q[0];\nreset q;\n",
        "OPENQASM 2.0;\nqreg q[2];creg c[2];\nmeasure q[1] -> c[0];\nmeasure q -> c[1];\n",
        "qreg q[4];\ncx q;\ncz q[0],q[1],q[2];\nfoo(0.5) q[0],q[3];\n",
        "OPENQASM 3;\nqubit[4] q;\nbit[2] c;\nh q[1:3];\nc[0] = measure q[0];\nbit b = measure q[3];\n",
        "OPENQASM 3.0;\nqubit q;\nbit c;\nc = measure q;\nctrl @ x q;\n",
        "OPENQASM 3;\nqubit[2] q;\nx q[0:3];\n",
        "OPENQASM 3;\nqubit[2] q;\nbit[2] c;\nc = measure q[0];\n",
        "/* header */ OPENQASM 2.0; // comment\ninclude \"qelib1.inc\";\nqreg q[2];\nrzz(1e5.3) q[0],q[1];\n",
        "OPENQASM 2.0;\nqreg q[2];\nu2(.5, 2.) q[0];\np(1e400) q[1];\n",
    ]
    texts = [t for t in texts if not UNDEFINED.search(t) and not BARE_EXPONENT.search(t)]
    paths = []
    for i, t in enumerate(texts):
        p = tmp_path / f"t{i}.qasm"
        p.write_bytes(t.encode("latin-1", errors="replace"))
        paths.append(str(p))
    r = subprocess.run([DUMP, *paths], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    lines = r.stdout.splitlines()
    assert len(lines) == len(texts)
    accepted = refused = 0
    for t, line in zip(texts, lines):
        want = theirs(line)
        got = ours(t)
        if want is None:
            assert got is None, f"the reference refuses, the engine accepts:\n{t!r}"
            refused += 1
            continue
        assert got is not None, f"the reference accepts, the engine refuses:\n{t!r}"
        assert len(got) == len(want), t
        for (op, qs, ps, nq), (rop, rqs, rps) in zip(got, want):
            assert op == rop and nq == len(rqs) and qs == rqs[: min(4, nq)], t
            ps = ps[:3]
            assert len(ps) == min(3, len(rps)) and all(same_double(a, b) for a, b in zip(ps, rps)), t
        accepted += 1
    assert accepted > 100 and refused > 100, (accepted, refused)
