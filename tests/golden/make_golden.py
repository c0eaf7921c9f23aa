"""Regenerate the golden fixtures in tests/golden/ from the reference itself.

The fixtures pin the oracle and the B200 engine to r-ccs-cms/tnbp's own code:
the reference's unchanged headers and apps are compiled by oracle/Makefile
(against the project's CPU gqten and single-rank MPI stand-ins) into
oracle/_ref/, and this script runs them on seeded synthetic inputs:

  probe_<name>.npz   every intermediate tensor of the estimator loop
                     (oracle/ref_probe.cc): TPO layers, V/E after AbsorbTPO,
                     E after the first BP sweep and after BP, conditions,
                     truncation dims/errors, V/E after truncation, one- and
                     two-site expectation values
  host_<name>.json   lattice edges, greedy layers, leg order, BFS paths,
                     parsed QASM instructions, TPO layer shapes, Pauli
                     classification (oracle/ref_hostparity.cc)
  opttpo_<name>.npz  TPO layers before and after the reference's OptTPObySVD
                     (small circuits: every site operator)
  opttpo_kobe.json   the same on the reference's kicked_ising.qasm, reduced
                     to gauge-invariant data (bond dimensions, per-leg
                     singular values of every site operator)
  opt_<name>.json    the estimator app's printed values with --do_opt_tpo 1
  tpocount_<name>.npz  TPO layers of the reference's manual gate-number
                     layering (QasmToTPO with num_gates) for several splits
  count_<name>.json  the estimator app's printed values with --num_gates
  ckpt_<name>000000.dat + ckpt_<name>.json
                     a checkpoint the reference's estimator_restart app saved
                     after one pass of a circuit (SaveTPS, iotps.h) and the
                     values it printed after a second pass loaded from it
  config1.json       observables of the 4x4 kicked-Ising workload from the
                     reference apps kicked_ising_lattice and estimator
  est_rc10x10.json   the estimator app's printed values on the benchmark's
                     random-circuit workload at full size (10x10, 12 U3 + CZ
                     layers, chi 32, 64-term observable; --only est_rc10)

usage: python tests/golden/make_golden.py [--ref <reference tree>]   (default: $TNBP_REFERENCE)
Needs the reference sources (only in the build container); the fixtures it
writes are what the tests read everywhere else.
"""
import argparse
import json
import math
import os
import re
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, HERE)
from records import read_records  # noqa: E402

sys.path.insert(0, os.path.join(ROOT, "oracle"))
from reference_root import reference_root  # noqa: E402

INPUTS = os.path.join(HERE, "inputs")
REF_BIN = os.path.join(ROOT, "oracle", "_ref")


# ----------------------------------------------------------- input writers
def lattice_edges(L):
    e = []
    for iy in range(L):
        for ix in range(L):
            s = ix + L * iy
            if ix + 1 < L:
                e.append((s, s + 1))
            if iy + 1 < L:
                e.append((s, s + L))
    return e


def kicked_ising_qasm(Lx, Ly, steps, theta_j, theta_h):
    """RZZ(theta_j) on horizontal then vertical edges, RX(theta_h) on every
    site, one barrier per step (the 4x4 kicked-Ising workload's form)."""
    n = Lx * Ly
    out = ["OPENQASM 2.0;", 'include "qelib1.inc";', f"qreg q[{n}];"]
    for _ in range(steps):
        for iy in range(Ly):
            for ix in range(Lx - 1):
                i = ix + Lx * iy
                out.append(f"rzz({theta_j!r}) q[{i}],q[{i + 1}];")
        for iy in range(Ly - 1):
            for ix in range(Lx):
                i = ix + Lx * iy
                out.append(f"rzz({theta_j!r}) q[{i}],q[{i + Lx}];")
        for i in range(n):
            out.append(f"rx({theta_h!r}) q[{i}];")
        out.append("barrier q;")
    return "\n".join(out) + "\n"


def colourings(Lx, Ly):
    hev = [(ix + Lx * iy, ix + 1 + Lx * iy) for iy in range(Ly) for ix in range(0, Lx - 1, 2)]
    hod = [(ix + Lx * iy, ix + 1 + Lx * iy) for iy in range(Ly) for ix in range(1, Lx - 1, 2)]
    vev = [(ix + Lx * iy, ix + Lx * (iy + 1)) for iy in range(0, Ly - 1, 2) for ix in range(Lx)]
    vod = [(ix + Lx * iy, ix + Lx * (iy + 1)) for iy in range(1, Ly - 1, 2) for ix in range(Lx)]
    return [hev, hod, vev, vod]


def random_circuit_qasm(Lx, Ly, layers, rng):
    """U3(theta, phi, lambda ~ U[0, 2pi)) on every qubit, then CZ on edge
    colouring (layer mod 4): H-even, H-odd, V-even, V-odd."""
    n = Lx * Ly
    out = ["OPENQASM 2.0;", 'include "qelib1.inc";', f"qreg q[{n}];"]
    # every lattice edge appears once in a leading identity-free CZ^2 pass so
    # the edge list (EdgesFromQasm) is the full lattice
    cols = colourings(Lx, Ly)
    for layer in range(layers):
        for i in range(n):
            a, b, c = (float(v) for v in rng.uniform(0, 2 * math.pi, 3))
            out.append(f"u3({a!r},{b!r},{c!r}) q[{i}];")
        for (i, j) in cols[layer % 4]:
            out.append(f"cz q[{i}],q[{j}];")
        out.append("barrier q;")
    return "\n".join(out) + "\n"


def zz_cx_qasm(Lx, Ly, steps, theta, theta_h):
    """Kicked Ising with each ZZ rotation compiled as cx, rz, cx (the form of
    the reference's apps/estimator/kicked_ising.qasm): operator rank 4 per
    bond before OptTPObySVD, 2 after."""
    n = Lx * Ly
    out = ["OPENQASM 2.0;", 'include "qelib1.inc";', f"qreg q[{n}];"]
    for _ in range(steps):
        for (i, j) in lattice_edges_rect(Lx, Ly):
            out += [f"cx q[{i}],q[{j}];", f"rz({theta!r}) q[{j}];", f"cx q[{i}],q[{j}];"]
        for i in range(n):
            out.append(f"rx({theta_h!r}) q[{i}];")
        out.append("barrier q;")
    return "\n".join(out) + "\n"


def opt_mix_qasm():
    """2x3 lattice: CZ twice on one edge (rank 4, compresses to 1), a
    distance-2 cx (pass-through bonds), rzz and cx on one edge, U3s."""
    lines = ["OPENQASM 2.0;", 'include "qelib1.inc";', "qreg q[6];"]
    for (i, j) in lattice_edges_rect(3, 2):
        lines.append(f"cz q[{i}],q[{j}];")
    lines += ["cz q[0],q[1];", "u3(0.3,1.1,-0.4) q[1];", "cx q[0],q[2];", "rzz(0.37) q[4],q[5];",
              "cx q[4],q[5];", "barrier q;", "h q[3];", "cz q[3],q[4];", "cz q[3],q[4];", "cx q[1],q[4];",
              "barrier q;"]
    return "\n".join(lines) + "\n"


def leg_spectra(t):
    """Singular values of every bond-leg unfolding of a site operator: equal
    for two TPOs that differ by unitaries on their bonds."""
    out = []
    for k in range(t.ndim - 2):
        out.append(np.linalg.svd(np.moveaxis(t, k, 0).reshape(t.shape[k], -1), compute_uv=False).tolist())
    return out


def run_opttpo(name, qasm_path, eps_list, lattice=None, full=True):
    arrays = {}
    summary = {}
    for eps in eps_list:
        args = [os.path.join(REF_BIN, "ref_hostparity"), "opttpo", qasm_path, repr(eps)]
        if lattice:
            args += [str(lattice[0]), str(lattice[1])]
        d = json.loads(subprocess.check_output(args, text=True))
        arrays["edges"] = np.array(d["edges"], np.int32)
        tag = f"eps{eps:g}"
        layers = []
        for stage in ("before", "after"):
            for l, layer in enumerate(d[stage]):
                for s, (shape, flat) in enumerate(layer):
                    a = np.array(flat, np.float64).reshape(-1, 2)
                    t = (a[:, 0] + 1j * a[:, 1]).reshape(shape, order="F")
                    if full:
                        arrays[f"{tag}/{stage}/{l}/{s}"] = t
                    elif stage == "after":
                        while len(layers) <= l:
                            layers.append([])
                        layers[l].append(dict(shape=list(shape), norm=float(np.linalg.norm(t)),
                                              legs=leg_spectra(t)))
        summary[tag] = dict(eps=eps, layers=layers)
    if full:
        np.savez_compressed(os.path.join(HERE, f"opttpo_{name}.npz"), **arrays)
    else:
        summary["edges"] = arrays["edges"].tolist()
        with open(os.path.join(HERE, f"opttpo_{name}.json"), "w") as f:
            json.dump(summary, f, separators=(",", ":"))
    print(f"opttpo_{name}: eps {eps_list}")


def run_opt_estimator(name, qasm, pauli, chi, sv_min, tol, maxit, eps):
    """The reference estimator app with --do_opt_tpo 1: its printed values."""
    qp = os.path.join(INPUTS, f"{name}.qasm")
    pp = os.path.join(INPUTS, f"{name}.txt")
    with open(qp, "w") as f:
        f.write(qasm)
    with open(pp, "w") as f:
        f.write(pauli)
    out = subprocess.check_output(
        [os.path.join(REF_BIN, "estimator"), "--circuit", qp, "--sparse_pauli", pp, "--max_bond_dim", str(chi),
         "--bp_tolerance", repr(tol), "--max_bp_iterations", str(maxit), "--sv_min", repr(sv_min),
         "--do_opt_tpo", "1", "--eps_opt_tpo", repr(eps)], text=True)
    one = [float(v) for v in re.findall(r"single site operator at site \d+ (\S+)", out)]
    two = [float(v) for v in re.findall(r"two site operator at sites \(\d+,\d+\) (\S+)", out)]
    dims = [int(v) for v in re.findall(r"bond dim = (\d+)", out)]
    conds = [float(v) for v in re.findall(r"condition at step \d+ = (\S+)", out)]
    res = dict(chi=chi, sv_min=sv_min, tol=tol, maxit=maxit, eps_opt_tpo=eps, one=one, two=two, bond_dims=dims,
               conditions=conds)
    with open(os.path.join(HERE, f"opt_{name}.json"), "w") as f:
        json.dump(res, f, indent=1)
    print(f"opt_{name}: {len(one)} one-site, {len(two)} two-site values, conditions {conds}")


def run_estimator_values(name, qp, pp, chi, sv_min, tol, maxit):
    """The reference estimator app on an input pair: every printed value
    (one- and two-site terms in print order, conditions, bond dims) and the
    app's wall time."""
    import time
    t = time.perf_counter()
    out = subprocess.check_output(
        [os.path.join(REF_BIN, "estimator"), "--circuit", qp, "--sparse_pauli", pp, "--max_bond_dim", str(chi),
         "--bp_tolerance", repr(tol), "--max_bp_iterations", str(maxit), "--sv_min", repr(sv_min)], text=True)
    dt = time.perf_counter() - t
    one = [[int(s_), float(v)] for s_, v in re.findall(r"single site operator at site (\d+) (\S+)", out)]
    two = [[int(a_), int(b_), float(v)] for a_, b_, v in
           re.findall(r"two site operator at sites \((\d+),(\d+)\) (\S+)", out)]
    dims = [int(v) for v in re.findall(r"bond dim = (\d+)", out)]
    conds = [float(v) for v in re.findall(r"condition at step \d+ = (\S+)", out)]
    res = dict(chi=chi, sv_min=sv_min, tol=tol, maxit=maxit, one=one, two=two, final_bond_dims=dims[-200:],
               conditions=conds, seconds=dt)
    with open(os.path.join(HERE, f"est_{name}.json"), "w") as f:
        json.dump(res, f, indent=1)
    print(f"est_{name}: {len(one)} one-site, {len(two)} two-site values, {len(conds)} sweeps, {dt:.1f} s")


def kicked_ising_no_barrier(Lx, Ly, steps, theta_j, theta_h):
    """kicked_ising_qasm without barriers (manual layering counts instructions)."""
    return "\n".join(l for l in kicked_ising_qasm(Lx, Ly, steps, theta_j, theta_h).splitlines()
                     if not l.startswith("barrier")) + "\n"


def run_tpocount(name, qasm, splits):
    qp = os.path.join(INPUTS, f"{name}.qasm")
    with open(qp, "w") as f:
        f.write(qasm)
    arrays = {}
    for k, split in enumerate(splits):
        arg = ",".join(str(n) for n in split)
        d = json.loads(subprocess.check_output([os.path.join(REF_BIN, "ref_hostparity"), "tpocount", qp, arg],
                                               text=True))
        arrays["edges"] = np.array(d["edges"], np.int32)
        arrays[f"split{k}"] = np.array(split, np.int32)
        for l, layer in enumerate(d["layers"]):
            for s_, (shape, flat) in enumerate(layer):
                a = np.array(flat, np.float64).reshape(-1, 2)
                arrays[f"split{k}/{l}/{s_}"] = (a[:, 0] + 1j * a[:, 1]).reshape(shape, order="F")
    np.savez_compressed(os.path.join(HERE, f"tpocount_{name}.npz"), **arrays)
    print(f"tpocount_{name}: {len(splits)} splits")


def run_count_estimator(name, qasm, pauli, chi, sv_min, tol, maxit, split):
    """The reference estimator app with --num_gates: its printed values."""
    qp = os.path.join(INPUTS, f"{name}.qasm")
    pp = os.path.join(INPUTS, f"{name}.txt")
    with open(qp, "w") as f:
        f.write(qasm)
    with open(pp, "w") as f:
        f.write(pauli)
    out = subprocess.check_output(
        [os.path.join(REF_BIN, "estimator"), "--circuit", qp, "--sparse_pauli", pp, "--max_bond_dim", str(chi),
         "--bp_tolerance", repr(tol), "--max_bp_iterations", str(maxit), "--sv_min", repr(sv_min),
         "--num_gates", ",".join(str(n) for n in split)], text=True)
    one = [float(v) for v in re.findall(r"single site operator at site \d+ (\S+)", out)]
    two = [float(v) for v in re.findall(r"two site operator at sites \(\d+,\d+\) (\S+)", out)]
    dims = [int(v) for v in re.findall(r"bond dim = (\d+)", out)]
    res = dict(chi=chi, sv_min=sv_min, tol=tol, maxit=maxit, num_gates=list(split), one=one, two=two,
               bond_dims=dims)
    with open(os.path.join(HERE, f"count_{name}.json"), "w") as f:
        json.dump(res, f, indent=1)
    print(f"count_{name}: {len(one)} one-site, {len(two)} two-site values")


def run_checkpoint(name, qasm, pauli, chi, sv_min, tol, maxit, nlayers):
    qp = os.path.join(INPUTS, f"{name}.qasm")
    pp = os.path.join(INPUTS, f"{name}.txt")
    with open(qp, "w") as f:
        f.write(qasm)
    with open(pp, "w") as f:
        f.write(pauli)
    app = os.path.join(REF_BIN, "estimator_restart")
    base = [app, "--circuit", qp, "--sparse_pauli", pp, "--max_bond_dim", str(chi), "--bp_tolerance", repr(tol),
            "--max_bp_iterations", str(maxit), "--sv_min", repr(sv_min)]
    prefix = os.path.join(HERE, f"ckpt_{name}")
    subprocess.check_output(base + ["--step_end", "1", "--savename", prefix], text=True)
    out = subprocess.check_output(base + ["--loadname", prefix, "--step_start", "1", "--step_end", "2",
                                          "--measurement_barrier", str(nlayers - 1)], text=True)
    one = [float(v) for v in re.findall(r"single site operator for step 1 barrier \d+ at site \d+ (\S+)", out)]
    two = [float(v) for v in re.findall(r"two site operator for step 1 barrier \d+ at sites \(\d+,\d+\) (\S+)", out)]
    dims = [int(v) for v in re.findall(r"bond dim = (\d+)", out)]
    res = dict(chi=chi, sv_min=sv_min, tol=tol, maxit=maxit, one=one, two=two, bond_dims=dims)
    with open(os.path.join(HERE, f"ckpt_{name}.json"), "w") as f:
        json.dump(res, f, indent=1)
    print(f"ckpt_{name}: {len(one)} one-site, {len(two)} two-site values after the restart")


def random_paulis(n, edges, nterms, rng, extra_text=True):
    lines = ["# seeded sparse Pauli observable", "// second comment style", ""]
    letters = "XYZ"
    for t in range(nterms):
        k = int(rng.integers(1, 5))
        if t % 5 == 0:
            a, b = edges[int(rng.integers(0, len(edges)))]
            qs = [a, b]
        else:
            qs = list(rng.choice(n, size=min(k, n), replace=False))
        s = ["I"] * n
        for q in qs:
            s[n - 1 - int(q)] = letters[int(rng.integers(0, 3))]
        c = float(rng.normal())
        if t % 3 == 0:
            lines.append(f"{c!r} {float(rng.normal())!r} {''.join(s)}")
        else:
            lines.append(f"{c!r} {''.join(s).lower() if t % 7 == 0 else ''.join(s)}")
    lines.append(f"0.5 {'I' * n}")  # identity term: dropped by ClassifyOps
    return "\n".join(lines) + "\n"


# ------------------------------------------------------------------ runners
def run_probe(name, qasm, pauli, chi, sv_min, tol, maxit, lattice=None):
    qp = os.path.join(INPUTS, f"{name}.qasm")
    pp = os.path.join(INPUTS, f"{name}.txt")
    with open(qp, "w") as f:
        f.write(qasm)
    with open(pp, "w") as f:
        f.write(pauli)
    out = os.path.join("/tmp", f"probe_{name}.bin")
    extra = [str(lattice[0]), str(lattice[1])] if lattice else []
    subprocess.check_call([os.path.join(REF_BIN, "ref_probe"), qp, pp, out, str(chi), repr(sv_min),
                           repr(tol), str(maxit)] + extra)
    recs = read_records(out)
    meta = dict(chi=chi, sv_min=sv_min, tol=tol, maxit=maxit, lattice=lattice)
    np.savez_compressed(os.path.join(HERE, f"probe_{name}.npz"), __meta__=json.dumps(meta), **recs)
    print(f"probe_{name}: {len(recs)} records")


def run_hostparity(name, args):
    out = subprocess.check_output([os.path.join(REF_BIN, "ref_hostparity")] + args, text=True)
    data = json.loads(out)
    with open(os.path.join(HERE, f"host_{name}.json"), "w") as f:
        json.dump(data, f, separators=(",", ":"))
    print(f"host_{name}: keys {sorted(data)}")


def run_config1():
    """4x4 open lattice, 5 steps of RZZ(-pi/2) on every edge then RX(0.8),
    chi = 4, BP tolerance 1e-10, at most 50 sweeps; <Z> on site 5 = (1,1).
    kicked_ising_lattice flags: dt*Jz = theta_J/2 with dt = 0.25 (x pi),
    Jz = -1; dt*hx = 0.4 -> hx = 1.6/pi."""
    res = {}
    hx = 1.6 / math.pi
    out = subprocess.check_output(
        [os.path.join(REF_BIN, "kicked_ising_lattice"), "--lattice", "square", "--L", "4", "--dt", "0.25",
         "--Jz", "-1", "--hz", "0", "--hx", repr(hx), "--num_steps", "5", "--max_bond_dim", "4",
         "--bp_tolerance", "1e-10", "--max_bp_iterations", "50"], text=True)
    z = {}
    x = {}
    zz = {}
    conds = []
    for line in out.splitlines():
        m = re.search(r"measurement of Z at site (\d+) time step (\d+) = (\S+)", line)
        if m:
            z[f"{m.group(2)}/{m.group(1)}"] = float(m.group(3))
        m = re.search(r"measurement of X at site (\d+) time step (\d+) = (\S+)", line)
        if m:
            x[f"{m.group(2)}/{m.group(1)}"] = float(m.group(3))
        m = re.search(r"measurement of ZZ at sites \((\d+),(\d+)\) time step (\d+) = (\S+)", line)
        if m:
            zz[f"{m.group(3)}/{m.group(1)},{m.group(2)}"] = float(m.group(4))
        m = re.search(r"condition at time step (\d+) = (\S+)", line)
        if m:
            conds.append([int(m.group(1)), float(m.group(2))])
    res["kicked_ising_lattice"] = dict(Z=z, X=x, ZZ=zz, conditions=conds, hx=hx)
    qasm = kicked_ising_qasm(4, 4, 5, -math.pi / 2, 0.8)
    qp = os.path.join(INPUTS, "config1.qasm")
    pp = os.path.join(INPUTS, "config1.txt")
    with open(qp, "w") as f:
        f.write(qasm)
    with open(pp, "w") as f:
        f.write("1.0 0.0 " + "".join("Z" if 15 - k == 5 else "I" for k in range(16)) + "\n")
    out = subprocess.check_output(
        [os.path.join(REF_BIN, "estimator"), "--circuit", qp, "--sparse_pauli", pp, "--max_bond_dim", "4",
         "--bp_tolerance", "1e-10", "--max_bp_iterations", "50", "--sv_min", "1e-8"], text=True)
    m = re.search(r"single site operator at site 5 (\S+)", out)
    dims = [int(v) for v in re.findall(r"bond dim = (\d+)", out)]
    errs = [float(v) for v in re.findall(r"truncation error for edge \(\d+,\d+\) = (\S+)", out)]
    conds = [float(v) for v in re.findall(r"condition at step \d+ = (\S+)", out)]
    res["estimator"] = dict(Z5=float(m.group(1)), bond_dims=dims, trunc_errs=errs, conditions=conds)
    with open(os.path.join(HERE, "config1.json"), "w") as f:
        json.dump(res, f, indent=1)
    print("config1:", res["estimator"]["Z5"], res["kicked_ising_lattice"]["Z"].get("4/5"))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=reference_root())
    ap.add_argument("--only", default="")
    a = ap.parse_args()
    subprocess.check_call(["make", "-C", os.path.join(ROOT, "oracle"), f"REF={a.ref}"])
    os.makedirs(INPUTS, exist_ok=True)
    rng = np.random.default_rng(20261203)
    jobs = a.only.split(",") if a.only else ["probe", "host", "config1"]
    if "probe" in jobs:
        # P1: 3x3 kicked Ising, 3 steps, chi 2 (BP at D <= 4)
        q = kicked_ising_qasm(3, 3, 3, -math.pi / 2, 0.8)
        run_probe("ki3x3", q, random_paulis(9, lattice_edges(3), 12, rng), 2, 1e-8, 1e-10, 30)
        # P2: 3x3 random circuit, 4 layers, chi 4
        q = random_circuit_qasm(3, 3, 4, rng)
        # the colourings of 4 layers cover every edge, so EdgesFromQasm = lattice
        run_probe("rc3x3", q, random_paulis(9, lattice_edges(3), 16, rng), 4, 1e-8, 1e-10, 30)
        # P3: open chain of 6 (a tree: BP is exact), random circuit, no truncation
        chain = [(i, i + 1) for i in range(5)]
        lines = ["OPENQASM 2.0;", 'include "qelib1.inc";', "qreg q[6];"]
        for layer in range(3):
            for i in range(6):
                a_, b_, c_ = (float(v) for v in rng.uniform(0, 2 * math.pi, 3))
                lines.append(f"u3({a_!r},{b_!r},{c_!r}) q[{i}];")
            for i in range(layer % 2, 5, 2):
                lines.append(f"cx q[{i}],q[{i + 1}];")
            lines.append("barrier q;")
        run_probe("chain6", "\n".join(lines) + "\n", random_paulis(6, chain, 10, rng), 64, 1e-12, 1e-13, 40)
        # P4: 2x3 lattice with a distance-2 gate (identity pass-through tensor)
        lines = ["OPENQASM 2.0;", 'include "qelib1.inc";', "qreg q[6];"]
        for (i, j) in lattice_edges_rect(3, 2):
            lines.append(f"cz q[{i}],q[{j}];")
        lines.append("barrier q;")
        for i in range(6):
            lines.append(f"h q[{i}];")
        lines.append("cx q[0],q[2];")
        lines.append("rzz(0.37) q[3],q[5];")
        lines.append("barrier q;")
        lines.append("ry(0.3) q[1];")
        lines.append("barrier q;")
        run_probe("pass2x3", "\n".join(lines) + "\n", random_paulis(6, lattice_edges_rect(3, 2), 10, rng), 8,
                  1e-10, 1e-12, 40, lattice=(3, 2))
    if "host" in jobs:
        run_hostparity("lattice4x4", ["lattice", "4", "4"])
        run_hostparity("lattice16x16", ["lattice", "16", "16"])
        run_hostparity("lattice5x3", ["lattice", "5", "3"])
        for nm in ["ki3x3", "rc3x3", "chain6"]:
            run_hostparity(nm, ["qasm", os.path.join(INPUTS, f"{nm}.qasm"), os.path.join(INPUTS, f"{nm}.txt")])
        run_hostparity("pass2x3", ["qasm", os.path.join(INPUTS, "pass2x3.qasm"),
                                   os.path.join(INPUTS, "pass2x3.txt"), "3", "2"])
        kob = os.path.join(a.ref, "apps", "estimator")
        run_hostparity("kobe", ["qasm", os.path.join(kob, "kicked_ising.qasm"), os.path.join(kob, "H_ising_kobe.txt")])
        run_hostparity("ising_circuit", ["qasm", os.path.join(a.ref, "apps", "qasm_tpo", "ising_circuit.qasm")])
        # a v3-syntax program exercising slices, bit declarations and measure assignments
        v3 = ("OPENQASM 3;\ninclude \"stdgates.inc\";\nqubit[5] q;\nbit[2] c;\n"
              "h q[0:3];\ncx q[0], q[1];\nrz(-pi/4 + 2*0.1) q[2];\nrzz(tau/8) q[2],q[3];\n"
              "/* block */ cz q[3],q[4]; // tail\nbarrier q;\nu(1e-1, .5, -2.5e0) q[4];\n"
              "c[0] = measure q[0];\nbit x = measure q[1];\n")
        with open(os.path.join(INPUTS, "v3.qasm"), "w") as f:
            f.write(v3)
        run_hostparity("v3", ["qasm", os.path.join(INPUTS, "v3.qasm")])
    if "host_rc10" in jobs:
        # the benchmark's random-circuit workload (bench.py): 10x10, 12 layers
        sys.path.insert(0, ROOT)
        import bench
        q, p = bench.random_circuit_workload()
        for ext, txt in (("qasm", q), ("txt", p)):
            with open(os.path.join(INPUTS, f"rc10x10.{ext}"), "w") as f:
                f.write(txt)
        run_hostparity("rc10x10", ["qasm", os.path.join(INPUTS, "rc10x10.qasm"), os.path.join(INPUTS, "rc10x10.txt")])
    if "est_rc10" in jobs:
        # the benchmark's random-circuit workload at full size through the
        # reference app (BP at bond dimension <= 8, so the CPU run is short)
        sys.path.insert(0, ROOT)
        import bench
        q, p = bench.random_circuit_workload()
        for ext, txt in (("qasm", q), ("txt", p)):
            with open(os.path.join(INPUTS, f"rc10x10.{ext}"), "w") as f:
                f.write(txt)
        run_estimator_values("rc10x10", os.path.join(INPUTS, "rc10x10.qasm"), os.path.join(INPUTS, "rc10x10.txt"),
                             32, bench.SV_MIN, bench.BP_TOL, bench.BP_MAXIT)
    if "opttpo" in jobs:
        q = zz_cx_qasm(3, 3, 2, -0.7, 0.8)  # generic angle: no tie at a rank-1 cut
        qp = os.path.join(INPUTS, "zzcx3x3.qasm")
        with open(qp, "w") as f:
            f.write(q)
        run_opttpo("zzcx3x3", qp, [1e-8, 1e3])
        qp = os.path.join(INPUTS, "optmix2x3.qasm")
        with open(qp, "w") as f:
            f.write(opt_mix_qasm())
        run_opttpo("optmix2x3", qp, [1e-8], lattice=(3, 2))
        run_opttpo("kobe", os.path.join(a.ref, "apps", "estimator", "kicked_ising.qasm"), [1e-8], full=False)
        orng = np.random.default_rng(20261204)
        q = zz_cx_qasm(3, 3, 3, -math.pi / 4, 0.7)
        run_opt_estimator("optzz3x3", q, random_paulis(9, lattice_edges(3), 30, orng), 4, 1e-8, 1e-10, 50, 1e-8)
    if "tpocount" in jobs:
        q = kicked_ising_no_barrier(3, 3, 2, -0.6, 0.7)  # 2 x (12 rzz + 9 rx) = 42 instructions
        run_tpocount("kinb3x3", q, [[21, 21], [10, 15, 17], [5, 30, 40], [42]])
        crng = np.random.default_rng(20261206)
        run_count_estimator("kinb3x3", q, random_paulis(9, lattice_edges(3), 30, crng), 4, 1e-8, 1e-10, 50,
                            [10, 15, 17])
    if "ckpt" in jobs:
        crng = np.random.default_rng(20261205)
        q = kicked_ising_qasm(3, 3, 3, -0.8, 0.6)
        run_checkpoint("ki3x3r", q, random_paulis(9, lattice_edges(3), 30, crng), 4, 1e-8, 1e-10, 50, 3)
    if "config1" in jobs:
        run_config1()


def lattice_edges_rect(Lx, Ly):
    e = []
    for iy in range(Ly):
        for ix in range(Lx):
            s = ix + Lx * iy
            if ix + 1 < Lx:
                e.append((s, s + 1))
            if iy + 1 < Ly:
                e.append((s, s + Lx))
    return e


if __name__ == "__main__":
    main()
