"""Checkpoint files (SaveTPS / LoadTPS, include/tnbp/ptns/function/iotps.h:37-105)
through the engine's host calls tnbp_tps_write / tnbp_tps_read, against a
file the reference's own estimator_restart app saved (tests/golden/
ckpt_ki3x3r000000.dat, made by tests/golden/make_golden.py).  Runs on the CPU
(no device needed); the device-state calls are in test_gpu_checkpoint.py."""
import os
import struct

import numpy as np
import pytest

import bp_numpy as bn

tb = pytest.importorskip("tnbp_b200")
HERE = os.path.dirname(os.path.abspath(__file__))
G = os.path.join(HERE, "golden")
REF_FILE = os.path.join(G, "ckpt_ki3x3r000000.dat")


def _edges():
    return tb.EdgesFromQasm(open(os.path.join(G, "inputs", "ki3x3r.qasm")).read())


def _parse(path):
    """The file read field by field as iotps.h:69-105 reads it, each tensor as
    uint64 order, int32 shape, complex128 scale, complex128 data."""
    b = open(path, "rb").read()
    p = [0]

    def take(fmt):
        v = struct.unpack_from("<" + fmt, b, p[0])
        p[0] += struct.calcsize("<" + fmt)
        return v

    def tensor():
        (r,) = take("Q")
        shape = list(take(f"{r}i"))
        take("2d")
        n = int(np.prod(shape))
        a = np.frombuffer(b, np.complex128, n, p[0])
        p[0] += 16 * n
        return a.reshape(shape, order="F")

    nV, nM, nE = take("3Q")
    V = [tensor() for _ in range(nV)]
    sites = list(take(f"{nV}i"))
    ranks = [take("2i") for _ in range(nM)]
    E = [tensor() for _ in range(2 * nE)]
    eidx = list(take(f"{nE}i"))
    assert p[0] == len(b)
    return V, sites, ranks, E, eidx


def _write_raw(path, V, sites, ranks, E, eidx):
    """SaveTPS (iotps.h:37-67) field by field, for files the engine must reject."""
    with open(path, "wb") as f:
        f.write(struct.pack("<3Q", len(V), len(ranks), len(eidx)))
        for t in list(V):
            f.write(struct.pack("<Q", t.ndim) + struct.pack(f"<{t.ndim}i", *t.shape) + struct.pack("<2d", 1, 0))
            f.write(np.asarray(t, np.complex128).reshape(-1, order="F").tobytes())
        f.write(struct.pack(f"<{len(sites)}i", *sites))
        for k, v in ranks:
            f.write(struct.pack("<2i", k, v))
        for t in list(E):
            f.write(struct.pack("<Q", t.ndim) + struct.pack(f"<{t.ndim}i", *t.shape) + struct.pack("<2d", 1, 0))
            f.write(np.asarray(t, np.complex128).reshape(-1, order="F").tobytes())
        f.write(struct.pack(f"<{len(eidx)}i", *eidx))


def test_reads_the_reference_checkpoint():
    edges = _edges()
    V, E = tb.LoadTPS(REF_FILE, edges)
    rV, sites, ranks, rE, eidx = _parse(REF_FILE)
    assert sites == tb.GetSiteIndexFromBond(edges)
    assert ranks == [(s, 0) for s in sites]
    assert eidx == list(range(len(edges)))
    assert len(V) == len(rV) and len(E) == len(rE) == 2 * len(edges)
    for a, b in zip(V + E, rV + rE):
        assert a.shape == b.shape
        np.testing.assert_array_equal(a, b)
    assert max(max(v.shape[:-1]) for v in V) == 4  # bonds at chi = 4


def test_rewrite_is_byte_identical(tmp_path):
    edges = _edges()
    V, E = tb.LoadTPS(REF_FILE, edges)
    out = tmp_path / "rt.dat"
    tb.SaveTPS(str(out), edges, V, E)
    assert out.read_bytes() == open(REF_FILE, "rb").read()


def test_round_trip_uneven_dims_and_phys(tmp_path):
    """Random state with different bond dims per edge and physical dim 3."""
    rng = np.random.default_rng(5)
    edges = tb.bond_square_lattice(3, 2)
    dims = [1 + (m % 3) for m in range(len(edges))]
    V = []
    for s in bn.sites_of(edges):
        sh = [dims[m] for m in bn.bonds_of(edges, s)] + [3]
        V.append(rng.normal(size=sh) + 1j * rng.normal(size=sh))
    E = [rng.normal(size=(dims[m % len(edges)],) * 2) + 0j for m in range(2 * len(edges))]
    path = str(tmp_path / "u.dat")
    tb.SaveTPS(path, edges, V, E)
    V2, E2 = tb.LoadTPS(path, edges)
    for a, b in zip(V + E, V2 + E2):
        np.testing.assert_array_equal(a, b)
    pV, sites, ranks, pE, eidx = _parse(path)
    for a, b in zip(V + E, pV + pE):
        np.testing.assert_array_equal(a, b)


def test_rejects_files_that_do_not_hold_this_state(tmp_path):
    edges = _edges()
    V, sites, ranks, E, eidx = _parse(REF_FILE)
    raw = open(REF_FILE, "rb").read()
    # truncated
    p = tmp_path / "cut.dat"
    p.write_bytes(raw[:-9])
    with pytest.raises(tb.TnbpError, match="end of file"):
        tb.LoadTPS(str(p), edges)
    # another edge list
    with pytest.raises(tb.TnbpError):
        tb.LoadTPS(REF_FILE, tb.bond_square_lattice(4, 3))
    # one rank's part of a two-rank run: sites 0..3 and the edges touching them
    keep = [m for m, (a, b) in enumerate(edges) if a <= 3 or b <= 3]
    ne = len(edges)
    part = tmp_path / "rank0.dat"
    _write_raw(str(part), V[:4], sites[:4], [(s, 0 if s <= 3 else 1) for s in sites],
               [E[m] for m in keep] + [E[m + ne] for m in keep], keep)
    with pytest.raises(tb.TnbpError, match="rank"):
        tb.LoadTPS(str(part), edges)
    # inconsistent bond dimension between a site tensor and a message
    bad = tmp_path / "bad.dat"
    E2 = list(E)
    E2[0] = np.zeros((3, 3), np.complex128)
    _write_raw(str(bad), V, sites, ranks, E2, eidx)
    with pytest.raises(tb.TnbpError, match="message shape"):
        tb.LoadTPS(str(bad), edges)
    with pytest.raises(tb.TnbpError, match="cannot open"):
        tb.LoadTPS(str(tmp_path / "missing.dat"), edges)
