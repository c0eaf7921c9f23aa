"""Build libtnbp_b200.so in-tree for sm_100a with nvcc.

Usage: python tnbp_b200/build.py (it does not import the package, which needs
the built library).
Objects are cached under tnbp_b200/_build/ and rebuilt when a source or
header is newer than its object.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libtnbp_b200.so")
APP = os.path.join(HERE, "tnbp_estimator")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
SOURCES = ["engine.cu", "capi.cu", "server.cu", "noalloc.cu", "host_setup.cpp", "qasm_text.cpp", "tps_io.cpp", "trace.cpp"]


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    hs.append(os.path.join(INCLUDE, "tnbp_b200.h"))
    return hs


def _stale(obj, src):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(p) > t for p in [src] + _headers())


def build(verbose=True, jobs=4):
    os.makedirs(BUILD, exist_ok=True)
    objs, procs = [], []
    for s in SOURCES:
        src = os.path.join(CSRC, s)
        if not os.path.exists(src):
            continue
        obj = os.path.join(BUILD, s + ".o")
        objs.append(obj)
        if not _stale(obj, src):
            continue
        if s.endswith(".cu"):
            cmd = [NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                   "--expt-relaxed-constexpr", "-c", src, "-o", obj]
        else:
            cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-I", os.path.join(os.path.dirname(os.path.dirname(NVCC)),
                                                                        "include"), "-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        procs.append((subprocess.Popen(cmd), cmd))
        if len(procs) >= jobs:
            p, c = procs.pop(0)
            if p.wait() != 0:
                raise RuntimeError("compile failed: " + " ".join(c))
    for p, c in procs:
        if p.wait() != 0:
            raise RuntimeError("compile failed: " + " ".join(c))
    if not os.path.exists(LIB) or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        cmd = [NVCC, *ARCH, "-shared", "-Xcompiler", "-fPIC", *objs, "-o", LIB, "-lcudart_static",
               "-lrt", "-lpthread", "-ldl"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd)
    # the estimator app over the C ABI (C++, host only)
    app_src = os.path.join(HERE, "apps", "estimator.cc")
    if os.path.exists(app_src) and (not os.path.exists(APP) or
                                    max(os.path.getmtime(app_src), os.path.getmtime(LIB)) > os.path.getmtime(APP)):
        cmd = ["g++", "-O2", "-std=c++17", "-I", INCLUDE, app_src, "-L", HERE, "-ltnbp_b200",
               "-Wl,-rpath,$ORIGIN", "-o", APP]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd)
    return LIB


DROPIN_DIR = os.path.join(HERE, "apps", "_dropin")
DROPIN_INC = os.path.join(INCLUDE, "tnbp_dropin")
DROPIN_SRC = os.path.join(HERE, "dropin", "device_overloads.cpp")
# (app, C++ standard): the reference's own app sources, compiled unchanged
DROPIN_APPS = (("estimator", "c++17"), ("kicked_ising_lattice", "c++20"))


def build_dropin(ref, verbose=True):
    """Compile tnbp's apps (apps/estimator, apps/kicked_ising_lattice) from
    the reference tree `ref`, unchanged, against this library: the tensor
    backend header include/tnbp_dropin/gqten/gqten.h (first on the include
    path) and the GPU overloads of tnbp's hot-path functions
    (tnbp_b200/dropin/device_overloads.cpp), linked to libtnbp_b200.so.  The
    binaries go to tnbp_b200/apps/_dropin/.  Needs the reference sources,
    which only the build machine has; the binaries travel with the tree."""
    os.makedirs(DROPIN_DIR, exist_ok=True)
    deps = [DROPIN_SRC, LIB, os.path.join(DROPIN_INC, "gqten", "gqten.h"), os.path.join(DROPIN_INC, "mpi.h"),
            os.path.join(INCLUDE, "tnbp_b200.h")]
    for app, std in DROPIN_APPS:
        src = os.path.join(ref, "apps", app, "main.cc")
        out = os.path.join(DROPIN_DIR, app)
        if not os.path.exists(src):
            continue
        if os.path.exists(out) and os.path.getmtime(out) >= max(os.path.getmtime(p) for p in deps + [src]):
            continue
        cmd = ["g++", f"-std={std}", "-O2", "-I", DROPIN_INC, "-I", INCLUDE, "-I",
               os.path.join(ref, "external", "min-tci", "include"), "-I", os.path.join(ref, "include"), src,
               DROPIN_SRC, "-L", HERE, "-ltnbp_b200", "-Wl,-rpath,$ORIGIN/../..", "-o", out]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd)


if __name__ == "__main__":
    build()
    sys.exit(0)
