"""Reader for the record files written by oracle/ref_probe.cc.

Record: u32 name_len, name, u32 rank, i32 shape[rank], u64 n, n complex128.
Arrays are returned in the reference's column-major order reshaped with
order="F", so a[i0, i1, ...] is the element at coordinates (i0, i1, ...).
"""
import struct

import numpy as np


def read_records(path):
    out = {}
    with open(path, "rb") as f:
        buf = f.read()
    o = 0
    while o < len(buf):
        (nl,) = struct.unpack_from("<I", buf, o)
        o += 4
        name = buf[o:o + nl].decode()
        o += nl
        (rank,) = struct.unpack_from("<I", buf, o)
        o += 4
        shape = struct.unpack_from("<%di" % rank, buf, o)
        o += 4 * rank
        (n,) = struct.unpack_from("<Q", buf, o)
        o += 8
        a = np.frombuffer(buf, dtype=np.complex128, count=n, offset=o).copy()
        o += 16 * n
        out[name] = a.reshape(shape, order="F") if rank else a.reshape(())
    return out


def load_probe(path):
    """Load a probe_*.npz fixture into {name: array} plus its metadata dict."""
    import json
    z = np.load(path, allow_pickle=False)
    meta = json.loads(str(z["__meta__"]))
    return {k: z[k] for k in z.files if k != "__meta__"}, meta
