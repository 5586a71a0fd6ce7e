"""Reader for the golden-vector dumps written by oracle/ref/ref_harness.cpp.

Test infrastructure only (the oracle side): it turns the sectioned binary dump of one
reference CCD solve into a dict of numpy arrays.  Section layout: u32 name length, name,
u32 dtype code (1 = f64, 2 = u64, 3 = i64), u64 element count, raw little-endian data.
"""
import struct

import numpy as np

_DTYPES = {1: np.float64, 2: np.uint64, 3: np.int64}


def read_dump(path):
    out = {}
    with open(path, "rb") as f:
        data = f.read()
    pos = 0
    while pos < len(data):
        (nlen,) = struct.unpack_from("<I", data, pos)
        pos += 4
        name = data[pos:pos + nlen].decode()
        pos += nlen
        dtype_code, count = struct.unpack_from("<IQ", data, pos)
        pos += 12
        dt = np.dtype(_DTYPES[dtype_code])
        nbytes = count * dt.itemsize
        out[name] = np.frombuffer(data, dtype=dt, count=count, offset=pos).copy()
        pos += nbytes
    return out
