"""Reader/writer of the .sphd array files exchanged with the reference
harness (oracle/ref_harness.cpp). Test infrastructure only."""
import struct

import numpy as np

_DT = {"f": np.float32, "d": np.float64, "i": np.int32, "u": np.uint32}
_CODE = {np.dtype(np.float32): "f", np.dtype(np.float64): "d", np.dtype(np.int32): "i", np.dtype(np.uint32): "u"}


def read(path):
    out = {}
    with open(path, "rb") as f:
        if f.read(8) != b"SPHD0001":
            raise ValueError(f"{path}: not an .sphd file")
        while True:
            head = f.read(4)
            if len(head) < 4:
                break
            (nl,) = struct.unpack("<I", head)
            name = f.read(nl).decode()
            dt = f.read(1).decode()
            (nd,) = struct.unpack("<I", f.read(4))
            shape = struct.unpack("<" + "Q" * nd, f.read(8 * nd))
            dtype = np.dtype(_DT[dt])
            count = int(np.prod(shape)) if nd else 1
            out[name] = np.frombuffer(f.read(count * dtype.itemsize), dtype).reshape(shape).copy()
    return out


def write(path, arrays):
    with open(path, "wb") as f:
        f.write(b"SPHD0001")
        for name, a in arrays.items():
            a = np.ascontiguousarray(a)
            nb = name.encode()
            f.write(struct.pack("<I", len(nb)) + nb + _CODE[a.dtype].encode())
            f.write(struct.pack("<I", a.ndim) + struct.pack("<" + "Q" * a.ndim, *a.shape))
            f.write(a.tobytes())
