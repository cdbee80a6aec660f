"""Cartesian Binary Data files (the reference's CBD module, src/fileio.jl:1-114).

Layout, all little-endian: an 8-byte identifier (bytes 0-1 the magic number
0xCB 0xDF, byte 2 the format version 1, byte 7 the bytes per value, 8 or 4),
the grid size (3 x uint64), xmin and xmax (3 x float64 each), the x1, x2 and x3
coordinates (float64), then the values (float64 or float32) with x1 fastest,
then x2, then x3.
"""

import os

import numpy as np

MAGIC = bytes.fromhex("CBDF")
VERSION = 1


def writecbd(dtype, filename, field, x1, x2, x3, xmin, xmax):
    """``writecbd(T, filename, field, x1, x2, x3, xmin, xmax)`` (src/fileio.jl:26-62).

    ``field`` is indexed [x3][x2][x1] (C order), i.e. the reference's column-major
    (x1, x2, x3) array."""
    dtype = np.dtype(dtype)
    if dtype not in (np.dtype(np.float64), np.dtype(np.float32)):
        raise ValueError("Only 64-bit and 32-bit precision is supported.")
    field = np.asarray(field)
    n3, n2, n1 = field.shape
    if len(x1) != n1:
        raise ValueError("Length of x1-values incompatible with dimensions of field.")
    if len(x2) != n2:
        raise ValueError("Length of x2-values incompatible with dimensions of field.")
    if len(x3) != n3:
        raise ValueError("Length of x3-values incompatible with dimensions of field.")
    ident = bytearray(8)
    ident[0:2] = MAGIC
    ident[2] = VERSION
    ident[7] = dtype.itemsize
    d = os.path.dirname(filename)
    if d:
        os.makedirs(d, exist_ok=True)
    with open(filename, "wb") as f:
        f.write(bytes(ident))
        f.write(np.array([n1, n2, n3], dtype="<u8").tobytes())
        f.write(np.asarray(xmin, dtype="<f8").tobytes())
        f.write(np.asarray(xmax, dtype="<f8").tobytes())
        f.write(np.asarray(x1, dtype="<f8").tobytes())
        f.write(np.asarray(x2, dtype="<f8").tobytes())
        f.write(np.asarray(x3, dtype="<f8").tobytes())
        f.write(np.ascontiguousarray(field, dtype=dtype.newbyteorder("<")).tobytes())


def readcbd(filename, x3range=(-np.inf, np.inf), tol=1e-9):
    """``readcbd(filename, x3range)`` (src/fileio.jl:64-108): returns
    (xmin, xmax, x1, x2, x3, data) with data indexed [x3][x2][x1], restricted to the
    layers inside ``x3range`` (widened by ``tol``)."""
    with open(filename, "rb") as f:
        ident = f.read(8)
        if ident[0:2] != MAGIC:
            raise ValueError("Not a CBD file (magic number not matching).")
        if ident[2] != VERSION:
            raise ValueError("Unsupported version of CBD format.")
        if ident[7] == 4:
            dtype = np.dtype("<f4")
        elif ident[7] == 8:
            dtype = np.dtype("<f8")
        else:
            raise ValueError("Unsupported data type: Only 32-bit and 64-bit precision is supported.")
        n1, n2, n3 = (int(v) for v in np.frombuffer(f.read(24), dtype="<u8"))
        xmin = tuple(np.frombuffer(f.read(24), dtype="<f8"))
        xmax = tuple(np.frombuffer(f.read(24), dtype="<f8"))
        x1 = np.frombuffer(f.read(8 * n1), dtype="<f8").copy()
        x2 = np.frombuffer(f.read(8 * n2), dtype="<f8").copy()
        x3 = np.frombuffer(f.read(8 * n3), dtype="<f8").copy()
        x3range = list(x3range)
        if len(x3range) == 0:
            i3min, i3max = 0, -1
        else:
            lo = max(x3[0], min(x3range))
            hi = min(x3[-1], max(x3range))
            i3min = max(i for i in range(n3) if x3[i] < lo + tol)
            i3max = min(i for i in range(n3) if x3[i] > hi - tol)
        count = max(0, i3max - i3min + 1)
        f.seek(n1 * n2 * i3min * dtype.itemsize, 1)
        data = np.frombuffer(f.read(n1 * n2 * count * dtype.itemsize), dtype=dtype).reshape(count, n2, n1)
    return xmin, xmax, x1, x2, x3[i3min:i3min + count], data.astype(dtype.newbyteorder("="))
