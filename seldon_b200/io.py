"""Seldon's binary storage formats, read and written on the host.

These are the files Seldon's own Write/Read produce and consume, so a system
saved by a Seldon program loads here and the other way round (checkpoint and
resume, or shared inputs):

  sparse matrix  Matrix_Sparse::Write / Read (Matrix_Sparse.cxx:1531-1556,
                 1650-1680), and Matrix_SymSparse's (Matrix_SymSparse.cxx:
                 1440-1457), which writes the row count where n would be:
                 int32 m, int32 n, int32 nz, int32 ptr[m+1], int32 ind[nz],
                 float64 data[nz], native byte order;
  vector         Vector<VectFull>::Write / Read (Vector.cxx:848-870): an
                 optional int32 length, then float64 values.
"""
import os

import numpy as np

_I4 = np.dtype(np.int32)
_F8 = np.dtype(np.float64)


def write_csr(path, m, n, ptr, ind, val):
    """Write ptr/ind/val (Seldon's ptr_, ind_, data_) in Seldon's format."""
    ptr = np.ascontiguousarray(ptr, dtype=_I4)
    ind = np.ascontiguousarray(ind, dtype=_I4)
    val = np.ascontiguousarray(val, dtype=_F8)
    if ptr.size != m + 1 or ind.size != val.size:
        raise ValueError("WrongDim: ptr must hold m+1 entries and ind/val nz entries")
    with open(path, "wb") as f:
        np.array([m, n, ind.size], dtype=_I4).tofile(f)
        ptr.tofile(f)
        ind.tofile(f)
        val.tofile(f)


def read_csr(path):
    """Read a file in Seldon's sparse format: (m, n, ptr, ind, val)."""
    size = os.path.getsize(path)
    with open(path, "rb") as f:
        head = np.fromfile(f, dtype=_I4, count=3)
        if head.size != 3:
            raise ValueError(f"{path}: not a Seldon sparse matrix (short header)")
        m, n, nz = (int(v) for v in head)
        if m < 0 or n < 0 or nz < 0 or size != 12 + 4 * (m + 1) + 12 * nz:
            raise ValueError(f"{path}: sizes m={m} n={n} nz={nz} do not match the file "
                             f"({size} bytes)")
        ptr = np.fromfile(f, dtype=_I4, count=m + 1)
        ind = np.fromfile(f, dtype=_I4, count=nz)
        val = np.fromfile(f, dtype=_F8, count=nz)
    return m, n, ptr, ind, val


def write_vector(path, x, with_size=True):
    """Write a vector in Seldon's format (length first when with_size)."""
    x = np.ascontiguousarray(x, dtype=_F8)
    with open(path, "wb") as f:
        if with_size:
            np.array([x.size], dtype=_I4).tofile(f)
        x.tofile(f)


def read_vector(path, n=None):
    """Read a vector in Seldon's format: the length from the file when `n` is
    None (written with_size), else `n` values with no length."""
    size = os.path.getsize(path)
    with open(path, "rb") as f:
        if n is None:
            head = np.fromfile(f, dtype=_I4, count=1)
            if head.size != 1 or head[0] < 0 or size != 4 + 8 * int(head[0]):
                raise ValueError(f"{path}: not a Seldon vector written with its size")
            n = int(head[0])
        elif size < 8 * n:
            raise ValueError(f"{path}: holds fewer than {n} values")
        return np.fromfile(f, dtype=_F8, count=n)
