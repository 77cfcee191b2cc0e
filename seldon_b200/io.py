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
                 optional int32 length, then float64 values;
  text           Matrix_Sparse::WriteText / ReadText (Matrix_Sparse.cxx:
                 1568-1616, 1692-1724): one "row column value" line per entry,
                 1-based, values with 14 significant digits.  RowSymSparse
                 writes both triangles ordered by (row, column)
                 (ConvertMatrix_to_Coordinates, Matrix_Conversions.cxx:
                 100-171).  Reading yields triplets; the matrix is assembled
                 from them as ConvertMatrix_from_Coordinates does.
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


def coordinates(ptr, ind, val, sym=False):
    """0-based (row, col, val) in the order Seldon's
    ConvertMatrix_to_Coordinates lists a matrix: stored order for RowSparse;
    for RowSymSparse every stored entry and its mirror, ordered by
    (row, column) with ties kept in listing order."""
    ptr = np.asarray(ptr, dtype=np.int64)
    ind = np.asarray(ind, dtype=np.int64)
    val = np.asarray(val, dtype=_F8)
    rows = np.repeat(np.arange(ptr.size - 1, dtype=np.int64), np.diff(ptr))
    if not sym:
        return rows, ind, val
    off = ind != rows
    # listing order: each stored entry, then its mirror when off the diagonal
    k = np.arange(ind.size)
    slot = 2 * k
    r = np.concatenate([rows, ind[off]])
    c = np.concatenate([ind, rows[off]])
    v = np.concatenate([val, val[off]])
    o = np.concatenate([slot, slot[off] + 1])
    listing = np.argsort(o, kind="stable")
    r, c, v = r[listing], c[listing], v[listing]
    order = np.lexsort((c, r))
    return r[order], c[order], v[order]


def write_text(path, ptr, ind, val, sym=False):
    """Matrix_Sparse::WriteText: "row column value" lines, 1-based, the value
    as an ostream with precision 14 prints it (%.14g)."""
    r, c, v = coordinates(ptr, ind, val, sym)
    with open(path, "w") as f:
        f.write("".join(f"{a + 1} {b + 1} {x:.14g}\n"
                        for a, b, x in zip(r.tolist(), c.tolist(), v.tolist())))


def read_text(path):
    """ReadCoordinateMatrix (Matrix_Sparse.cxx:1885-1950): 1-based triplets
    (row, col, val) up to the first line that does not parse.  A row or
    column below 1 raises ValueError (Seldon's IOError)."""
    with open(path) as f:
        tok = f.read().split()
    rows, cols, vals = [], [], []
    for k in range(0, len(tok) - 2, 3):
        try:
            a, b, x = int(tok[k]), int(tok[k + 1]), float(tok[k + 2])
        except ValueError:
            break
        if a < 1:
            raise ValueError(f"{path}: Row number should be greater than 0 but is equal to {a}")
        if b < 1:
            raise ValueError(f"{path}: Column number should be greater than 0 but is equal "
                             f"to {b}")
        rows.append(a)
        cols.append(b)
        vals.append(x)
    return (np.array(rows, dtype=np.int32), np.array(cols, dtype=np.int32),
            np.array(vals, dtype=_F8))
