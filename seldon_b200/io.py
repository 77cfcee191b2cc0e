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
                 from them as ConvertMatrix_from_Coordinates does;
  Harwell-Boeing WriteHarwellBoeing / ReadHarwellBoeing (IOMatrixMarket.cxx):
                 fixed-width text in compressed columns.
"""
import math
import os
import re

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


# `stream >> int` and `stream >> double` as libstdc++ extracts them: skip
# white space, then an int is a sign and digits (within int32), and a double
# takes the longest prefix of sign, digits, point, digits, exponent, which
# must then be a whole finite number (so "nan", "inf", "1e400" and "1e"
# fail).  The first failed extraction ends the reading.
_WS = re.compile(r"\s*")
_INT_PREFIX = re.compile(r"[+-]?[0-9]+")
_FLOAT_PREFIX = re.compile(r"[+-]?[0-9]*(?:\.[0-9]*)?(?:[eE][+-]?[0-9]*)?")
_FLOAT_WHOLE = r"[+-]?(?:[0-9]+\.?[0-9]*|\.[0-9]+)(?:[eE][+-]?[0-9]+)?"
_FLOAT_TOKEN = re.compile(_FLOAT_WHOLE)
# whole files of such tokens take the vectorised path
_INT_FIELDS = re.compile(r"(?:[+-]?[0-9]+ )*[+-]?[0-9]+")
_FLOAT_FIELDS = re.compile(f"(?:{_FLOAT_WHOLE} )*{_FLOAT_WHOLE}")


def _extract_int(text, pos):
    pos = _WS.match(text, pos).end()
    m = _INT_PREFIX.match(text, pos)
    if m is None:
        return None, pos
    v = int(m.group())
    return (v if -2**31 <= v < 2**31 else None), m.end()


def _extract_double(text, pos):
    pos = _WS.match(text, pos).end()
    m = _FLOAT_PREFIX.match(text, pos)
    if not _FLOAT_TOKEN.fullmatch(m.group()):
        return None, pos
    x = float(m.group())
    return (x if math.isfinite(x) else None), m.end()


def read_text(path):
    """ReadCoordinateMatrix (Matrix_Sparse.cxx:1885-1950): 1-based triplets
    (row, col, val) read as `stream >> row >> col >> entry` reads them, up to
    the first extraction that fails.  A row or column below 1 raises
    ValueError (Seldon's IOError), for the first such entry in file order."""
    with open(path) as f:
        text = f.read()
    tok = text.split()
    n3 = len(tok) // 3
    # the common case, whole lines of numbers with integer row and column
    # fields: parsed at once
    r = None
    if tok and len(tok) % 3 == 0 and _INT_FIELDS.fullmatch(
            " ".join(tok[0::3]) + " " + " ".join(tok[1::3])) and _FLOAT_FIELDS.fullmatch(
            " ".join(tok[2::3])):
        try:
            a = np.fromstring(text, dtype=_F8, sep=" ").reshape(-1, 3)
        except ValueError:
            a = None
        if (a is not None and a.shape[0] == n3 and np.all(np.abs(a[:, :2]) < 2**31)
                and np.all(np.isfinite(a[:, 2]))):
            r, c, v = a[:, 0].astype(np.int64), a[:, 1].astype(np.int64), a[:, 2].copy()
    if r is not None:
        bad = (r < 1) | (c < 1)
        if bad.any():
            k = int(np.argmax(bad))
            name, x = ("Row", r[k]) if r[k] < 1 else ("Column", c[k])
            raise ValueError(f"{path}: {name} number should be greater than 0 but is equal "
                             f"to {int(x)}")
        return r.astype(np.int32), c.astype(np.int32), v
    rows, cols, vals = [], [], []
    pos = 0
    while True:
        # `stream >> row >> col >> entry` until an extraction fails
        a, pos = _extract_int(text, pos)
        if a is None:
            break
        b, pos = _extract_int(text, pos)
        if b is None:
            break
        x, pos = _extract_double(text, pos)
        if x is None:
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


# ------------------------------------------------------------------ Harwell-Boeing

def _hb_ptr_layout(n, nnz):
    # WriteHarwellBoeing's field widths and counts (IOMatrixMarket.cxx:415-440)
    ptr_len = int(math.ceil(math.log10(0.1 + nnz + 1))) + 1
    ptr_nperline = min(80 // ptr_len, n + 1)
    ind_len = int(math.ceil(math.log10(0.1 + n + 1))) + 1
    ind_nperline = min(80 // ind_len, nnz)
    return ptr_len, ptr_nperline, ind_len, ind_nperline


def write_harwell_boeing(path, m, n, ptr, ind, val):
    """WriteHarwellBoeing (IOMatrixMarket.cxx:394-511) of a RowSparse matrix:
    the matrix in compressed columns (ConvertToCSC keeps the rows of a column
    in increasing order), fixed-width fields, left-aligned, values as
    %-23.15e three to a line, type RUA (square) or RRA.  nnz must be > 0
    (the reference divides by the count per line, which is 0 otherwise)."""
    ptr = np.asarray(ptr, dtype=np.int64)
    ind = np.asarray(ind, dtype=np.int64)
    val = np.asarray(val, dtype=_F8)
    nnz = ind.size
    if nnz == 0:
        raise ValueError("WriteHarwellBoeing needs at least one entry")
    rows = np.repeat(np.arange(m, dtype=np.int64), np.diff(ptr))
    order = np.argsort(ind, kind="stable")
    rowind, colv = rows[order], val[order]
    colptr = np.zeros(n + 1, dtype=np.int64)
    np.add.at(colptr, ind + 1, 1)
    colptr = np.cumsum(colptr)
    ptr_len, ptr_nper, ind_len, ind_nper = _hb_ptr_layout(n, nnz)
    ptrcrd = n // ptr_nper + 1
    indcrd = (nnz - 1) // ind_nper + 1
    valcrd = (nnz - 1) // 3 + 1
    out = ["%-72s%-8s\n" % ("Seldon", "S0000008"),
           "%-14d%-14d%-14d%-14d%-14d\n" % (ptrcrd + indcrd + valcrd, ptrcrd, indcrd, valcrd, 0),
           "%s           %-14d%-14d%-14d%-14d\n" % ("RUA" if m == n else "RRA", m, n, nnz, 0),
           "%-16s%-16s%-20s%-20s\n" % (f"({ptr_nper}I{ptr_len})", f"({ind_nper}I{ind_len})",
                                      "(3D23.15)", "(3D23.15)")]
    fp, fi = "%%-%dd" % ptr_len, "%%-%dd" % ind_len
    p1 = (colptr + 1).tolist()
    for i in range(0, n + 1, ptr_nper):
        out.append("".join(fp % v for v in p1[i:i + ptr_nper]) + "\n")
    r1 = (rowind + 1).tolist()
    for i in range(0, nnz, ind_nper):
        out.append("".join(fi % v for v in r1[i:i + ind_nper]) + "\n")
    vl = colv.tolist()
    for i in range(0, nnz, 3):
        out.append("".join("%-23.15e" % v for v in vl[i:i + 3]) + "\n")
    with open(path, "w") as f:
        f.write("".join(out))


_LEADING_INT = re.compile(r"\s*[+-]?\d+")
_LEADING_FLOAT = re.compile(r"\s*[+-]?(\d+\.?\d*|\.\d+)([eE][+-]?\d+)?")


def _lead_int(s):
    mt = _LEADING_INT.match(s)
    if not mt:
        raise ValueError(f"no integer in {s!r}")
    return int(mt.group(0))


def _lead_float(s):
    mt = _LEADING_FLOAT.match(s.replace("D", "E").replace("d", "e"))
    if not mt:
        raise ValueError(f"no number in {s!r}")
    return float(mt.group(0))


def read_harwell_boeing(path):
    """ReadHarwellBoeing (IOMatrixMarket.cxx:45-329): a real ('R') or
    pattern ('P') assembled unsymmetric or rectangular matrix, returned as
    Seldon's ColSparse arrays (m, n, colptr, rowind, val), 0-based.  Types
    the reference rejects (complex, Hermitian, skew, symmetric, elemental)
    raise ValueError.  Beyond the reference, Fortran 'D' is read in the value
    format and in the values: the reference rejects its own writer's
    "(3D23.15)" format."""
    with open(path) as f:
        lines = f.read().split("\n")
    if len(lines) < 4:
        raise ValueError(f"{path}: incomplete Harwell-Boeing header")
    head2 = lines[1].split()
    head3 = lines[2].split()
    if len(head2) < 5 or len(head3) < 5:
        raise ValueError(f"{path}: incomplete Harwell-Boeing header")
    nl_ptr, nl_ind, nl_val, nl_rhs = (int(t) for t in head2[1:5])
    typ = head3[0]
    nrow, ncol, nnz, nelt = (int(t) for t in head3[1:5])
    if len(typ) != 3 or typ[0] not in "RCP":
        raise ValueError(f"{path}: type {typ!r} is not a valid type")
    if typ[0] == "C":
        raise ValueError(f"{path}: complex-valued matrices are not supported")
    if typ[1] in "HZS":
        raise ValueError(f"{path}: Hermitian, skew or symmetric matrices are not supported")
    if nelt != 0 or typ[2] == "E":
        raise ValueError(f"{path}: elemental matrices are not supported")
    fmt = lines[3]
    int_fmts = [re.match(r"\s*\((\d+)I(\d+)\)", fmt[a:a + 16]) for a in (0, 16)]
    if None in int_fmts:
        raise ValueError(f"{path}: pointer or index format {fmt[0:32]!r} could not be parsed")
    (lw_ptr, ew_ptr), (lw_ind, ew_ind) = ((int(t) for t in f.groups()) for f in int_fmts)
    lw_val = ew_val = 0
    if typ[0] != "P":
        nums = [int(t) for t in re.split(r"[ (ABDEFGILOPZ*.)]+", fmt[32:48]) if t.isdigit()]
        if len(nums) < 3:
            raise ValueError(f"{path}: value format {fmt[32:48]!r} could not be parsed")
        lw_val, ew_val = nums[-3], nums[-2]
    pos = 4 + (1 if nl_rhs != 0 else 0)

    def fixed(count, nlines, per_line, width, conv):
        nonlocal pos
        out = []
        for _ in range(nlines):
            if pos >= len(lines):
                raise ValueError(f"{path}: fewer lines than the header announces")
            line = lines[pos]
            pos += 1
            for j in range(per_line):
                out.append(conv(line[j * width:(j + 1) * width]))
                if len(out) == count:
                    return out
        if len(out) < count:
            raise ValueError(f"{path}: fewer entries than the header announces")
        return out

    colptr = np.array(fixed(ncol + 1, nl_ptr, lw_ptr, ew_ptr, _lead_int), dtype=np.int32) - 1
    rowind = np.array(fixed(nnz, nl_ind, lw_ind, ew_ind, _lead_int), dtype=np.int32) - 1
    if typ[0] == "P":
        val = np.ones(nnz)
    else:
        val = np.array(fixed(nnz, nl_val, lw_val, ew_val, _lead_float), dtype=_F8)
    return nrow, ncol, colptr, rowind, val
