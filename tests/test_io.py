"""Seldon's binary formats (seldon_b200/io.py) against the reference's own
Write/Read: files written here load in Seldon and the other way round, and
both sides write the same bytes."""
import numpy as np
import pytest

from seldon_b200 import io, matgen


def _cases():
    g = matgen.lap2d(9)
    rr = matgen.random_csr(40, 23, 0.2, seed=4, empty_rows=0.2)
    return {"general": (81, 81, *g, False), "symmetric": (81, 81, *matgen.upper(*g), True),
            "rect_empty_rows": (40, 23, *rr, False)}


@pytest.mark.parametrize("name", list(_cases()))
def test_csr_same_bytes_both_ways(reference, tmp_path, name):
    m, n, ptr, ind, val, sym = _cases()[name]
    ours, theirs = tmp_path / "ours.bin", tmp_path / "theirs.bin"
    io.write_csr(ours, m, n, ptr, ind, val)
    reference.write_csr(theirs, m, n, ptr, ind, val, sym=sym)
    assert ours.read_bytes() == theirs.read_bytes()
    # Seldon reads ours, we read Seldon's
    m2, n2, p2, i2, v2 = reference.read_csr(ours, sym=sym)
    m3, n3, p3, i3, v3 = io.read_csr(theirs)
    for mm, nn, pp, ii, vv in ((m2, n2, p2, i2, v2), (m3, n3, p3, i3, v3)):
        assert (mm, nn) == (m, n)
        assert np.array_equal(pp, ptr) and np.array_equal(ii, ind) and np.array_equal(vv, val)


@pytest.mark.parametrize("with_size", [True, False])
def test_vector_same_bytes(reference, tmp_path, with_size):
    x = np.random.default_rng(3).standard_normal(37)
    ours, theirs = tmp_path / "ours.bin", tmp_path / "theirs.bin"
    io.write_vector(ours, x, with_size=with_size)
    reference.write_vector(theirs, x, with_size=with_size)
    assert ours.read_bytes() == theirs.read_bytes()
    y = io.read_vector(theirs) if with_size else io.read_vector(theirs, n=37)
    assert np.array_equal(x, y)


def test_damaged_files_are_rejected(tmp_path):
    m, n, ptr, ind, val, _ = _cases()["general"]
    f = tmp_path / "a.bin"
    io.write_csr(f, m, n, ptr, ind, val)
    raw = f.read_bytes()
    (tmp_path / "short.bin").write_bytes(raw[:-8])
    with pytest.raises(ValueError):
        io.read_csr(tmp_path / "short.bin")
    (tmp_path / "head.bin").write_bytes(raw[:6])
    with pytest.raises(ValueError):
        io.read_csr(tmp_path / "head.bin")
    with pytest.raises(ValueError):
        io.write_csr(f, m, n, ptr[:-1], ind, val)
    v = tmp_path / "v.bin"
    io.write_vector(v, np.ones(5))
    (tmp_path / "vs.bin").write_bytes(v.read_bytes()[:-1])
    with pytest.raises(ValueError):
        io.read_vector(tmp_path / "vs.bin")


@pytest.mark.parametrize("name", list(_cases()))
def test_text_same_bytes_and_read_back(reference, oracle, tmp_path, name):
    """WriteText gives Seldon's bytes; ReadText's triplets assembled as
    ConvertMatrix_from_Coordinates does give the matrix Seldon reads."""
    m, n, ptr, ind, val, sym = _cases()[name]
    ours, theirs = tmp_path / "ours.txt", tmp_path / "theirs.txt"
    io.write_text(ours, ptr, ind, val, sym=sym)
    reference.write_text(theirs, m, n, ptr, ind, val, sym=sym)
    assert ours.read_bytes() == theirs.read_bytes()
    r, c, v = io.read_text(theirs)
    got = oracle.coo_to_csr(r, c, v, 1, 0, 0, sym)
    want = reference.read_text(theirs, sym=sym)
    assert got[:2] == want[:2]
    for a, b in zip(got[2:], want[2:]):
        assert np.array_equal(a, b)


def test_text_values_printed_like_ostream(reference, tmp_path):
    ptr = np.array([0, 4], dtype=np.int32)
    ind = np.array([0, 1, 2, 3], dtype=np.int32)
    val = np.array([1.0 / 3.0, -2.5e-300, 123456789012345.0, 0.1])
    ours, theirs = tmp_path / "ours.txt", tmp_path / "theirs.txt"
    io.write_text(ours, ptr, ind, val)
    reference.write_text(theirs, 1, 4, ptr, ind, val)
    assert ours.read_bytes() == theirs.read_bytes()


def test_text_read_stops_and_rejects(tmp_path):
    p = tmp_path / "t.txt"
    p.write_text("1 1 2.0\n2 3 -1\nnot a number\n4 4 4\n")
    r, c, v = io.read_text(p)
    assert r.tolist() == [1, 2] and c.tolist() == [1, 3] and v.tolist() == [2.0, -1.0]
    p.write_text("1 1 2.0\n0 3 -1\n")
    with pytest.raises(ValueError):
        io.read_text(p)


# ------------------------------------------------------------------ Harwell-Boeing

@pytest.mark.parametrize("name", ["general", "rect_empty_rows"])
def test_harwell_boeing_write_same_bytes(reference, tmp_path, name):
    m, n, ptr, ind, val, _ = _cases()[name]
    ours, theirs = tmp_path / "ours.rua", tmp_path / "theirs.rua"
    io.write_harwell_boeing(ours, m, n, ptr, ind, val)
    reference.write_hb(theirs, m, n, ptr, ind, val)
    assert ours.read_bytes() == theirs.read_bytes()


def _hb_case(seed, m, n):
    import scipy.sparse as sp
    rng = np.random.default_rng(seed)
    A = sp.random(m, n, density=0.08, random_state=seed, format="csc")
    A.data = rng.standard_normal(A.nnz) * 10.0 ** rng.integers(-30, 30, A.nnz)
    A.sort_indices()
    return A.indptr.astype(np.int32), A.indices.astype(np.int32), A.data


@pytest.mark.parametrize("typ,m,n", [("RUA", 60, 60), ("RRA", 45, 70), ("PUA", 50, 50)])
def test_harwell_boeing_read_like_seldon(reference, tmp_path, typ, m, n):
    """Files in the collection's layout (fields of width 6 with a blank, E
    format for values): the arrays Seldon reads, bit for bit."""
    colptr, rowind, val = _hb_case(m + n, m, n)
    path = tmp_path / "a.hb"
    _write_collection_hb(path, typ, m, n, colptr, rowind, val)
    ours = io.read_harwell_boeing(path)
    theirs = reference.read_hb(path)
    assert ours[:2] == theirs[:2] == (m, n)
    for a, b in zip(ours[2:], theirs[2:]):
        assert np.array_equal(a, b)


def _write_collection_hb(path, typ, m, n, colptr, rowind, val):
    nnz = rowind.size
    ptr_lines = ["".join("%6d" % (v + 1) for v in colptr[i:i + 10]) for i in range(0, n + 1, 10)]
    ind_lines = ["".join("%6d" % (v + 1) for v in rowind[i:i + 10]) for i in range(0, nnz, 10)]
    val_lines = [] if typ[0] == "P" else [
        "".join("%20.12E" % v for v in val[i:i + 4]) for i in range(0, nnz, 4)]
    with open(path, "w") as f:
        f.write("%-72s%-8s\n" % ("test matrix", "TEST"))
        tot = len(ptr_lines) + len(ind_lines) + len(val_lines)
        f.write("%14d%14d%14d%14d%14d\n" % (tot, len(ptr_lines), len(ind_lines),
                                             len(val_lines), 0))
        f.write("%-14s%14d%14d%14d%14d\n" % (typ, m, n, nnz, 0))
        f.write("%-16s%-16s%-20s\n" % ("(10I6)", "(10I6)",
                                       "(4E20.12)" if typ[0] != "P" else ""))
        f.write("".join(ln + "\n" for ln in ptr_lines + ind_lines + val_lines))


@pytest.mark.parametrize("typ", ["RSA", "CUA", "RUE"])
def test_harwell_boeing_rejects_like_seldon(reference, tmp_path, typ):
    colptr, rowind, val = _hb_case(3, 20, 20)
    path = tmp_path / "a.hb"
    _write_collection_hb(path, typ, 20, 20, colptr, rowind, val)
    with pytest.raises(ValueError):
        io.read_harwell_boeing(path)
    with pytest.raises(RuntimeError):
        reference.read_hb(path)


def test_harwell_boeing_reads_own_files(tmp_path):
    """The reference cannot read what its writer produces ("(3D23.15)" is
    not parsed); this reader can, to the 16 digits written."""
    g = matgen.lap2d(9)
    path = tmp_path / "a.rua"
    io.write_harwell_boeing(path, 81, 81, *g)
    m, n, cp, ri, v = io.read_harwell_boeing(path)
    import scipy.sparse as sp
    C = sp.csr_matrix((g[2], g[1], g[0]), shape=(81, 81)).tocsc()
    assert (m, n) == (81, 81)
    assert np.array_equal(cp, C.indptr) and np.array_equal(ri, C.indices)
    assert np.allclose(v, C.data, rtol=1e-15, atol=0)


@pytest.mark.parametrize("text", [
    "1 1 2.0\n2 99999999999 3.0\n3 3 1.0\n",      # an index past int32 ends the data
    "1 1 nan\n2 2 1\n",                              # libstdc++ reads no nan ...
    "1 1 2.5\n2 2 inf\n3 3 1\n",                     # ... nor inf
    "1 1 2.5\n2 2 1e400\n3 3 1\n",                   # an overflowing value fails
    "1 1 2.5\n2 2 1e-400\n3 3 1\n",                  # an underflowing one reads as 0
    "1 1 1_0\n2 2 3\n",                              # the numeric prefix is taken
    "1 2 0x10\n3 3 1\n",
    "1 1 1e\n2 2 2\n",                               # an exponent without digits fails
    "1.5 2 3\n",
    "+1 +2 +.5\n2 1 -2.\n",
    "1 1 5\n2 2\n",                                  # a trailing partial entry
    "",
])
def test_text_read_like_seldon_stream(reference, oracle, tmp_path, text):
    """ReadText on malformed files takes exactly the entries Seldon's
    `stream >> row >> col >> entry` loop takes (the reference itself reads
    the same file), before and after assembly."""
    p = tmp_path / "t.txt"
    p.write_text(text)
    r, c, v = io.read_text(p)
    want = reference.read_text(p)
    if r.size == 0:  # nothing read: ReadText leaves a 0 x 0 matrix
        assert want[:2] == (0, 0) and want[3].size == 0
        return
    got = oracle.coo_to_csr(r, c, v, 1, 0, 0, False)
    assert got[:2] == want[:2]
    for a, b in zip(got[2:], want[2:]):
        assert np.array_equal(a, b)


def test_damaged_text_and_hb_files_raise_value_error_only(tmp_path):
    """Randomly damaged text and Harwell-Boeing files are either read or
    refused with ValueError (Seldon's IOError), never another exception."""
    import random
    p, i, v = matgen.random_csr(30, 25, 0.1, seed=1)
    txt, hb = tmp_path / "a.txt", tmp_path / "a.rua"
    io.write_text(txt, p, i, v)
    io.write_harwell_boeing(hb, 30, 25, p, i, v)
    rnd = random.Random(0)
    for path, reader in ((txt, io.read_text), (hb, io.read_harwell_boeing)):
        base = path.read_bytes()
        bad = tmp_path / ("bad" + path.suffix)
        for _ in range(400):
            b = bytearray(base)
            for _ in range(rnd.randint(1, 6)):
                k = rnd.randrange(len(b))
                op = rnd.random()
                if op < 0.4:
                    b[k] = rnd.choice(b"0123456789 -+.eE\n\tx")
                elif op < 0.7:
                    del b[k:k + rnd.randint(1, 40)]
                else:
                    b[k:k] = rnd.choice([b"999999999", b"-1", b"nan", b"\n\n", b"1e308"])
            bad.write_bytes(bytes(b))
            try:
                reader(bad)
            except ValueError:
                pass
