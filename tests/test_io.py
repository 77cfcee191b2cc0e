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
