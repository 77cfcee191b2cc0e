"""Device assembly of CSR arrays from coordinate triplets (sb2_coo_to_csr,
ConvertMatrix_from_Coordinates) against the oracle and the reference's
golden arrays: same sizes, and ptr/ind/val identical bit for bit, which
checks Seldon's stable (row, column) order with duplicates kept."""
import os

import numpy as np
import pytest

from seldon_b200 import matgen

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "seldon_golden.npz")
COO_CASES = ["gen_dup_i1", "gen_min", "sym_both", "sym_i1_min", "empty_gen", "empty_sym"]


def _dev(a, dtype):
    import torch
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device="cuda")


def _assemble(row, col, val, index=0, m_min=0, n_min=0, sym=False):
    import torch
    from seldon_b200 import api
    m, n, p, i, v = api.ConvertMatrix_from_Coordinates(
        _dev(row, torch.int32), _dev(col, torch.int32), _dev(val, torch.float64), index, m_min,
        n_min, sym)
    torch.cuda.synchronize()
    return m, n, p.cpu().numpy(), i.cpu().numpy(), v.cpu().numpy()


def _same(a, b):
    assert a[:2] == b[:2]
    for u, v in zip(a[2:], b[2:]):
        assert u.shape == v.shape
        assert np.array_equal(u, v)


@pytest.mark.parametrize("name", COO_CASES)
def test_coo_golden(cuda, name):
    g = np.load(GOLDEN)
    k = f"coo/{name}"
    got = _assemble(g[k + "/row"], g[k + "/col"], g[k + "/val"], int(g[k + "/index"]),
                    int(g[k + "/m_min"]), int(g[k + "/n_min"]), bool(g[k + "/sym"]))
    _same(got, (int(g[k + "/m"]), int(g[k + "/n"]), g[k + "/ptr"], g[k + "/ind"],
                g[k + "/out"]))


# (nnz, rows, cols): one triplet, partial and exact tiles of 4096, several
# tiles, heavy duplication, and sizes whose packed key needs 64 bits
SIZES = [(1, 1, 1), (255, 7, 5), (4096, 300, 200), (4097, 50, 3000), (100_000, 64, 64),
         (250_000, 120_000, 90_000), (300_000, 2_000_000, 1_500_000)]


@pytest.mark.parametrize("nnz,m,n", SIZES)
@pytest.mark.parametrize("sym", [False, True])
def test_coo_random_vs_oracle(cuda, oracle, nnz, m, n, sym):
    rng = np.random.default_rng(nnz + m)
    if sym:
        n = m
    index = int(nnz % 2)
    row = rng.integers(0, m, nnz) + index
    col = rng.integers(0, n, nnz) + index
    val = rng.standard_normal(nnz)
    m_min, n_min = m // 2, n + 3
    _same(_assemble(row, col, val, index, m_min, n_min, sym),
          oracle.coo_to_csr(row, col, val, index, m_min, n_min, sym))


@pytest.mark.parametrize("order", ["sorted", "reversed", "constant_row"])
def test_coo_orders(cuda, oracle, order):
    rng = np.random.default_rng(5)
    nnz = 20_000
    row = np.sort(rng.integers(0, 3000, nnz))
    col = rng.integers(0, 3000, nnz)
    if order == "reversed":
        row, col = row[::-1].copy(), col[::-1].copy()
    elif order == "constant_row":  # one long row with repeated columns
        row = np.full(nnz, 17)
        col = rng.integers(0, 40, nnz)
    val = rng.standard_normal(nnz)
    for sym in (False, True):
        _same(_assemble(row, col, val, 0, 0, 0, sym), oracle.coo_to_csr(row, col, val, 0, 0, 0, sym))


def test_coo_all_lower_symmetric(cuda, oracle):
    row = np.array([3, 2, 5, 4])
    col = np.array([0, 1, 2, 0])
    val = np.arange(4.0)
    got = _assemble(row, col, val, 0, 0, 0, True)
    _same(got, oracle.coo_to_csr(row, col, val, 0, 0, 0, True))
    assert got[0] == 6 and got[3].size == 0 and not got[2].any()


@pytest.mark.parametrize("row,col,index", [([0, -1], [0, 0], 0), ([1, 1], [1, 0], 1)])
def test_coo_index_below_base_rejected(cuda, row, col, index):
    from seldon_b200._lib import SB2_ERR_INVALID_VALUE, SeldonB200Error
    with pytest.raises(SeldonB200Error) as e:
        _assemble(np.array(row), np.array(col), np.ones(2), index)
    assert e.value.status == SB2_ERR_INVALID_VALUE


def test_coo_full_size_round_trip(cuda):
    """The 128^3 convection-diffusion operator (2.1M rows, 14.6M entries)
    taken apart into triplets, shuffled on the device, and assembled again:
    the original CSR comes back exactly, and the assembled matrix multiplies
    identically."""
    import torch
    from seldon_b200 import api
    ptr, ind, val = matgen.convdiff3d(128)
    m = ptr.size - 1
    rows = np.repeat(np.arange(m, dtype=np.int32), np.diff(ptr))
    perm = torch.randperm(ind.size, device="cuda", generator=torch.Generator("cuda").manual_seed(3))
    r = _dev(rows, torch.int32)[perm].contiguous()
    c = _dev(ind, torch.int32)[perm].contiguous()
    v = _dev(val, torch.float64)[perm].contiguous()
    mm, nn, p2, i2, v2 = api.ConvertMatrix_from_Coordinates(r, c, v, 0, m, m)
    assert (mm, nn) == (m, m)
    assert torch.equal(p2.cpu(), torch.from_numpy(ptr))
    assert torch.equal(i2.cpu(), torch.from_numpy(ind))
    assert torch.equal(v2.cpu(), torch.from_numpy(val))
    A = api.RowSparse(m, m, ptr, ind, val)
    B = api.RowSparse.from_coordinates(r, c, v, 0, m, m)
    x = torch.randn(m, dtype=torch.float64, device="cuda")
    y1 = torch.zeros(m, dtype=torch.float64, device="cuda")
    y2 = torch.zeros_like(y1)
    api.Mlt(A, x, y1)
    api.Mlt(B, x, y2)
    torch.cuda.synchronize()
    assert torch.equal(y1, y2)


def test_symmetric_from_coordinates(cuda, oracle):
    """RowSymSparse built from both triangles' triplets keeps the upper part
    and multiplies like the matrix built from its upper CSR arrays."""
    import torch
    from seldon_b200 import api
    ptr, ind, val = matgen.lap2d(40)
    m = ptr.size - 1
    rows = np.repeat(np.arange(m, dtype=np.int32), np.diff(ptr))
    S = api.RowSymSparse.from_coordinates(_dev(rows, torch.int32), _dev(ind, torch.int32),
                                          _dev(val, torch.float64))
    up = matgen.upper(ptr, ind, val)
    ref = api.RowSymSparse(m, *up)
    for a, b in zip(S.download(), up):
        assert np.array_equal(a, b)
    x = torch.randn(m, dtype=torch.float64, device="cuda")
    y1 = torch.zeros_like(x)
    y2 = torch.zeros_like(x)
    api.Mlt(S, x, y1)
    api.Mlt(ref, x, y2)
    torch.cuda.synchronize()
    assert torch.equal(y1, y2)


@pytest.mark.parametrize("sym", [False, True])
def test_text_files_device(cuda, oracle, tmp_path, sym):
    """ReadText assembles on the device what the oracle assembles from the
    same lines; WriteText of the device matrix gives the same bytes as the
    host arrays written directly."""
    from seldon_b200 import api, io
    ptr, ind, val = matgen.convdiff3d(9)
    if sym:
        ptr, ind, val = matgen.upper(*matgen.lap2d(30))
    m = ptr.size - 1
    f1, f2 = tmp_path / "a.txt", tmp_path / "b.txt"
    io.write_text(f1, ptr, ind, val, sym=sym)
    cls = api.RowSymSparse if sym else api.RowSparse
    A = cls.ReadText(f1)
    r, c, v = io.read_text(f1)
    want = oracle.coo_to_csr(r, c, v, 1, 0, 0, sym)
    assert (A.m, A.n) == want[:2] == (m, m)
    for a, b in zip(A.download(), want[2:]):
        assert np.array_equal(a, b)
    A.WriteText(f2)
    assert f1.read_bytes() == f2.read_bytes()


def test_harwell_boeing_device(cuda, tmp_path):
    """WriteHarwellBoeing of a device matrix is the host writer's file; the
    file read back and assembled on the device has the same pattern and the
    values to the 16 digits the format keeps."""
    from seldon_b200 import api, io
    ptr, ind, val = matgen.random_csr(300, 200, 0.03, seed=9, empty_rows=0.1)
    A = api.RowSparse(300, 200, ptr, ind, val)
    f1, f2 = tmp_path / "a.rra", tmp_path / "b.rra"
    A.WriteHarwellBoeing(f1)
    io.write_harwell_boeing(f2, 300, 200, ptr, ind, val)
    assert f1.read_bytes() == f2.read_bytes()
    B = api.RowSparse.ReadHarwellBoeing(f1)
    p2, i2, v2 = B.download()
    assert (B.m, B.n) == (300, 200)
    assert np.array_equal(p2, ptr) and np.array_equal(i2, ind)
    assert np.allclose(v2, val, rtol=1e-15, atol=0)
