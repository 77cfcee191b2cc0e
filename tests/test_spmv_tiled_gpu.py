"""The x-tiled product of long rows (tiled.cu): rows longer than the
threshold are summed by one thread each, tile after tile of x staged in
shared memory, in stored order -- so with sorted columns they equal the
reference's MltAdd bit for bit; rows of up to 32 entries keep the slice
kernel (bit for bit too) and the rows in between the warp kernel (within the
1e-12 FP64 bound)."""
import numpy as np
import pytest

from seldon_b200 import matgen
from tests.helpers import abs_matvec, assert_spmv_close, to_dev, to_host

pytestmark = pytest.mark.gpu


@pytest.fixture
def tiling(cuda):
    """Tiling from rows of 64 entries on and for any entry count, restored
    afterwards (the setting applies to operators multiplied later)."""
    from seldon_b200 import _lib
    L = _lib.load()
    assert L.sb2_spmv_set_tiling(64, 0) == 0
    yield L
    assert L.sb2_spmv_set_tiling(128, 1 << 20) == 0


def _check(oracle, ptr, ind, val, m, n, y, alpha, x, beta, y0, exact_rows):
    ref = oracle.mltadd(m, n, ptr, ind, val, alpha, x, beta, y0)
    assert np.array_equal(y[exact_rows], ref[exact_rows])
    scale = abs(alpha) * abs_matvec(ptr, ind, val, x) + np.abs(beta * y0)
    assert_spmv_close(y, ref, scale)


@pytest.mark.parametrize("seed", [3, 4])
def test_tiled_zipf_bit_exact(tiling, oracle, seed):
    from seldon_b200 import api
    ptr, ind, val = matgen.zipf_csr(40000, seed=seed)  # x spans 4 tiles
    n = ptr.size - 1
    lens = np.diff(ptr)
    assert (lens > 64).sum() > 1000
    exact = (lens <= 32) | (lens > 64)
    rng = np.random.default_rng(seed)
    x, y0 = rng.standard_normal(n), rng.standard_normal(n)
    A = api.RowSparse(n, n, ptr, ind, val)
    for alpha, beta in ((1.0, 0.0), (-1.25, 0.5)):
        Y = to_dev(y0)
        api.MltAdd(alpha, A, to_dev(x), beta, Y)
        _check(oracle, ptr, ind, val, n, n, to_host(Y), alpha, x, beta, y0, exact)
    Y = to_dev(np.full(n, np.nan))  # Mlt overwrites
    api.Mlt(A, to_dev(x), Y)
    _check(oracle, ptr, ind, val, n, n, to_host(Y), 1.0, x, 0.0, np.zeros(n), exact)


def test_tiled_unsorted_rectangular_and_trans(tiling, oracle):
    """Unsorted columns (each tile's entries still in stored order): within
    the bound; a rectangular operator; the transposed product through the
    explicit transpose's own tiled layout."""
    from seldon_b200 import api
    rng = np.random.default_rng(7)
    m, n = 3000, 50000
    lens = rng.integers(1, 400, m)
    ptr = np.zeros(m + 1, dtype=np.int64)
    np.cumsum(lens, out=ptr[1:])
    ind = np.concatenate([rng.choice(n, l, replace=False) for l in lens]).astype(np.int32)
    val = rng.standard_normal(ind.size)
    ptr = ptr.astype(np.int32)
    A = api.RowSparse(m, n, ptr, ind, val)
    x, y0 = rng.standard_normal(n), rng.standard_normal(m)
    Y = to_dev(y0)
    api.MltAdd(0.75, A, to_dev(x), -2.0, Y)
    ref = oracle.mltadd(m, n, ptr, ind, val, 0.75, x, -2.0, y0)
    assert_spmv_close(to_host(Y), ref, 0.75 * abs_matvec(ptr, ind, val, x) + np.abs(2.0 * y0))
    xt, yt = rng.standard_normal(m), rng.standard_normal(n)
    Yt = to_dev(yt)
    api.MltAdd(1.5, A, to_dev(xt), 0.25, Yt, trans=api.SeldonTrans)
    ref = oracle.mltadd(m, n, ptr, ind, val, 1.5, xt, 0.25, yt, trans=True)
    assert np.allclose(to_host(Yt), ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())


def test_tiled_misaligned_x_takes_the_binned_product(tiling, oracle):
    import torch
    from seldon_b200 import api
    ptr, ind, val = matgen.zipf_csr(30000, seed=9)
    n = ptr.size - 1
    x = np.random.default_rng(2).standard_normal(n)
    A = api.RowSparse(n, n, ptr, ind, val)
    buf = torch.zeros(n + 1, dtype=torch.float64, device="cuda")
    buf[1:] = torch.as_tensor(x)
    Y = to_dev(np.zeros(n))
    api.Mlt(A, buf[1:], Y)  # 8-byte aligned only: no bulk copies of x
    ref = oracle.mltadd(n, n, ptr, ind, val, 1.0, x, 0.0, np.zeros(n))
    assert_spmv_close(to_host(Y), ref, abs_matvec(ptr, ind, val, x))
    Y2 = to_dev(np.zeros(n))
    api.Mlt(A, to_dev(x), Y2)  # aligned: the tiled product
    assert_spmv_close(to_host(Y2), ref, abs_matvec(ptr, ind, val, x))


def test_tiling_setter(cuda):
    from seldon_b200 import _lib
    L = _lib.load()
    assert L.sb2_spmv_set_tiling(16, 0) == _lib.SB2_ERR_INVALID_VALUE
    assert L.sb2_spmv_set_tiling(2048, 0) == _lib.SB2_ERR_INVALID_VALUE
    assert L.sb2_spmv_set_tiling(128, -1) == _lib.SB2_ERR_INVALID_VALUE
    assert L.sb2_spmv_set_tiling(128, 1 << 20) == 0
