"""GPU SpMV parity: libseldon_b200 (through the C ABI) against the oracle's
MltAdd restatement on the same seeded inputs.  Bar: FP64 normwise relative
error <= 1e-12 plus a scaled elementwise bound (tests/helpers.py); the
thread-per-row blocks sum in the reference's order and are bit-exact."""
import numpy as np
import pytest

from seldon_b200 import matgen
from tests.helpers import abs_matvec, assert_spmv_close, to_dev, to_host

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def api(cuda):
    from seldon_b200 import api
    return api


CASES = {
    "lap2d_30": lambda: (matgen.lap2d(30), 900, 900),
    "conv_12": lambda: (matgen.convdiff3d(12), 1728, 1728),
    "rand_rect": lambda: (matgen.random_csr(300, 211, 0.05, seed=2, empty_rows=0.3), 300, 211),
    "zipf_20k": lambda: (matgen.zipf_csr(20000, seed=3), 20000, 20000),
}


@pytest.mark.parametrize("case", list(CASES))
@pytest.mark.parametrize("alpha,beta", [(1.0, 0.0), (-1.3, 0.7), (2.5, 1.0)])
def test_mltadd(api, oracle, case, alpha, beta):
    (ptr, ind, val), m, n = CASES[case]()
    rng = np.random.default_rng(11)
    x, y = rng.standard_normal(n), rng.standard_normal(m)
    A = api.RowSparse(m, n, ptr, ind, val)
    X, Y = to_dev(x), to_dev(y)
    api.MltAdd(alpha, A, X, beta, Y)
    ref = oracle.mltadd(m, n, ptr, ind, val, alpha, x, beta, y)
    scale = np.abs(alpha) * abs_matvec(ptr, ind, val, x) + np.abs(beta * y)
    assert_spmv_close(to_host(Y), ref, scale)


@pytest.mark.parametrize("case", list(CASES))
def test_mlt_and_trans(api, oracle, case):
    (ptr, ind, val), m, n = CASES[case]()
    rng = np.random.default_rng(12)
    x = rng.standard_normal(n)
    A = api.RowSparse(m, n, ptr, ind, val)
    Y = to_dev(np.full(m, np.nan))          # Mlt overwrites: a NaN in Y must not survive
    api.Mlt(A, to_dev(x), Y)
    ref = oracle.mltadd(m, n, ptr, ind, val, 1.0, x, 0.0, np.zeros(m))
    assert_spmv_close(to_host(Y), ref, abs_matvec(ptr, ind, val, x))
    xt, yt = rng.standard_normal(m), rng.standard_normal(n)
    Yt = to_dev(yt)
    api.MltAdd(0.8, A, to_dev(xt), -1.5, Yt, trans=api.SeldonTrans)
    ref = oracle.mltadd(m, n, ptr, ind, val, 0.8, xt, -1.5, yt, trans=True)
    tp, ti, tv = _transpose(ptr, ind, val, n)
    scale = 0.8 * abs_matvec(tp, ti, tv, xt) + np.abs(1.5 * yt)
    assert_spmv_close(to_host(Yt), ref, scale)


def _transpose(ptr, ind, val, n):
    rows = np.repeat(np.arange(ptr.size - 1), np.diff(ptr))
    order = np.lexsort((rows, ind))
    tptr = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(np.bincount(ind, minlength=n), out=tptr[1:])
    return tptr, rows[order].astype(np.int32), val[order]


def test_thread_rows_bit_exact(api, oracle):
    # short rows go through the thread-per-row blocks: same order as Seldon
    (ptr, ind, val), m, n = CASES["conv_12"]()
    x = np.random.default_rng(5).standard_normal(n)
    A = api.RowSparse(m, n, ptr, ind, val)
    Y = to_dev(np.zeros(m))
    api.Mlt(A, to_dev(x), Y)
    assert np.array_equal(to_host(Y), oracle.mltadd(m, n, ptr, ind, val, 1.0, x, 0.0, np.zeros(m)))


def test_symmetric(api, oracle):
    ptr, ind, val = matgen.lap2d(40)
    up = matgen.upper(ptr, ind, val)
    m = ptr.size - 1
    rng = np.random.default_rng(3)
    x, y = rng.standard_normal(m), rng.standard_normal(m)
    S = api.RowSymSparse(m, *up)
    assert S.nnz_full == ind.size
    for trans in (0, 1):  # RowSymSparse Trans reduces to NoTrans
        Y = to_dev(y)
        api.MltAdd(1.2, S, to_dev(x), 0.4, Y, trans=trans)
        ref = oracle.mltadd(m, m, *up, 1.2, x, 0.4, y, sym=True)
        assert_spmv_close(to_host(Y), ref, 1.2 * abs_matvec(ptr, ind, val, x) + np.abs(0.4 * y))


def test_edge_cases(api, oracle):
    # beta = 0 keeps a NaN already in Y (Mlt(beta, Y) always multiplies)
    ptr, ind, val = matgen.lap2d(5)
    A = api.RowSparse(25, 25, ptr, ind, val)
    y = np.ones(25)
    y[3] = np.nan
    Y = to_dev(y)
    api.MltAdd(1.0, A, to_dev(np.ones(25)), 0.0, Y)
    out = to_host(Y)
    assert np.isnan(out[3]) and not np.isnan(np.delete(out, 3)).any()
    # alpha = 0 -> Y = beta*Y exactly
    y = np.random.default_rng(0).standard_normal(25)
    Y = to_dev(y)
    api.MltAdd(0.0, A, to_dev(np.ones(25)), 3.0, Y)
    assert np.array_equal(to_host(Y), 3.0 * y)
    # 1x1, single row of 2000 (CTA-per-row), all-empty matrix
    A1 = api.RowSparse(1, 1, np.array([0, 1]), np.array([0]), np.array([2.5]))
    Y = to_dev(np.zeros(1))
    api.Mlt(A1, to_dev(np.array([4.0])), Y)
    assert to_host(Y)[0] == 10.0
    n = 3000
    rng = np.random.default_rng(9)
    cols = np.sort(rng.choice(n, 2000, replace=False)).astype(np.int32)
    v = rng.standard_normal(2000)
    AL = api.RowSparse(1, n, np.array([0, 2000]), cols, v)
    x = rng.standard_normal(n)
    Y = to_dev(np.zeros(1))
    api.Mlt(AL, to_dev(x), Y)
    ref = oracle.mltadd(1, n, np.array([0, 2000]), cols, v, 1.0, x, 0.0, np.zeros(1))
    assert abs(to_host(Y)[0] - ref[0]) <= 1e-12 * np.abs(v * x[cols]).sum()
    E = api.RowSparse(7, 4, np.zeros(8, dtype=np.int32), np.zeros(0), np.zeros(0))
    Y = to_dev(np.full(7, 2.0))
    api.MltAdd(1.0, E, to_dev(np.ones(4)), 0.5, Y)
    assert np.array_equal(to_host(Y), np.full(7, 1.0))


def test_invalid_csr_rejected(api):
    from seldon_b200._lib import SeldonB200Error
    with pytest.raises(SeldonB200Error):
        api.RowSparse(2, 2, np.array([0, 1, 2]), np.array([0, 5]), np.array([1.0, 1.0]))
    with pytest.raises(SeldonB200Error):
        api.RowSymSparse(2, np.array([0, 1, 2]), np.array([0, 0]), np.array([1.0, 1.0]))


def test_host_buffers(cuda, oracle):
    """sb2_spmv_host / sb2_mlt_host: vectors in host memory, copies inside."""
    import ctypes
    from seldon_b200 import _lib
    from seldon_b200 import api
    L = _lib.load()
    (ptr, ind, val), m, n = CASES["conv_12"]()
    A = api.RowSparse(m, n, ptr, ind, val)
    rng = np.random.default_rng(4)
    x, y = rng.standard_normal(n), rng.standard_normal(m)
    yh = y.copy()
    st = L.sb2_spmv_host(A.handle, 0, 0.5, x.ctypes.data_as(ctypes.c_void_p), 2.0,
                         yh.ctypes.data_as(ctypes.c_void_p), None)
    assert st == 0
    ref = oracle.mltadd(m, n, ptr, ind, val, 0.5, x, 2.0, y)
    assert_spmv_close(yh, ref, 0.5 * abs_matvec(ptr, ind, val, x) + 2 * np.abs(y))
    yh = np.full(m, np.nan)
    st = L.sb2_mlt_host(A.handle, 0, 1.0, x.ctypes.data_as(ctypes.c_void_p),
                        yh.ctypes.data_as(ctypes.c_void_p), None)
    assert st == 0
    assert np.array_equal(yh, oracle.mltadd(m, n, ptr, ind, val, 1.0, x, 0.0, np.zeros(m)))


@pytest.mark.parametrize("n", [1, 7, 1000, 123457, 3_000_001])
def test_blas1(api, oracle, n):
    rng = np.random.default_rng(n)
    x, y = rng.standard_normal(n), rng.standard_normal(n)
    X, Y = to_dev(x), to_dev(y)
    d = api.DotProd(X, Y)
    assert abs(d - oracle.dot(x, y)) <= 1e-13 * np.abs(x * y).sum()
    assert api.DotProd(X, Y) == d  # deterministic
    nr = api.Norm2(X)
    # the oracle sums sequentially: its own error grows like n*eps
    assert abs(nr - oracle.nrm2(x)) <= 1e-12 * nr
    api.Add(0.75, X, Y)
    assert np.array_equal(to_host(Y), y + 0.75 * x)
    api.Mlt(-2.0, X)
    assert np.array_equal(to_host(X), -2.0 * x)
    Z = to_dev(np.zeros(n))
    api.Copy(Y, Z)
    assert np.array_equal(to_host(Z), to_host(Y))
    api.Add(0.0, to_dev(np.full(n, np.nan)), Z)  # alpha == 0 is a no-op
    assert not np.isnan(to_host(Z)).any()


@pytest.mark.parametrize("case", ["conv_12", "rand_rect"])
@pytest.mark.parametrize("trans", [0, 1])
@pytest.mark.parametrize("count,pinned", [(1, False), (2, True), (3, False), (5, True)])
def test_mlt_host_batch(api, case, trans, count, pinned):
    # pipelined host-buffer batch: every Y[i] is the same bits as the
    # single-vector product on the device
    import torch
    (ptr, ind, val), m, n = CASES[case]()
    A = api.RowSparse(m, n, ptr, ind, val)
    nx, ny = (m, n) if trans else (n, m)
    rng = np.random.default_rng(31 + count)
    X = rng.standard_normal((count, nx))
    if pinned:
        Xh = torch.from_numpy(X).pin_memory()
        Yh = torch.full((count, ny), np.nan, dtype=torch.float64).pin_memory()
    else:
        Xh, Yh = X, np.full((count, ny), np.nan)
    api.MltHostBatch(A, Xh, Yh, alpha=-0.75, trans=trans)
    Y = Yh.numpy() if pinned else Yh
    for i in range(count):
        Z = to_dev(np.zeros(ny))
        api.Mlt(-0.75, A, to_dev(X[i]), Z, trans=trans)
        assert np.array_equal(Y[i], to_host(Z)), i


@pytest.mark.parametrize("case", list(CASES))
@pytest.mark.parametrize("algo,threads,stages", [(1, 256, 4), (2, 256, 3), (2, 256, 4),
                                                 (2, 512, 3), (2, 512, 4)])
def test_spmv_engines(api, oracle, case, algo, threads, stages):
    # the other product engines sb2_spmv_set_config selects (row-block stream
    # kernel; TMA bulk-copy ring with 256/512 threads and 3/4 stages) against
    # the oracle, MltAdd and the overwriting Mlt
    from seldon_b200 import _lib
    L = _lib.load()
    (ptr, ind, val), m, n = CASES[case]()
    rng = np.random.default_rng(41)
    x, y = rng.standard_normal(n), rng.standard_normal(m)
    A = api.RowSparse(m, n, ptr, ind, val)
    _lib.check(L.sb2_spmv_set_config(algo, threads, stages), "sb2_spmv_set_config")
    try:
        Y = to_dev(y)
        api.MltAdd(-1.3, A, to_dev(x), 0.7, Y)
        Z = to_dev(np.full(m, np.nan))
        api.Mlt(A, to_dev(x), Z)
        import torch
        torch.cuda.synchronize()
    finally:
        _lib.check(L.sb2_spmv_set_config(0, 256, 4), "sb2_spmv_set_config")
    ref = oracle.mltadd(m, n, ptr, ind, val, -1.3, x, 0.7, y)
    assert_spmv_close(to_host(Y), ref, 1.3 * abs_matvec(ptr, ind, val, x) + np.abs(0.7 * y))
    ref0 = oracle.mltadd(m, n, ptr, ind, val, 1.0, x, 0.0, np.zeros(m))
    assert_spmv_close(to_host(Z), ref0, abs_matvec(ptr, ind, val, x))


@pytest.mark.parametrize("sym", [False, True])
def test_write_read_device_matrix(api, tmp_path, sym):
    # a device matrix saved in Seldon's binary format and loaded back gives
    # the same stored arrays and the same products
    ptr, ind, val = matgen.lap2d(20) if not sym else matgen.upper(*matgen.lap2d(20))
    n = ptr.size - 1
    A = api.RowSymSparse(n, ptr, ind, val) if sym else api.RowSparse(n, n, ptr, ind, val)
    path = tmp_path / "A.bin"
    A.Write(path)
    B = (api.RowSymSparse if sym else api.RowSparse).Read(path)
    for a, b in zip(A.download(), B.download()):
        assert np.array_equal(a, b)
    x = np.random.default_rng(2).standard_normal(n)
    Y1, Y2 = to_dev(np.zeros(n)), to_dev(np.zeros(n))
    api.Mlt(A, to_dev(x), Y1)
    api.Mlt(B, to_dev(x), Y2)
    assert np.array_equal(to_host(Y1), to_host(Y2))
