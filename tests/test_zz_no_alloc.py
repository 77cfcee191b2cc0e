"""sb2_cg_noalloc: the CG entry point for callers that cannot allocate device
memory (their GPU memory is owned by another allocator, or cudaMalloc's
implicit synchronization is not allowed where they run).  It keeps its work
vectors in a fixed array inside the library instead of allocating them, so
its results must equal those of sb2_cg running the same kernel, call after
call, and meet the oracle's Cg.

This file sorts last so that a run stopping at the first failure has run
every other test before it; it also passes on its own in a fresh process."""
import ctypes

import numpy as np
import pytest

from seldon_b200 import matgen

pytestmark = pytest.mark.gpu

MAX_N = 131072  # rows the fixed array holds


def _solve(L, fn, A, b, noalloc):
    import torch
    from seldon_b200._lib import IterParams, IterResult
    n = A.m
    X = torch.zeros(n, dtype=torch.float64, device="cuda")
    B = torch.as_tensor(b).cuda()
    prm = IterParams(1e-10, 5000, 10, 0, 1)
    res = IterResult()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    if noalloc:
        st = fn(A.handle, ctypes.c_void_p(X.data_ptr()), ctypes.c_void_p(B.data_ptr()),
                ctypes.byref(prm), ctypes.byref(res), stream)
    else:
        st = fn(A.handle, None, ctypes.c_void_p(X.data_ptr()), ctypes.c_void_p(B.data_ptr()),
                ctypes.byref(prm), ctypes.byref(res), None, None, 0, stream)
    return st, X.cpu().numpy(), res


def test_cg_noalloc_matches_cg(cuda, oracle):
    """Two calls in a row against sb2_cg on the same kernel (cluster-resident
    form off), bit for bit, and against the oracle's Cg."""
    from seldon_b200 import _lib, api
    L = _lib.load()
    ptr, ind, val = matgen.lap2d(60)
    n = ptr.size - 1
    b = matgen.matvec(ptr, ind, val, np.random.default_rng(5).uniform(-1, 1, n))
    A = api.RowSparse(n, n, ptr, ind, val)
    old = L.sb2_krylov_set_cluster(0)
    try:
        st, x_ref, r_ref = _solve(L, L.sb2_cg, A, b, noalloc=False)
    finally:
        L.sb2_krylov_set_cluster(old)
    assert st == 0 and r_ref.error_code == 0
    xo, co, no, _, _ = oracle.solve("cg", ptr, ind, val, b, tol=1e-10, max_iter=5000)
    for _ in range(2):  # the shared array keeps the last call's contents
        st, x, r = _solve(L, L.sb2_cg_noalloc, A, b, noalloc=True)
        assert st == 0
        assert (r.nb_iter, r.error_code) == (r_ref.nb_iter, r_ref.error_code)
        assert r.last_residual == r_ref.last_residual
        assert np.array_equal(x, x_ref)
        # the oracle sums dots sequentially: same stopping rule, iterates
        # equal to rounding
        assert r.error_code == co == 0 and abs(r.nb_iter - no) <= max(2, no // 20)
        assert np.linalg.norm(x - xo) / np.linalg.norm(xo) < 1e-8


def test_cg_noalloc_rejects_too_large(cuda):
    from seldon_b200 import _lib, api
    L = _lib.load()
    g = 363  # 131769 rows > MAX_N
    ptr, ind, val = matgen.lap2d(g)
    assert ptr.size - 1 > MAX_N
    A = api.RowSparse(ptr.size - 1, ptr.size - 1, ptr, ind, val)
    st, x, _ = _solve(L, L.sb2_cg_noalloc, A, np.ones(ptr.size - 1), noalloc=True)
    assert st == _lib.SB2_ERR_INVALID_VALUE
    assert not x.any()  # nothing ran
