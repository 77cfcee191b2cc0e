"""Cg, BiCgStab and Gmres with SOR or ILUT preconditioning as device-resident
chains.

The scalars of the iteration (rho, alpha, beta, the residual, the stop flag)
stay in device memory and the preconditioner's level-scheduled sweeps are
enqueued between the chain's passes, so no iteration waits on the host.
Against the oracle's Cg with the same preconditioner (Cg.cxx:45-116 with
SorPreconditioner, Precond_Ssor.cxx:62-74): same error code, iteration count
within max(2, 5%), solutions to the accuracy the tolerance implies; and
against the host-driven loop of library calls (sb2_krylov_set_pcg(0)).
BiCgStab follows BiCgStab.cxx:43-145: two iterations of the counter per
loop, Finished() on ||r|| and on ||s||.  Gmres follows Gmres.cxx:44-183:
restarts, Seldon's modified Gram-Schmidt, Givens rotations and the
back-solve, the inner test on |s(i+1)| and the outer one on the true
preconditioned residual."""
import time

import numpy as np
import pytest

from seldon_b200 import matgen
from tests.helpers import to_dev, to_host

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def api(cuda):
    from seldon_b200 import api
    return api


def _cg(api, A, b, M, tol=1e-10, max_iter=5000, solver="Cg", restart=None):
    X = to_dev(np.zeros(A.m))
    it = api.Iteration(max_iter, tol)
    it.HideMessages()
    if restart:
        it.SetRestart(restart)
    code = getattr(api, solver)(A, X, to_dev(b), M, it)
    return code, it, to_host(X)


def _both(api, A, b, M, **kw):
    """Device-resident chain, then the host-driven loop; with timings."""
    import torch
    from seldon_b200 import _lib
    L = _lib.load()
    out = []
    for dev in (1, 0):
        old = L.sb2_krylov_set_pcg(dev)
        try:
            _cg(api, A, b, M, **kw)  # warm: plans and recorded sweeps
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            r = _cg(api, A, b, M, **kw)
            torch.cuda.synchronize()
            out.append(r + (time.perf_counter() - t0,))
        finally:
            L.sb2_krylov_set_pcg(old)
    return out


@pytest.mark.parametrize("sym", [False, True])
def test_ssor_cg_poisson64(api, oracle, sym):
    full = matgen.poisson3d(64)  # 262,144 rows: sweeps launch per level (replayed graphs)
    A = matgen.upper(*full) if sym else full
    n = full[0].size - 1
    b = matgen.matvec(*full, np.random.default_rng(64).uniform(-1, 1, n))
    M = api.RowSymSparse(n, *A) if sym else api.RowSparse(n, n, *A)
    S = api.SorPreconditioner()
    S.SetParameterRelaxation(1.5)
    (code, it, x, t_dev), (code_h, it_h, x_h, t_host) = _both(api, M, b, S)
    xo, co, no, _, _ = oracle.solve("cg", *A, b, sym=sym, precond=2, omega=1.5, tol=1e-10,
                                    max_iter=5000)
    assert code == code_h == co == 0
    assert abs(it.GetNumberIteration() - no) <= max(2, no // 20), (it.GetNumberIteration(), no)
    assert abs(it.GetNumberIteration() - it_h.GetNumberIteration()) <= 2
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) < 1e-8
    assert np.linalg.norm(x - x_h) / np.linalg.norm(x_h) < 1e-8
    # the history is Seldon's: one Finished() test per iteration, from 0
    assert [h[0] for h in it.history] == list(range(it.GetNumberIteration() + 1))
    print(f"SSOR-CG 64^3 sym={sym}: {it.GetNumberIteration()} it, device chain {t_dev * 1e3:.1f} ms, "
          f"host-driven {t_host * 1e3:.1f} ms")


def test_ilut_cg_device_chain(api, oracle):
    full = matgen.lap2d(300)  # 90,000 rows
    up = matgen.upper(*full)
    n = up[0].size - 1
    S = api.RowSymSparse(n, *up)
    M = api.IlutPreconditioning()
    M.SetSymmetricAlgorithm()
    M.SetDroppingThreshold(1e-3)
    M.FactorizeMatrix(S)
    b = matgen.matvec(*full, np.random.default_rng(3).uniform(-1, 1, n))
    (code, it, x, _), (code_h, it_h, x_h, _) = _both(api, S, b, M)
    assert code == code_h == 0
    assert abs(it.GetNumberIteration() - it_h.GetNumberIteration()) <= 2
    assert np.linalg.norm(x - x_h) / np.linalg.norm(x_h) < 1e-8
    r = oracle.mltadd(n, n, *full, -1.0, x, 1.0, b)
    assert np.linalg.norm(r) / np.linalg.norm(b) < 1.05e-10


def test_device_chain_edge_cases(api, oracle):
    full = matgen.lap2d(20)
    n = full[0].size - 1
    A = api.RowSparse(n, n, *full)
    S = api.SorPreconditioner()
    code, it, x = _cg(api, A, np.zeros(n), S)
    assert code == 0 and it.GetNumberIteration() == 0 and not x.any()
    b = matgen.matvec(*full, np.random.default_rng(1).uniform(-1, 1, n))
    code, it, x = _cg(api, A, b, S, max_iter=3)
    xo, co, no, _, _ = oracle.solve("cg", *full, b, precond=2, tol=1e-10, max_iter=3)
    assert code == co == -2 and it.GetNumberIteration() == no == 3
    np.testing.assert_allclose(x, xo, rtol=1e-12, atol=1e-14)
    # repeated solves give the same bits (fixed-order reductions)
    _, _, x1 = _cg(api, A, b, S)
    _, _, x2 = _cg(api, A, b, S)
    assert np.array_equal(x1, x2)


# ------------------------------------------------------------------ BiCgStab

@pytest.mark.parametrize("sym", [False, True])
def test_ssor_bicgstab_convdiff(api, oracle, sym):
    full = matgen.convdiff3d(40) if not sym else matgen.poisson3d(40)  # 64,000 rows
    A = matgen.upper(*full) if sym else full
    n = full[0].size - 1
    b = matgen.matvec(*full, np.random.default_rng(40).uniform(-1, 1, n))
    M = api.RowSymSparse(n, *A) if sym else api.RowSparse(n, n, *A)
    S = api.SorPreconditioner()
    S.SetParameterRelaxation(1.2)
    (code, it, x, t_dev), (code_h, it_h, x_h, t_host) = _both(api, M, b, S, solver="BiCgStab")
    xo, co, no, _, _ = oracle.solve("bicgstab", *A, b, sym=sym, precond=2, omega=1.2, tol=1e-10,
                                    max_iter=5000)
    assert code == code_h == co == 0
    assert abs(it.GetNumberIteration() - no) <= max(2, no // 10), (it.GetNumberIteration(), no)
    assert abs(it.GetNumberIteration() - it_h.GetNumberIteration()) <= max(2, no // 10)
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) < 1e-7
    assert np.linalg.norm(x - x_h) / np.linalg.norm(x_h) < 1e-7
    r = oracle.mltadd(n, n, *full, -1.0, x, 1.0, b)
    assert np.linalg.norm(r) / np.linalg.norm(b) < 1.05e-10
    # the history is Seldon's: Finished() on ||r|| and on ||s||, the counter
    # rising by one each time
    hs = [h[0] for h in it.history]
    assert hs == list(range(it.GetNumberIteration() + 1))
    print(f"SSOR-BiCgStab 40^3 sym={sym}: {it.GetNumberIteration()} it, device chain "
          f"{t_dev * 1e3:.1f} ms, host-driven {t_host * 1e3:.1f} ms")


def test_ilut_bicgstab_device_chain(api, oracle):
    ptr, ind, val = matgen.convdiff3d(30)
    n = ptr.size - 1
    S = api.RowSparse(n, n, ptr, ind, val)
    M = api.IlutPreconditioning()
    M.SetDroppingThreshold(1e-2)
    M.FactorizeMatrix(S)
    b = matgen.matvec(ptr, ind, val, np.random.default_rng(5).uniform(-1, 1, n))
    (code, it, x, _), (code_h, it_h, x_h, _) = _both(api, S, b, M, solver="BiCgStab")
    assert code == code_h == 0
    assert abs(it.GetNumberIteration() - it_h.GetNumberIteration()) <= 2
    assert np.linalg.norm(x - x_h) / np.linalg.norm(x_h) < 1e-8
    r = oracle.mltadd(n, n, ptr, ind, val, -1.0, x, 1.0, b)
    assert np.linalg.norm(r) / np.linalg.norm(b) < 1.05e-10


def test_ilut_sym_bicgstab_device_chain(api, oracle):
    full = matgen.lap2d(200)
    up = matgen.upper(*full)
    n = up[0].size - 1
    S = api.RowSymSparse(n, *up)
    M = api.IlutPreconditioning()
    M.SetSymmetricAlgorithm()
    M.SetDroppingThreshold(1e-3)
    M.FactorizeMatrix(S)
    b = matgen.matvec(*full, np.random.default_rng(8).uniform(-1, 1, n))
    (code, it, x, _), (code_h, it_h, x_h, _) = _both(api, S, b, M, solver="BiCgStab")
    assert code == code_h == 0
    assert abs(it.GetNumberIteration() - it_h.GetNumberIteration()) <= 2
    assert np.linalg.norm(x - x_h) / np.linalg.norm(x_h) < 1e-8
    r = oracle.mltadd(n, n, *full, -1.0, x, 1.0, b)
    assert np.linalg.norm(r) / np.linalg.norm(b) < 1.05e-10


def test_bicgstab_device_chain_edge_cases(api, oracle):
    full = matgen.convdiff3d(12)
    n = full[0].size - 1
    A = api.RowSparse(n, n, *full)
    S = api.SorPreconditioner()
    code, it, x = _cg(api, A, np.zeros(n), S, solver="BiCgStab")
    assert code == 0 and it.GetNumberIteration() == 0 and not x.any()
    b = matgen.matvec(*full, np.random.default_rng(2).uniform(-1, 1, n))
    for max_iter in (3, 4):  # stops on ||s|| (odd) and on ||r|| (even)
        code, it, x = _cg(api, A, b, S, solver="BiCgStab", max_iter=max_iter)
        xo, co, no, _, _ = oracle.solve("bicgstab", *full, b, precond=2, tol=1e-10,
                                        max_iter=max_iter)
        assert code == co == -2 and it.GetNumberIteration() == no == max_iter
        np.testing.assert_allclose(x, xo, rtol=1e-10, atol=1e-13)
    _, _, x1 = _cg(api, A, b, S, solver="BiCgStab")
    _, _, x2 = _cg(api, A, b, S, solver="BiCgStab")
    assert np.array_equal(x1, x2)


# ------------------------------------------------------------------ Gmres

@pytest.mark.parametrize("restart", [5, 20])
def test_ssor_gmres_convdiff(api, oracle, restart):
    full = matgen.convdiff3d(40)  # 64,000 rows
    n = full[0].size - 1
    b = matgen.matvec(*full, np.random.default_rng(41).uniform(-1, 1, n))
    M = api.RowSparse(n, n, *full)
    S = api.SorPreconditioner()
    S.SetParameterRelaxation(1.2)
    (code, it, x, t_dev), (code_h, it_h, x_h, t_host) = _both(api, M, b, S, solver="Gmres",
                                                             restart=restart)
    xo, co, no, _, _ = oracle.solve("gmres", *full, b, precond=2, omega=1.2, tol=1e-10,
                                    max_iter=5000, restart=restart)
    assert code == code_h == co == 0
    assert abs(it.GetNumberIteration() - no) <= max(2, no // 20), (it.GetNumberIteration(), no)
    assert abs(it.GetNumberIteration() - it_h.GetNumberIteration()) <= max(2, no // 20)
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) < 1e-7
    assert np.linalg.norm(x - x_h) / np.linalg.norm(x_h) < 1e-7
    # the history: the outer test at 0 and after each cycle, the inner test
    # after every step (the counter repeats where a cycle ends)
    its = [h[0] for h in it.history]
    assert it.history[0] == (0, 1.0) and its == sorted(its) and its[-1] == it.GetNumberIteration()
    assert it.history[-1][1] < 1e-10
    print(f"SSOR-Gmres({restart}) 40^3: {it.GetNumberIteration()} it, device chain "
          f"{t_dev * 1e3:.1f} ms, host-driven {t_host * 1e3:.1f} ms")


def test_ilut_gmres_device_chain(api, oracle):
    ptr, ind, val = matgen.convdiff3d(30)
    n = ptr.size - 1
    S = api.RowSparse(n, n, ptr, ind, val)
    M = api.IlutPreconditioning()
    M.SetDroppingThreshold(1e-2)
    M.FactorizeMatrix(S)
    b = matgen.matvec(ptr, ind, val, np.random.default_rng(6).uniform(-1, 1, n))
    (code, it, x, _), (code_h, it_h, x_h, _) = _both(api, S, b, M, solver="Gmres", restart=10)
    assert code == code_h == 0
    assert abs(it.GetNumberIteration() - it_h.GetNumberIteration()) <= 2
    assert np.linalg.norm(x - x_h) / np.linalg.norm(x_h) < 1e-8
    assert [h[0] for h in it.history] == [h[0] for h in it_h.history] or \
        abs(len(it.history) - len(it_h.history)) <= 2


def test_gmres_device_chain_edge_cases(api, oracle):
    full = matgen.convdiff3d(12)
    n = full[0].size - 1
    A = api.RowSparse(n, n, *full)
    S = api.SorPreconditioner()
    code, it, x = _cg(api, A, np.zeros(n), S, solver="Gmres", restart=10)
    assert code == 0 and it.GetNumberIteration() == 0 and not x.any()
    b = matgen.matvec(*full, np.random.default_rng(3).uniform(-1, 1, n))
    # the iteration limit is tested after a whole cycle, as in the reference
    code, it, x = _cg(api, A, b, S, solver="Gmres", restart=10, max_iter=7)
    xo, co, no, _, _ = oracle.solve("gmres", *full, b, precond=2, tol=1e-10, max_iter=7,
                                    restart=10)
    assert code == co == -2 and it.GetNumberIteration() == no
    np.testing.assert_allclose(x, xo, rtol=1e-10, atol=1e-13)
    # the identity: one step, a lucky breakdown (H(1,0) = 0)
    eye = (np.arange(n + 1, dtype=np.int32), np.arange(n, dtype=np.int32), np.ones(n))
    I = api.RowSparse(n, n, *eye)
    code, it, x = _cg(api, I, b, api.SorPreconditioner(), solver="Gmres", restart=10)
    xo, co, no, _, _ = oracle.solve("gmres", *eye, b, precond=2, tol=1e-10, max_iter=5000,
                                    restart=10)
    assert code == co == 0 and it.GetNumberIteration() == no
    np.testing.assert_allclose(x, b, rtol=1e-14)
    _, _, x1 = _cg(api, A, b, S, solver="Gmres", restart=10)
    _, _, x2 = _cg(api, A, b, S, solver="Gmres", restart=10)
    assert np.array_equal(x1, x2)
