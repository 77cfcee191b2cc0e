"""GMRES with classical Gram-Schmidt applied twice (sb2_gmres_cgs2), and the
iterative refinement whose inner solve is GMRES with an FP32 Arnoldi basis
(sb2_ir_solve, solver 1), against the oracle's and the reference's Gmres.

CGS2 orthogonalizes in a different order than the reference's modified
Gram-Schmidt loop, so its iterates agree to rounding, not bit for bit: the
bar is the same error code, iteration counts within max(2, 5%), solutions
that meet the stopping rule and agree to what the tolerance implies.  The
refinement form must reach an FP64 ||b - A x|| / ||b|| below tol (recomputed
by the oracle's MltAdd) within a few percent more Arnoldi steps than FP64
GMRES(m)."""
import numpy as np
import pytest

from seldon_b200 import matgen
from tests.helpers import to_dev, to_host

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def api(cuda):
    from seldon_b200 import api
    return api


def _close_iters(a, b, frac=20):
    return abs(a - b) <= max(2, b // frac)


def _relres(oracle, ptr, ind, val, x, b):
    n = ptr.size - 1
    r = oracle.mltadd(n, n, ptr, ind, val, -1.0, x, 1.0, b)
    return np.linalg.norm(r) / np.linalg.norm(b)


def _system(name):
    if name == "conv7":  # 343 rows: the last lane of the last slice is partial
        p = matgen.convdiff3d(7)
    elif name == "conv16":
        p = matgen.convdiff3d(16)
    elif name == "zipf":  # warp- and CTA-bin rows, sorted (scattered) slices
        p = matgen.zipf_csr(6000, seed=4, hi=1500)
    elif name == "lap":
        p = matgen.lap2d(40)
    else:
        raise KeyError(name)
    ptr, ind, val = p
    n = ptr.size - 1
    b = matgen.matvec(ptr, ind, val, np.random.default_rng(n).uniform(-1, 1, n))
    return ptr, ind, val, b


def _gmres(api, A, b, M, restart, tol=1e-10, max_iter=5000, orth="cgs2", x0=None):
    X = to_dev(np.zeros(A.m) if x0 is None else x0)
    it = api.Iteration(max_iter, tol)
    it.HideMessages()
    it.SetRestart(restart)
    if x0 is not None:
        it.SetInitGuess(False)
    code = api.Gmres(A, X, to_dev(b), M, it, orthogonalization=orth)
    return code, it, to_host(X)


@pytest.mark.parametrize("name", ["conv7", "conv16", "zipf", "lap"])
@pytest.mark.parametrize("restart", [1, 2, 5, 20, 30, 32])
@pytest.mark.parametrize("jacobi", [False, True])
def test_cgs2_matches_oracle(api, oracle, name, restart, jacobi):
    ptr, ind, val, b = _system(name)
    n = ptr.size - 1
    A = api.RowSparse(n, n, ptr, ind, val)
    M = api.JacobiPreconditioner() if jacobi else api.Preconditioner_Base()
    code, it, x = _gmres(api, A, b, M, restart)
    xo, co, no, ho, hio = oracle.solve("gmres", ptr, ind, val, b, precond=int(jacobi), tol=1e-10,
                                       max_iter=5000, restart=restart, hist_cap=20000)
    assert code == co == 0
    assert _close_iters(it.GetNumberIteration(), no), (it.GetNumberIteration(), no)
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) < 1e-8
    # the history is Seldon's: every Finished() test, first the initial one
    its = [h[0] for h in it.history]
    assert it.history[0] == (0, 1.0) and it.history[-1][1] < 1e-10
    assert its == sorted(its) and its[-1] == it.GetNumberIteration()


@pytest.mark.parametrize("g", [32, 48])
def test_cgs2_restart30_jacobi_vs_reference(api, reference, g):
    ptr, ind, val = matgen.convdiff3d(g)
    n = ptr.size - 1
    xs = np.random.default_rng(g).uniform(-1, 1, n)
    b = reference.mltadd(n, n, ptr, ind, val, 1.0, xs, 0.0, np.zeros(n))
    xr, cr, nr = reference.solve("gmres", ptr, ind, val, b, precond=1, tol=1e-10,
                                 max_iter=20000, restart=30)
    A = api.RowSparse(n, n, ptr, ind, val)
    code, it, x = _gmres(api, A, b, api.JacobiPreconditioner(), 30, max_iter=20000)
    assert code == cr == 0
    assert _close_iters(it.GetNumberIteration(), nr), (it.GetNumberIteration(), nr)
    r = reference.mltadd(n, n, ptr, ind, val, -1.0, x, 1.0, b)
    assert np.linalg.norm(r) / np.linalg.norm(b) < 2e-10
    assert np.linalg.norm(x - xr) / np.linalg.norm(xr) < 1e-8


def test_cgs2_deterministic_and_initial_guess(api, oracle):
    ptr, ind, val, b = _system("conv16")
    n = ptr.size - 1
    A = api.RowSparse(n, n, ptr, ind, val)
    J = api.JacobiPreconditioner()
    _, it1, x1 = _gmres(api, A, b, J, 20)
    _, it2, x2 = _gmres(api, A, b, J, 20)
    assert np.array_equal(x1, x2) and it1.history == it2.history
    # a nonzero initial guess: the residual b - A x0 starts the first cycle
    x0 = np.random.default_rng(9).standard_normal(n)
    code, it, x = _gmres(api, A, b, J, 20, x0=x0)
    xo, co, no, _, _ = oracle.solve("gmres", ptr, ind, val, b, x0=x0, precond=1, tol=1e-10,
                                    max_iter=5000, restart=20)
    assert code == co == 0 and _close_iters(it.GetNumberIteration(), no)
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) < 1e-8


def test_cgs2_edge_cases(api, oracle):
    from seldon_b200 import _lib
    ptr, ind, val, b = _system("conv7")
    n = ptr.size - 1
    A = api.RowSparse(n, n, ptr, ind, val)
    # zero right-hand side: Init fails, x untouched is zero, ErrorCode 0
    code, it, x = _gmres(api, A, np.zeros(n), api.Preconditioner_Base(), 10)
    assert code == 0 and it.GetNumberIteration() == 0 and not x.any()
    # iteration limit: -2 after max_iter steps, as Seldon's
    code, it, x = _gmres(api, A, b, api.Preconditioner_Base(), 10, max_iter=7)
    xo, co, no, _, _ = oracle.solve("gmres", ptr, ind, val, b, tol=1e-10, max_iter=7, restart=10)
    assert code == co == -2 and it.GetNumberIteration() == no
    # the identity: one step reaches the solution (h(1,0) = 0, lucky breakdown)
    eye = (np.arange(n + 1, dtype=np.int32), np.arange(n, dtype=np.int32), np.ones(n))
    code, it, x = _gmres(api, api.RowSparse(n, n, *eye), b, api.Preconditioner_Base(), 10)
    assert code == 0 and it.GetNumberIteration() == 1 and np.allclose(x, b, rtol=1e-15)
    # restart above 32 and SOR are not supported by this variant
    with pytest.raises(_lib.SeldonB200Error) as e:
        _gmres(api, A, b, api.Preconditioner_Base(), 33)
    assert e.value.status == _lib.SB2_ERR_NOT_SUPPORTED
    S = api.SorPreconditioner()
    with pytest.raises(_lib.SeldonB200Error) as e:
        _gmres(api, A, b, S, 10)
    assert e.value.status == _lib.SB2_ERR_NOT_SUPPORTED
    with pytest.raises(ValueError):
        _gmres(api, A, b, api.Preconditioner_Base(), 10, orth="cgs")


# ------------------------------------------------------------------ refinement with GMRES

@pytest.mark.parametrize("name", ["conv16", "zipf", "lap"])
@pytest.mark.parametrize("jacobi", [False, True])
def test_ir_gmres_reaches_fp64_tolerance(api, oracle, name, jacobi):
    ptr, ind, val, b = _system(name)
    n = ptr.size - 1
    A = api.RowSparse(n, n, ptr, ind, val)
    M = api.JacobiPreconditioner() if jacobi else None
    X = to_dev(np.zeros(n))
    code, info = api.IterativeRefinement(A, X, to_dev(b), M=M, tol=1e-10, solver="gmres",
                                         restart=20)
    x = to_host(X)
    assert code == 0
    rel = _relres(oracle, ptr, ind, val, x, b)
    assert rel < 1e-10 and abs(rel - info["rel_residual"]) <= 1e-3 * rel
    # the history holds the FP64 residual of every restart, the last below tol
    assert len(info["history"]) == info["outer_iter"] + 1 and info["history"][-1] == info["rel_residual"]
    xo, co, no, _, _ = oracle.solve("gmres", ptr, ind, val, b, precond=int(jacobi), tol=1e-10,
                                    max_iter=5000, restart=20)
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) < 1e-7
    # an FP32 basis costs few extra steps against FP64 GMRES(20)
    assert info["inner_iter"] <= int(1.25 * no) + 4, (info["inner_iter"], no)


def test_ir_gmres_convdiff48_vs_reference(api, reference):
    ptr, ind, val = matgen.convdiff3d(48)
    n = ptr.size - 1
    xs = np.random.default_rng(48).uniform(-1, 1, n)
    b = reference.mltadd(n, n, ptr, ind, val, 1.0, xs, 0.0, np.zeros(n))
    xr, cr, nr = reference.solve("gmres", ptr, ind, val, b, precond=1, tol=1e-10,
                                 max_iter=20000, restart=30)
    A = api.RowSparse(n, n, ptr, ind, val)
    X = to_dev(np.zeros(n))
    code, info = api.IterativeRefinement(A, X, to_dev(b), M=api.JacobiPreconditioner(),
                                         tol=1e-10, solver="gmres", restart=30)
    x = to_host(X)
    r = reference.mltadd(n, n, ptr, ind, val, -1.0, x, 1.0, b)
    assert code == 0 and np.linalg.norm(r) / np.linalg.norm(b) < 1e-10
    assert np.linalg.norm(x - xr) / np.linalg.norm(xr) < 1e-8
    assert info["inner_iter"] <= int(1.25 * nr) + 4, (info["inner_iter"], nr)


def test_ir_gmres_edge_cases(api):
    from seldon_b200 import _lib
    ptr, ind, val, b = _system("conv7")
    n = ptr.size - 1
    A = api.RowSparse(n, n, ptr, ind, val)
    X = to_dev(np.ones(n))
    code, info = api.IterativeRefinement(A, X, to_dev(np.zeros(n)), solver="gmres")
    assert code == 0 and info["init_failed"] and np.all(to_host(X) == 1.0)
    # the exact solution as the initial guess: converged before any cycle
    xs = np.random.default_rng(1).uniform(-1, 1, n)
    bb = matgen.matvec(ptr, ind, val, xs)
    code, info = api.IterativeRefinement(A, to_dev(xs), to_dev(bb), solver="gmres",
                                         init_guess_null=False, tol=1e-10)
    assert code == 0 and info["outer_iter"] == 0 and info["inner_iter"] == 0
    # too few cycles: -2 with the residual reached so far
    code, info = api.IterativeRefinement(A, to_dev(np.zeros(n)), to_dev(b), solver="gmres",
                                         restart=2, max_outer=1, tol=1e-10)
    assert code == -2 and info["outer_iter"] == 1 and info["rel_residual"] > 1e-10
    with pytest.raises(_lib.SeldonB200Error) as e:
        api.IterativeRefinement(A, to_dev(np.zeros(n)), to_dev(b), solver="gmres", restart=40)
    assert e.value.status == _lib.SB2_ERR_NOT_SUPPORTED
