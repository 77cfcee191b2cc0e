"""GPU parity of the preconditioners and Krylov drivers against the oracle.

SOR must be bit-exact (level scheduling reproduces the sequential sweep).
Solvers: same error code, iteration count within a few percent of the
oracle's (reductions are summed in a different order), both solutions meet
the stopping rule, and they agree to the accuracy the tolerance implies."""
import numpy as np
import pytest

from seldon_b200 import matgen
from tests.helpers import to_dev, to_host

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def api(cuda):
    from seldon_b200 import api
    return api


def _mats():
    lp = matgen.lap2d(24)
    up = matgen.upper(*lp)
    cd = matgen.convdiff3d(7)
    return {"lap": lp, "lap_up": up, "conv": cd}


# ------------------------------------------------------------------ SOR

@pytest.mark.parametrize("g", [12, 310])  # single-CTA path and per-level launches
@pytest.mark.parametrize("sym", [False, True])
@pytest.mark.parametrize("t", [0, 2, 3])
def test_sor_bit_exact(api, oracle, g, sym, t):
    full = matgen.lap2d(g) if sym else matgen.convdiff3d(max(4, g // 15))
    A = matgen.upper(*full) if sym else full
    n = A[0].size - 1
    rng = np.random.default_rng(g + t)
    x0, b = rng.standard_normal(n), rng.standard_normal(n)
    M = api.RowSymSparse(n, *A) if sym else api.RowSparse(n, n, *A)
    X = to_dev(x0)
    api.SOR(M, X, to_dev(b), 1.37, 2, t)
    ref = oracle.sor(*A, x0, b, 1.37, 2, t, sym=sym)
    assert np.array_equal(to_host(X), ref)


def test_precond_solve(api, oracle):
    ptr, ind, val = matgen.convdiff3d(6)
    n = ptr.size - 1
    A = api.RowSparse(n, n, ptr, ind, val)
    r = np.random.default_rng(2).standard_normal(n)
    J = api.JacobiPreconditioner()
    Z = to_dev(np.zeros(n))
    J.Solve(A, to_dev(r), Z)
    diag = np.array([val[ptr[i]:ptr[i + 1]][ind[ptr[i]:ptr[i + 1]] == i][0] for i in range(n)])
    assert np.array_equal(to_host(Z), r / diag)
    S = api.SorPreconditioner()
    S.SetParameterRelaxation(1.2)
    S.InitUnSymmetricPreconditioning()
    S.Solve(A, to_dev(r), Z)
    assert np.array_equal(to_host(Z), oracle.sor(ptr, ind, val, np.zeros(n), r, 1.2, 1, 2))
    S.TransSolve(A, to_dev(r), Z)
    assert np.array_equal(to_host(Z), oracle.sor(ptr, ind, val, np.zeros(n), r, 1.2, 1, 3))
    S.InitSymmetricPreconditioning()
    S.Solve(A, to_dev(r), Z)
    assert np.array_equal(to_host(Z), oracle.sor(ptr, ind, val, np.zeros(n), r, 1.2, 1, 0))


# ------------------------------------------------------------------ drivers

def _precond(api, pc):
    if pc == 0:
        return api.Preconditioner_Base()
    if pc == 1:
        return api.JacobiPreconditioner()
    S = api.SorPreconditioner()
    S.SetParameterRelaxation(1.2)
    return S


SOLVER_CASES = [
    ("cg", "lap", 0), ("cg", "lap", 1), ("cg", "lap", 2),
    ("cg", "lap_up", 0), ("cg", "lap_up", 1), ("cg", "lap_up", 2),
    ("bicgstab", "conv", 0), ("bicgstab", "conv", 1), ("bicgstab", "conv", 2),
    ("gmres", "conv", 0), ("gmres", "conv", 1), ("gmres", "conv", 2),
    ("gmres", "lap_up", 1),
]


@pytest.mark.parametrize("which,mname,pc", SOLVER_CASES)
def test_solver_parity(api, oracle, which, mname, pc):
    mats = _mats()
    sym = mname.endswith("_up")
    A = mats[mname]
    full = mats["lap"] if sym else A
    n = A[0].size - 1
    rng = np.random.default_rng(3)
    b = matgen.matvec(*full, rng.uniform(-1, 1, n))
    tol, restart = 1e-10, 8
    xo, co, no, ho, hio = oracle.solve(which, *A, b, sym=sym, precond=pc, omega=1.2, tol=tol,
                                       max_iter=2000, restart=restart, hist_cap=10000)
    M = api.RowSymSparse(n, *A) if sym else api.RowSparse(n, n, *A)
    X = to_dev(np.zeros(n))
    it = api.Iteration(2000, tol)
    it.SetRestart(restart)
    it.HideMessages()
    fn = {"cg": api.Cg, "bicgstab": api.BiCgStab, "gmres": api.Gmres}[which]
    code = fn(M, X, to_dev(b), _precond(api, pc), it)
    x = to_host(X)
    assert code == co == 0
    nb = it.GetNumberIteration()
    assert abs(nb - no) <= max(2, int(0.05 * no)), (nb, no)
    # both meet the rule on the true residual to within the recurrence drift
    for xx in (x, xo):
        r = b - matgen.matvec(*full, xx)
        assert np.linalg.norm(r) / np.linalg.norm(b) < 50 * tol
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) < 1e-7
    # residual history: same length as the oracle's within the iteration slack,
    # same first entry, decreasing to below tol
    h = np.array([r for _, r in it.history])
    assert h[0] == pytest.approx(ho[0], rel=1e-12)
    assert h[-1] < tol


def test_cg_deterministic(api):
    ptr, ind, val = matgen.lap2d(40)
    n = ptr.size - 1
    b = matgen.matvec(ptr, ind, val, np.random.default_rng(1).uniform(-1, 1, n))
    A = api.RowSparse(n, n, ptr, ind, val)
    outs = []
    for _ in range(2):
        X = to_dev(np.zeros(n))
        it = api.Iteration(5000, 1e-10)
        it.HideMessages()
        api.Cg(A, X, to_dev(b), api.Preconditioner_Base(), it)
        outs.append((to_host(X), it.GetNumberIteration()))
    assert outs[0][1] == outs[1][1]
    assert np.array_equal(outs[0][0], outs[1][0])


@pytest.mark.parametrize("which", ["cg", "bicgstab", "gmres"])
def test_zero_rhs_and_max_iter(api, oracle, which):
    ptr, ind, val = matgen.lap2d(6)
    n = 36
    A = api.RowSparse(n, n, ptr, ind, val)
    fn = {"cg": api.Cg, "bicgstab": api.BiCgStab, "gmres": api.Gmres}[which]
    # zero right-hand side.  Cg/BiCgStab test Init(b): it fails, x is left
    # untouched and ErrorCode() is 0.  Gmres tests Init(M^{-1}(b - A x0))
    # (Gmres.cxx:82-93), so with x0 != 0 it solves A x = 0 like the oracle.
    x0 = np.arange(n, dtype=float)
    X = to_dev(x0)
    it = api.Iteration(100, 1e-10)
    it.HideMessages()
    it.SetInitGuess(False)
    assert fn(A, X, to_dev(np.zeros(n)), api.Preconditioner_Base(), it) == 0
    if which == "gmres":
        xo, co, no, _, _ = oracle.solve(which, ptr, ind, val, np.zeros(n), x0=x0, tol=1e-10,
                                        max_iter=100)
        assert co == 0 and abs(it.GetNumberIteration() - no) <= 2
        assert np.abs(to_host(X)).max() < 1e-7 * np.abs(x0).max()
    else:
        assert np.array_equal(to_host(X), x0)
    X = to_dev(x0)
    it.SetInitGuess(True)
    assert fn(A, X, to_dev(np.zeros(n)), api.Preconditioner_Base(), it) == 0
    # null guess: Cg/BiCgStab return from Init(b) before x.Zero() (Cg.cxx:57-67);
    # Gmres zeroes x before Init (Gmres.cxx:82-93)
    assert np.array_equal(to_host(X), np.zeros(n) if which == "gmres" else x0)
    # max_iter reached -> -2 with exactly max_iter iterations (GMRES: a multiple
    # of the restart length may overshoot exactly like the reference)
    b = np.ones(n)
    X = to_dev(np.zeros(n))
    it = api.Iteration(3, 1e-30)
    it.HideMessages()
    it.SetRestart(2)
    code = fn(A, X, to_dev(b), api.Preconditioner_Base(), it)
    _, co, no, _, _ = oracle.solve(which, ptr, ind, val, b, tol=1e-30, max_iter=3, restart=2)
    assert code == co == -2
    assert it.GetNumberIteration() == no


def test_warm_start(api, oracle):
    ptr, ind, val = matgen.lap2d(20)
    n = ptr.size - 1
    rng = np.random.default_rng(8)
    b = rng.standard_normal(n)
    x0 = rng.standard_normal(n)
    A = api.RowSparse(n, n, ptr, ind, val)
    for which, fn in (("cg", api.Cg), ("bicgstab", api.BiCgStab), ("gmres", api.Gmres)):
        X = to_dev(x0)
        it = api.Iteration(1000, 1e-9)
        it.HideMessages()
        it.SetInitGuess(False)
        it.SetRestart(15)
        assert fn(A, X, to_dev(b), api.Preconditioner_Base(), it) == 0
        xo, co, no, _, _ = oracle.solve(which, ptr, ind, val, b, x0=x0, tol=1e-9, max_iter=1000,
                                        restart=15)
        assert abs(it.GetNumberIteration() - no) <= max(2, no // 20)
        assert np.linalg.norm(to_host(X) - xo) / np.linalg.norm(xo) < 1e-6


def test_breakdowns(api, oracle):
    # CG breakdown #2: (p, Ap) == 0 on diag(1, -1)
    A = api.RowSparse(2, 2, np.array([0, 1, 2]), np.array([0, 1]), np.array([1.0, -1.0]))
    it = api.Iteration(10, 1e-12)
    it.HideMessages()
    X = to_dev(np.zeros(2))
    assert api.Cg(A, X, to_dev(np.array([1.0, 1.0])), api.Preconditioner_Base(), it) == 2
    # BiCGSTAB breakdown #3: (rtilde, A p) == 0 for the swap matrix
    P = api.RowSparse(2, 2, np.array([0, 1, 2]), np.array([1, 0]), np.array([1.0, 1.0]))
    it = api.Iteration(10, 1e-12)
    it.HideMessages()
    X = to_dev(np.zeros(2))
    code = api.BiCgStab(P, X, to_dev(np.array([1.0, 0.0])), api.Preconditioner_Base(), it)
    _, co, _, _, _ = oracle.solve("bicgstab", np.array([0, 1, 2]), np.array([1, 0]),
                                  np.array([1.0, 1.0]), np.array([1.0, 0.0]), tol=1e-12,
                                  max_iter=10)
    assert code == co == 3


def test_history_matches_oracle(api, oracle):
    ptr, ind, val = matgen.convdiff3d(6)
    n = ptr.size - 1
    b = np.random.default_rng(4).standard_normal(n)
    A = api.RowSparse(n, n, ptr, ind, val)
    X = to_dev(np.zeros(n))
    it = api.Iteration(500, 1e-10)
    it.HideMessages()
    it.SetRestart(5)
    api.Gmres(A, X, to_dev(b), api.JacobiPreconditioner(), it)
    _, _, _, ho, hio = oracle.solve("gmres", ptr, ind, val, b, precond=1, tol=1e-10, max_iter=500,
                                    restart=5, hist_cap=5000)
    its = [i for i, _ in it.history]
    res = np.array([r for _, r in it.history])
    k = min(len(res), len(ho)) - 2
    assert its[:k] == hio[:k].tolist()
    np.testing.assert_allclose(res[:k], ho[:k], rtol=1e-6)


# ------------------------------------------------------------------ chained CG

@pytest.fixture
def chain_everywhere(api):
    """Run Cg through the kernel chain at every size, then restore."""
    from seldon_b200 import _lib
    L = _lib.load()
    old = L.sb2_krylov_set_config(0)
    yield
    L.sb2_krylov_set_config(old)


@pytest.mark.parametrize("mname,pc", [("lap", 0), ("lap", 1), ("lap_up", 0), ("conv_spd", 1)])
def test_chain_cg_parity(api, oracle, chain_everywhere, mname, pc):
    mats = _mats()
    if mname == "conv_spd":
        A = matgen.poisson3d(14)
    else:
        A = mats[mname]
    sym = mname.endswith("_up")
    full = mats["lap"] if sym else A
    n = A[0].size - 1
    b = matgen.matvec(*full, np.random.default_rng(6).uniform(-1, 1, n))
    xo, co, no, ho, hio = oracle.solve("cg", *A, b, sym=sym, precond=pc, tol=1e-10, max_iter=3000,
                                       hist_cap=4000)
    M = api.RowSymSparse(n, *A) if sym else api.RowSparse(n, n, *A)
    X = to_dev(np.zeros(n))
    it = api.Iteration(3000, 1e-10)
    it.HideMessages()
    code = api.Cg(M, X, to_dev(b), api.JacobiPreconditioner() if pc else api.Preconditioner_Base(), it)
    assert code == co == 0
    assert abs(it.GetNumberIteration() - no) <= max(2, no // 20)
    assert np.linalg.norm(to_host(X) - xo) / np.linalg.norm(xo) < 1e-7
    assert len(it.history) == it.GetNumberIteration() + 1
    assert it.history[0][1] == pytest.approx(ho[0], rel=1e-12)


def test_chain_cg_edges(api, oracle, chain_everywhere):
    # zero right-hand side, max_iter, breakdown #2, warm start -- through the chain
    ptr, ind, val = matgen.lap2d(6)
    A = api.RowSparse(36, 36, ptr, ind, val)
    x0 = np.arange(36.0)
    X = to_dev(x0)
    it = api.Iteration(100, 1e-10)
    it.HideMessages()
    assert api.Cg(A, X, to_dev(np.zeros(36)), api.Preconditioner_Base(), it) == 0
    assert np.array_equal(to_host(X), x0)
    it = api.Iteration(3, 1e-30)
    it.HideMessages()
    assert api.Cg(A, to_dev(np.zeros(36)), to_dev(np.ones(36)), api.Preconditioner_Base(), it) == -2
    assert it.GetNumberIteration() == 3
    D = api.RowSparse(2, 2, np.array([0, 1, 2]), np.array([0, 1]), np.array([1.0, -1.0]))
    it = api.Iteration(10, 1e-12)
    it.HideMessages()
    assert api.Cg(D, to_dev(np.zeros(2)), to_dev(np.ones(2)), api.Preconditioner_Base(), it) == 2
    rng = np.random.default_rng(3)
    b, x0 = rng.standard_normal(36), rng.standard_normal(36)
    X = to_dev(x0)
    it = api.Iteration(1000, 1e-9)
    it.HideMessages()
    it.SetInitGuess(False)
    assert api.Cg(A, X, to_dev(b), api.Preconditioner_Base(), it) == 0
    xo, co, no, _, _ = oracle.solve("cg", ptr, ind, val, b, x0=x0, tol=1e-9, max_iter=1000)
    assert abs(it.GetNumberIteration() - no) <= 2
    assert np.linalg.norm(to_host(X) - xo) / np.linalg.norm(xo) < 1e-6


def test_chain_cg_large_vs_oracle(api, oracle):
    """Default dispatch at n = 250000 (chain path) against the oracle."""
    ptr, ind, val = matgen.lap2d(500)
    n = ptr.size - 1
    b = matgen.matvec(ptr, ind, val, np.random.default_rng(9).uniform(-1, 1, n))
    xo, co, no, _, _ = oracle.solve("cg", ptr, ind, val, b, tol=1e-8, max_iter=5000)
    A = api.RowSparse(n, n, ptr, ind, val)
    X = to_dev(np.zeros(n))
    it = api.Iteration(5000, 1e-8)
    it.HideMessages()
    assert api.Cg(A, X, to_dev(b), api.Preconditioner_Base(), it) == co == 0
    assert abs(it.GetNumberIteration() - no) <= max(2, no // 50)
    assert np.linalg.norm(to_host(X) - xo) / np.linalg.norm(xo) < 1e-5


# ------------------------------------------------------------------ chained BiCgStab

@pytest.mark.parametrize("mname,pc", [("conv", 0), ("conv", 1), ("conv16", 1), ("zipf", 0),
                                      ("lap_up", 0)])
def test_chain_bicgstab_parity(api, oracle, chain_everywhere, mname, pc):
    """BiCgStab (identity, Jacobi) through the chain of full-occupancy kernels
    that large systems take, against the oracle and the persistent kernel."""
    from seldon_b200 import _lib
    mats = _mats()
    if mname == "conv16":
        A = matgen.convdiff3d(16)
    elif mname == "zipf":
        A = matgen.zipf_csr(6000, seed=4, hi=1500)
    else:
        A = mats[mname]
    sym = mname.endswith("_up")
    full = mats["lap"] if sym else A
    n = A[0].size - 1
    b = matgen.matvec(*full, np.random.default_rng(7).uniform(-1, 1, n))
    xo, co, no, ho, hio = oracle.solve("bicgstab", *A, b, sym=sym, precond=pc, tol=1e-10,
                                       max_iter=5000, hist_cap=10000)
    M = api.RowSymSparse(n, *A) if sym else api.RowSparse(n, n, *A)

    def run():
        X = to_dev(np.zeros(n))
        it = api.Iteration(5000, 1e-10)
        it.HideMessages()
        P = api.JacobiPreconditioner() if pc else api.Preconditioner_Base()
        return api.BiCgStab(M, X, to_dev(b), P, it), it, to_host(X)
    code, it, x = run()
    assert code == co == 0
    assert abs(it.GetNumberIteration() - no) <= max(2, no // 10), (it.GetNumberIteration(), no)
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) < 1e-7
    # Finished() on ||r|| and on ||s||: the counter rises by one each time
    assert [h[0] for h in it.history] == list(range(it.GetNumberIteration() + 1))
    assert it.history[0][1] == pytest.approx(ho[0], rel=1e-12)
    # the persistent kernel: same stopping rule, agreement to rounding
    L = _lib.load()
    L.sb2_krylov_set_config(1 << 30)
    try:
        code_p, it_p, x_p = run()
    finally:
        L.sb2_krylov_set_config(0)
    assert code_p == 0 and abs(it_p.GetNumberIteration() - it.GetNumberIteration()) <= max(2, no // 10)
    assert np.linalg.norm(x - x_p) / np.linalg.norm(x_p) < 1e-7


def test_chain_bicgstab_edges(api, oracle, chain_everywhere):
    ptr, ind, val = matgen.convdiff3d(6)
    n = ptr.size - 1
    A = api.RowSparse(n, n, ptr, ind, val)
    P = api.Preconditioner_Base()
    # zero right-hand side: x untouched, ErrorCode 0
    x0 = np.arange(float(n))
    X = to_dev(x0)
    it = api.Iteration(100, 1e-10)
    it.HideMessages()
    assert api.BiCgStab(A, X, to_dev(np.zeros(n)), P, it) == 0
    assert np.array_equal(to_host(X), x0)
    b = matgen.matvec(ptr, ind, val, np.random.default_rng(4).uniform(-1, 1, n))
    # iteration limits: a stop on ||s|| (odd) and on ||r|| (even)
    for max_iter in (3, 4):
        X = to_dev(np.zeros(n))
        it = api.Iteration(max_iter, 1e-30)
        it.HideMessages()
        code = api.BiCgStab(A, X, to_dev(b), P, it)
        xo, co, no, _, _ = oracle.solve("bicgstab", ptr, ind, val, b, tol=1e-30, max_iter=max_iter)
        assert code == co == -2 and it.GetNumberIteration() == no == max_iter
        np.testing.assert_allclose(to_host(X), xo, rtol=1e-10, atol=1e-13)
    # warm start
    rng = np.random.default_rng(5)
    x0 = rng.standard_normal(n)
    X = to_dev(x0)
    it = api.Iteration(1000, 1e-9)
    it.HideMessages()
    it.SetInitGuess(False)
    assert api.BiCgStab(A, X, to_dev(b), P, it) == 0
    xo, co, no, _, _ = oracle.solve("bicgstab", ptr, ind, val, b, x0=x0, tol=1e-9, max_iter=1000)
    assert co == 0 and abs(it.GetNumberIteration() - no) <= max(2, no // 10)
    assert np.linalg.norm(to_host(X) - xo) / np.linalg.norm(xo) < 1e-6


# ------------------------------------------------------------------ cluster-resident CG

def _cluster_case(mat):
    if mat == "lap60":
        return matgen.lap2d(60)
    if mat == "poisson20":
        return matgen.poisson3d(20)
    if mat == "lap_odd":
        return matgen.lap2d(37, shift=0.3)
    return matgen.lap2d(50)


@pytest.mark.parametrize("mat,pc,warm", [("lap60", 0, False), ("lap60", 1, True),
                                         ("poisson20", 1, False), ("lap_odd", 0, True),
                                         ("sym_up", 0, False)])
def test_cluster_cg_matches_persistent(api, oracle, mat, pc, warm):
    # small systems run CG inside one thread-block cluster (shared and
    # distributed shared memory); the persistent kernel is the other path:
    # same stopping rule, iterations within the reduction-order slack,
    # solutions within the parity bound, both against the oracle
    from seldon_b200 import _lib
    L = _lib.load()
    ptr, ind, val = _cluster_case(mat)
    n = ptr.size - 1
    rng = np.random.default_rng(7)
    b = matgen.matvec(ptr, ind, val, rng.uniform(-1, 1, n))
    x0 = rng.uniform(-1, 1, n) if warm else np.zeros(n)
    A = api.RowSymSparse(n, *matgen.upper(ptr, ind, val)) if mat == "sym_up" else \
        api.RowSparse(n, n, ptr, ind, val)
    out = {}
    for on in (1, 0):
        old = L.sb2_krylov_set_cluster(on)
        try:
            X = to_dev(x0)
            it = api.Iteration(3000, 1e-10)
            it.HideMessages()
            it.SetInitGuess(not warm)
            code = api.Cg(A, X, to_dev(b), _precond(api, pc), it)
        finally:
            L.sb2_krylov_set_cluster(old)
        out[on] = (code, it.GetNumberIteration(), to_host(X), [r for _, r in it.history])
    (c1, n1, x1, h1), (c0, n0, x0_, h0) = out[1], out[0]
    assert c1 == c0 == 0
    assert abs(n1 - n0) <= 2, (n1, n0)
    assert h1[0] == pytest.approx(h0[0], rel=1e-13)
    assert np.linalg.norm(x1 - x0_) / np.linalg.norm(x0_) < 1e-8
    for xx in (x1, x0_):
        r = b - matgen.matvec(ptr, ind, val, xx)
        assert np.linalg.norm(r) / np.linalg.norm(b) < 50 * 1e-10
    _, co, no, _, _ = oracle.solve("cg", ptr, ind, val, b, x0=x0 if warm else None, precond=pc,
                                   tol=1e-10, max_iter=3000)
    assert co == 0 and abs(n1 - no) <= max(2, int(0.05 * no)), (n1, no)


def test_cluster_cg_edges(api):
    # zero right-hand side (x untouched, code 0) and a max_iter stop (-2),
    # on a system small enough for the cluster path
    ptr, ind, val = matgen.lap2d(40)
    n = ptr.size - 1
    A = api.RowSparse(n, n, ptr, ind, val)
    x0 = np.arange(n, dtype=float)
    X = to_dev(x0)
    it = api.Iteration(100, 1e-10)
    it.HideMessages()
    it.SetInitGuess(False)
    assert api.Cg(A, X, to_dev(np.zeros(n)), api.Preconditioner_Base(), it) == 0
    assert np.array_equal(to_host(X), x0)
    b = matgen.matvec(ptr, ind, val, np.ones(n))
    X = to_dev(np.zeros(n))
    it = api.Iteration(7, 1e-14)
    it.HideMessages()
    assert api.Cg(A, X, to_dev(b), api.Preconditioner_Base(), it) == -2
    assert it.GetNumberIteration() == 7


# ------------------------------------------------------------------ non-finite input

def _nonfinite(name):
    p, i, v = matgen.lap2d(12)
    n = p.size - 1
    b, x0 = np.ones(n), None
    v = v.copy()
    if name == "nan_b":
        b[5] = np.nan
    elif name == "inf_b":
        b[3] = np.inf
    elif name == "nan_A":
        v[7] = np.nan
    elif name == "inf_A":
        v[10] = np.inf
    elif name == "nan_x0":
        x0 = np.zeros(n)
        x0[2] = np.nan
    return p, i, v, b, x0


@pytest.mark.parametrize("name", ["nan_b", "inf_b", "nan_A", "inf_A", "nan_x0"])
@pytest.mark.parametrize("which", ["cg", "bicgstab", "gmres"])
@pytest.mark.parametrize("pc", [0, 1, 2])
@pytest.mark.parametrize("cluster", [True, False])
def test_nonfinite_inputs(api, oracle, name, which, pc, cluster):
    """NaN / Inf in b, A or x0: the same exit code (-2, max_iter reached) and
    iteration count as the oracle (pinned to Seldon), and NaN where the
    oracle has NaN."""
    from seldon_b200 import _lib
    p, i, v, b, x0 = _nonfinite(name)
    n = p.size - 1
    xo, co, no, _, _ = oracle.solve(which, p, i, v, b, x0=x0, precond=pc, omega=1.2,
                                    tol=1e-10, max_iter=25, restart=5)
    A = api.RowSparse(n, n, p, i, v, validate=True)
    X = to_dev(np.zeros(n) if x0 is None else x0)
    it = api.Iteration(25, 1e-10)
    it.SetRestart(5)
    it.HideMessages()
    if x0 is not None:
        it.SetInitGuess(False)
    old = _lib.load().sb2_krylov_set_cluster(int(cluster))
    try:
        fn = {"cg": api.Cg, "bicgstab": api.BiCgStab, "gmres": api.Gmres}[which]
        code = fn(A, X, to_dev(b), _precond(api, pc), it)
    finally:
        _lib.load().sb2_krylov_set_cluster(old)
    x = to_host(X)
    assert (code, it.GetNumberIteration()) == (co, no) == (-2, 25)
    assert np.array_equal(np.isnan(x), np.isnan(xo))


def _cg_by_hand(api, A, x, b, M, it):
    """Cg.cxx:45-116 written over the Python mirror's operations and
    Iteration's loop interface, as a user's own driver would be."""
    if A.GetM() <= 0:
        return 0
    p, q, r, z = (b.clone() for _ in range(4))
    if it.Init(b) != 0:
        return it.ErrorCode()
    api.Copy(b, r)
    if not it.IsInitGuess_Null():
        api.MltAdd(-1.0, A, x, 1.0, r)
    else:
        api.Fill(x, 0.0)
    it.SetNumberIteration(0)
    rho_1 = 1.0
    while not it.Finished(r):
        M.Solve(A, r, z)
        rho = api.DotProd(r, z)
        if rho == 0.0:
            it.Fail(1, "Cg breakdown #1")
            break
        if it.First():
            api.Copy(z, p)
        else:
            api.Mlt(rho / rho_1, p)
            api.Add(1.0, z, p)
        api.Mlt(A, p, q)
        delta = api.DotProd(p, q)
        if delta == 0.0:
            it.Fail(2, "Cg breakdown #2")
            break
        alpha = rho / delta
        api.Add(alpha, p, x)
        api.Add(-alpha, q, r)
        rho_1 = rho
        it += 1
    return it.ErrorCode()


@pytest.mark.parametrize("pc", [0, 1])
def test_hand_written_driver(api, pc):
    """A driver written against the Python mirror (its BLAS-1, MltAdd, the
    preconditioners' Solve and Iteration's Init/Finished/First/Fail/++)
    reaches the fused Cg's iterate: same exit code, iteration count within
    the reduction-order slack, same solution to 1e-8."""
    ptr, ind, val = matgen.lap2d(40)
    n = ptr.size - 1
    A = api.RowSparse(n, n, ptr, ind, val)
    b = to_dev(matgen.matvec(ptr, ind, val, np.random.default_rng(21).uniform(-1, 1, n)))
    out = []
    for solve in (_cg_by_hand, lambda api_, *a: api_.Cg(*a)):
        X = to_dev(np.zeros(n))
        it = api.Iteration(2000, 1e-10)
        it.HideMessages()
        code = solve(api, A, X, b, _precond(api, pc), it)
        out.append((code, it.GetNumberIteration(), to_host(X), it.ErrorCode()))
    (c0, n0, x0, e0), (c1, n1, x1, e1) = out
    assert c0 == c1 == e0 == e1 == 0
    assert abs(n0 - n1) <= max(2, n1 // 50), (n0, n1)
    assert np.linalg.norm(x0 - x1) / np.linalg.norm(x1) < 1e-8
