"""Mixed-precision iterative refinement (FP32 inner CG, FP64 outer): reaches
the FP64 tolerance on the true residual, and its forward error against the
FP64 oracle solution stays at the level that tolerance implies."""
import numpy as np
import pytest

from seldon_b200 import matgen
from tests.helpers import to_dev, to_host

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def api(cuda):
    from seldon_b200 import api
    return api


@pytest.mark.parametrize("restarted", [False, True])
@pytest.mark.parametrize("g,pc", [(16, 0), (24, 1), (40, 0)])
def test_ir_reaches_fp64_tolerance(api, oracle, g, pc, restarted):
    ptr, ind, val = matgen.poisson3d(g)
    n = ptr.size - 1
    xs = np.random.default_rng(g).uniform(-1, 1, n)
    b = matgen.matvec(ptr, ind, val, xs)
    A = api.RowSparse(n, n, ptr, ind, val)
    X = to_dev(np.zeros(n))
    M = api.JacobiPreconditioner() if pc else None
    code, info = api.IterativeRefinement(A, X, to_dev(b), M, tol=1e-10, restarted=restarted)
    x = to_host(X)
    assert code == 0, info
    assert info["outer_iter"] >= 2
    rel = np.linalg.norm(b - matgen.matvec(ptr, ind, val, x)) / np.linalg.norm(b)
    assert rel < 1e-10 and rel == pytest.approx(info["rel_residual"], rel=1e-6)
    xo, co, no, _, _ = oracle.solve("cg", ptr, ind, val, b, precond=pc, tol=1e-10, max_iter=5000)
    if not restarted:
        # reliable updates keep CG's Krylov space: the FP32 iteration count
        # stays close to the FP64 oracle's
        assert info["inner_iter"] <= 1.3 * no + 10, (info["inner_iter"], no)
    # both solutions meet ||r||/||b|| < 1e-10; their distance is bounded by
    # the conditioning of the Laplacian (kappa ~ g^2) times the tolerance
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) < 1e-10 * 4 * g * g
    h = info["history"]
    assert h[0] == pytest.approx(1.0) and h[-1] < 1e-10
    assert all(h[i + 1] < h[i] for i in range(len(h) - 1))


def test_ir_warm_start_and_edges(api):
    ptr, ind, val = matgen.poisson3d(10)
    n = ptr.size - 1
    A = api.RowSparse(n, n, ptr, ind, val)
    # zero right-hand side: nothing to do, x untouched
    x0 = np.arange(n, dtype=float)
    X = to_dev(x0)
    code, info = api.IterativeRefinement(A, X, to_dev(np.zeros(n)), init_guess_null=False)
    assert code == 0 and info["init_failed"] and np.array_equal(to_host(X), x0)
    # warm start from an exact solution: converged before any step
    xs = np.random.default_rng(1).standard_normal(n)
    b = matgen.matvec(ptr, ind, val, xs)
    X = to_dev(xs)
    code, info = api.IterativeRefinement(A, X, to_dev(b), init_guess_null=False)
    assert code == 0 and info["outer_iter"] == 0
    # max_outer reached -> -2
    X = to_dev(np.zeros(n))
    code, info = api.IterativeRefinement(A, X, to_dev(b), tol=1e-30, max_outer=2)
    assert code == -2 and info["outer_iter"] == 2
    # SOR has no FP32 inner form
    from seldon_b200._lib import SeldonB200Error
    with pytest.raises(SeldonB200Error):
        api.IterativeRefinement(A, X, to_dev(b), api.SorPreconditioner())


@pytest.mark.parametrize("restarted", [False, True])
def test_ir_large_chained(api, restarted):
    # 128^3: the chained FP32 kernels with many slices per reduction; the true
    # residual is recomputed here, independent of the solver's own report
    ptr, ind, val = matgen.poisson3d(128)
    n = ptr.size - 1
    xs = np.random.default_rng(5).uniform(-1, 1, n)
    b = matgen.matvec(ptr, ind, val, xs)
    A = api.RowSparse(n, n, ptr, ind, val)
    X = to_dev(np.zeros(n))
    code, info = api.IterativeRefinement(A, X, to_dev(b), tol=1e-10, restarted=restarted)
    x = to_host(X)
    assert code == 0, info
    rel = np.linalg.norm(b - matgen.matvec(ptr, ind, val, x)) / np.linalg.norm(b)
    assert rel < 1e-10 and rel == pytest.approx(info["rel_residual"], rel=1e-6)
    X64 = to_dev(np.zeros(n))
    it = api.Iteration(20000, 1e-10)
    it.HideMessages()
    assert api.Cg(A, X64, to_dev(b), api.Preconditioner_Base(), it) == 0
    nb = it.GetNumberIteration()
    if not restarted:
        # FP32 CG with reliable updates needs about the FP64 iteration count:
        # not fewer (CG's optimality) and not many more
        assert 0.9 * nb <= info["inner_iter"] <= 1.2 * nb + 10, (info["inner_iter"], nb)
    assert np.linalg.norm(x - to_host(X64)) / np.linalg.norm(xs) < 1e-7
