"""ILUT preconditioner apply on the device (sb2_precond_create_ilut):
Solve and TransSolve against the reference's golden vectors and the oracle
bit for bit, from factors Seldon's GetIlut computed, on level schedules of
one CTA (n <= 65536) and of one launch per level; and Cg / BiCgStab / Gmres
preconditioned by it against the reference's own preconditioned solves."""
import os

import numpy as np
import pytest

from seldon_b200 import matgen
from tests.helpers import to_dev, to_host

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "seldon_golden.npz")
ILUT_CASES = ["conv5_ilut", "conv5_perm_piv", "conv5_ilu0", "conv5_iluk2", "lap9_sym"]


@pytest.fixture(scope="module")
def api(cuda):
    from seldon_b200 import api as a
    return a


def _precond(api, factor, sym):
    M = api.IlutPreconditioning()
    fptr, find, fval, prow, pcol = factor
    M.SetFactor(fptr, find, fval, prow, pcol, symmetric=sym)
    return M


def _apply(api, M, A, r, trans):
    R = to_dev(r)
    Z = to_dev(np.zeros_like(r))
    (M.TransSolve if trans else M.Solve)(A, R, Z)
    return to_host(Z)


def _dummy(api, n):
    ptr = np.arange(n + 1, dtype=np.int32)
    return api.RowSparse(n, n, ptr, np.arange(n, dtype=np.int32), np.ones(n))


@pytest.mark.parametrize("name", ILUT_CASES)
def test_ilut_golden(api, name):
    g = np.load(GOLDEN)
    k = f"ilut/{name}"
    factor = tuple(g[f"{k}/{a}"] for a in ("fptr", "find", "fval", "prow", "pcol"))
    sym = bool(g[k + "/sym"])
    n = factor[0].size - 1
    M = _precond(api, factor, sym)
    A = _dummy(api, n)
    assert np.array_equal(_apply(api, M, A, g[k + "/r"], False), g[k + "/z"])
    assert np.array_equal(_apply(api, M, A, g[k + "/r"], True), g[k + "/zt"])


# (matrix, symmetric storage, factor options): the 3D ones are large enough
# for one launch per level (n > 65536)
LARGE = [
    ("conv20", lambda: matgen.convdiff3d(20), False, dict(droptol=1e-3)),
    ("conv20_perm", lambda: matgen.convdiff3d(20), False, dict(droptol=1e-3, permtol=0.3)),
    ("conv42", lambda: matgen.convdiff3d(42), False, dict(droptol=1e-2)),
    ("conv42_ilu0", lambda: matgen.convdiff3d(42), False, dict(type_ilu=3)),
    ("lap300_sym", lambda: matgen.upper(*matgen.lap2d(300)), True, dict(droptol=1e-2)),
]


@pytest.mark.parametrize("name,make,sym,kw", LARGE, ids=[c[0] for c in LARGE])
def test_ilut_vs_oracle(api, oracle, reference, name, make, sym, kw):
    p, i, v = make()
    n = p.size - 1
    rng = np.random.default_rng(n)
    perm = rng.permutation(n) if name.endswith("_perm") else None
    factor = reference.ilut_factor(p, i, v, sym=sym, perm=perm, **kw)
    M = _precond(api, factor, sym)
    A = _dummy(api, n)
    for trans in (False, True):
        r = rng.standard_normal(n)
        z = _apply(api, M, A, r, trans)
        assert np.array_equal(z, oracle.ilut_solve(factor, r, sym=sym, trans=trans))


def test_ilut_rejects_bad_factor(api):
    from seldon_b200._lib import SeldonB200Error
    # a row without a diagonal position (all columns below the row)
    fptr = np.array([0, 1, 2], dtype=np.int32)
    find = np.array([0, 0], dtype=np.int32)
    M = api.IlutPreconditioning()
    M.SetFactor(fptr, find, np.ones(2), np.arange(2), np.arange(2))
    with pytest.raises(SeldonB200Error):
        M.Solve(_dummy(api, 2), to_dev(np.ones(2)), to_dev(np.zeros(2)))
    # a permutation that is not one
    fptr = np.array([0, 1, 2], dtype=np.int32)
    find = np.array([0, 1], dtype=np.int32)
    M.SetFactor(fptr, find, np.ones(2), np.array([0, 0]), np.arange(2))
    with pytest.raises(SeldonB200Error):
        M.Solve(_dummy(api, 2), to_dev(np.ones(2)), to_dev(np.zeros(2)))


@pytest.mark.parametrize("which,sym", [("bicgstab", False), ("gmres", False), ("cg", True),
                                       ("gmres", True)])
def test_krylov_with_ilut(api, reference, which, sym):
    """Preconditioned drivers reach the reference's iterate: same exit code,
    iteration count within the drift of the dot products' summation order,
    and the same solution to 1e-7."""
    if sym:
        full = matgen.lap2d(40)
        A = matgen.upper(*full)
    else:
        A = full = matgen.convdiff3d(14)
    n = A[0].size - 1
    factor = reference.ilut_factor(*A, sym=sym, droptol=1e-2)
    b = matgen.matvec(*full, np.random.default_rng(5).uniform(-1, 1, n))
    tol, restart = 1e-10, 10
    xr, cr, nr = reference.solve_ilut(which, *A, b, sym=sym, tol=tol, max_iter=500,
                                      restart=restart)
    M = api.RowSymSparse(n, *A) if sym else api.RowSparse(n, n, *A)
    X = to_dev(np.zeros(n))
    it = api.Iteration(500, tol)
    it.SetRestart(restart)
    it.HideMessages()
    fn = {"cg": api.Cg, "bicgstab": api.BiCgStab, "gmres": api.Gmres}[which]
    code = fn(M, X, to_dev(b), _precond(api, factor, sym), it)
    x = to_host(X)
    assert code == cr == 0
    nb = it.GetNumberIteration()
    assert abs(nb - nr) <= max(1, int(0.05 * nr)), (nb, nr)
    assert np.linalg.norm(x - xr) / np.linalg.norm(xr) < 1e-7
    assert nb < 0.5 * _plain_iterations(api, M, b, which, tol, restart)


def _plain_iterations(api, M, b, which, tol, restart):
    X = to_dev(np.zeros(b.size))
    it = api.Iteration(5000, tol)
    it.SetRestart(restart)
    it.HideMessages()
    fn = {"cg": api.Cg, "bicgstab": api.BiCgStab, "gmres": api.Gmres}[which]
    fn(M, X, to_dev(b), api.Preconditioner_Base(), it)
    return it.GetNumberIteration()


@pytest.mark.parametrize("name,make", [
    ("conv9", lambda: matgen.convdiff3d(9)),
    ("conv45", lambda: matgen.convdiff3d(45)),          # one launch per level
    ("rand", lambda: _diag_dominant(3000, 0.004, 2)),
])
@pytest.mark.parametrize("milu", [False, True])
def test_ilu0_device_factor(api, oracle, reference, name, make, milu):
    """ILU(0) and MILU(0) factored on the device apply exactly like the
    factor Seldon's GetIlu0 / GetMilu0 computes (so the factors agree bit for
    bit)."""
    p, i, v = make()
    n = p.size - 1
    A = api.RowSparse(n, n, p, i, v)
    M = api.IlutPreconditioning()
    M.SetFactorisationType(M.MILU_0 if milu else M.ILU_0)
    M.FactorizeMatrix(A)
    factor = reference.ilut_factor(p, i, v,
                                   type_ilu=reference.MILU_0 if milu else reference.ILU_0)
    rng = np.random.default_rng(7)
    for trans in (False, True):
        r = rng.standard_normal(n)
        assert np.array_equal(_apply(api, M, A, r, trans),
                              oracle.ilut_solve(factor, r, trans=trans))


def test_ilu0_rejects_unsorted_and_missing_diagonal(api):
    from seldon_b200._lib import SeldonB200Error
    ptr = np.array([0, 2, 3], dtype=np.int32)
    M = api.IlutPreconditioning()
    M.SetFactorisationType(M.ILU_0)
    A = api.RowSparse(2, 2, ptr, np.array([1, 0, 1], dtype=np.int32), np.ones(3))
    with pytest.raises(SeldonB200Error):
        M.FactorizeMatrix(A)
    A = api.RowSparse(2, 2, ptr, np.array([0, 1, 0], dtype=np.int32), np.ones(3))
    with pytest.raises(SeldonB200Error):
        M.FactorizeMatrix(A)


def _diag_dominant(n, density, seed):
    import scipy.sparse as sp
    p, i, v = matgen.random_csr(n, n, density, seed=seed)
    S = sp.csr_matrix((v, i, p), shape=(n, n)) + sp.identity(n) * 4.0
    S.sort_indices()
    return S.indptr.astype(np.int32), S.indices.astype(np.int32), S.data


def test_factor_types(api, oracle, reference):
    """ILUT (the default) is factored on the host in GetIlut's order and
    applied on the device like Seldon's; ILU_K asks for Seldon's factor."""
    p, i, v = matgen.convdiff3d(12)
    n = p.size - 1
    A = api.RowSparse(n, n, p, i, v)
    M = api.IlutPreconditioning()
    assert M.GetFactorisationType() == M.ILUT
    M.SetDroppingThreshold(1e-3)
    perm = np.random.default_rng(2).permutation(n)
    M.FactorizeMatrix(A, perm=perm)
    factor = reference.ilut_factor(p, i, v, perm=perm, droptol=1e-3)
    r = np.random.default_rng(4).standard_normal(n)
    for trans in (False, True):
        assert np.array_equal(_apply(api, M, A, r, trans),
                              oracle.ilut_solve(factor, r, trans=trans))
    M.SetFactorisationType(M.ILU_K)
    with pytest.raises(NotImplementedError):
        M.FactorizeMatrix(A)


def test_symmetric_factor_on_host_and_cg(api, oracle, reference):
    """The symmetric algorithm factored on the host (GetIlut of the symmetric
    preconditioner, bit for bit) applies on the device like Seldon's factor,
    and preconditions CG."""
    full = matgen.lap2d(60)
    up = matgen.upper(*full)
    n = up[0].size - 1
    S = api.RowSymSparse(n, *up)
    M = api.IlutPreconditioning()
    M.SetSymmetricAlgorithm()
    M.SetDroppingThreshold(1e-3)
    M.FactorizeMatrix(S)
    factor = reference.ilut_factor(*up, sym=True, droptol=1e-3)
    r = np.random.default_rng(8).standard_normal(n)
    assert np.array_equal(_apply(api, M, S, r, False), oracle.ilut_solve(factor, r, sym=True))
    b = matgen.matvec(*full, np.random.default_rng(9).uniform(-1, 1, n))
    X = to_dev(np.zeros(n))
    it = api.Iteration(1000, 1e-10)
    it.HideMessages()
    assert api.Cg(S, X, to_dev(b), M, it) == 0
    assert it.GetNumberIteration() < 0.5 * _plain_iterations(api, S, b, "cg", 1e-10, 10)
    with pytest.raises(NotImplementedError):  # symmetric storage needs the symmetric algorithm
        api.IlutPreconditioning().FactorizeMatrix(S)


def test_reference_call_forms(api, oracle, reference):
    """The reference's FactorizeMatrix(perm, A) clears A (keep_matrix false);
    the device ILU(0) factor keeps no reference to A and applies to another
    matrix of the same order, in Solve / TransSolve and in BiCgStab; the
    in-place forms Solve(z), TransSolve(z) and Solve(SeldonTrans, z) equal
    the three-argument ones, for a device and a host factor."""
    p, i, v = matgen.convdiff3d(9)
    n = p.size - 1
    rng = np.random.default_rng(12)
    r = rng.standard_normal(n)
    A = api.RowSparse(n, n, p, i, v)
    M = api.IlutPreconditioning()
    M.SetFactorisationType(M.ILU_0)
    M.FactorizeMatrix(np.arange(n), A)
    assert A.GetM() == 0
    A2 = api.RowSparse(n, n, p, i, v)
    factor = reference.ilut_factor(p, i, v, type_ilu=reference.ILU_0)
    for trans in (False, True):
        assert np.array_equal(_apply(api, M, A2, r, trans),
                              oracle.ilut_solve(factor, r, trans=trans))
    b = matgen.matvec(p, i, v, rng.uniform(-1, 1, n))
    X = to_dev(np.zeros(n))
    it = api.Iteration(500, 1e-10)
    it.HideMessages()
    assert api.BiCgStab(A2, X, to_dev(b), M, it) == 0
    H = api.IlutPreconditioning()
    H.SetDroppingThreshold(1e-3)
    H.FactorizeMatrix(rng.permutation(n), A2, True)
    assert A2.GetM() == n
    for P in (M, H):
        want, want_t = _apply(api, P, A2, r, False), _apply(api, P, A2, r, True)
        Z = to_dev(r)
        P.Solve(Z)
        assert np.array_equal(to_host(Z), want)
        Z = to_dev(r)
        P.TransSolve(Z)
        assert np.array_equal(to_host(Z), want_t)
        Z = to_dev(r)
        P.Solve(api.SeldonTrans, Z)
        assert np.array_equal(to_host(Z), want_t)
