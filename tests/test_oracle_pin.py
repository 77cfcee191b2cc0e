"""The oracle (oracle/seldon_oracle.c) is pinned before it is trusted:
bit-for-bit against golden vectors produced by the reference itself, and
against the live reference build where oracle/_ref exists."""
import os

import numpy as np
import pytest

from seldon_b200 import matgen

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "seldon_golden.npz")


@pytest.fixture(scope="module")
def golden():
    return np.load(GOLDEN)


def _mat(g, name):
    return (g[f"mat/{name}/ptr"], g[f"mat/{name}/ind"], g[f"mat/{name}/val"],
            int(g[f"mat/{name}/m"]), int(g[f"mat/{name}/n"]))


@pytest.mark.parametrize("name", ["lap2d_9", "conv_4", "rand_37x29"])
def test_mltadd_golden(golden, oracle, name):
    ptr, ind, val, m, n = _mat(golden, name)
    k = f"mltadd/{name}"
    out = oracle.mltadd(m, n, ptr, ind, val, float(golden[k + "/alpha"]), golden[k + "/x"],
                        float(golden[k + "/beta"]), golden[k + "/y"])
    assert np.array_equal(out, golden[k + "/out"])
    k = f"mltadd_t/{name}"
    out = oracle.mltadd(m, n, ptr, ind, val, float(golden[k + "/alpha"]), golden[k + "/x"],
                        float(golden[k + "/beta"]), golden[k + "/y"], trans=True)
    assert np.array_equal(out, golden[k + "/out"])


def test_mltadd_sym_golden(golden, oracle):
    ptr, ind, val, m, n = _mat(golden, "lap2d_9_upper")
    k = "mltadd_sym/lap2d_9"
    out = oracle.mltadd(m, n, ptr, ind, val, float(golden[k + "/alpha"]), golden[k + "/x"],
                        float(golden[k + "/beta"]), golden[k + "/y"], sym=True)
    assert np.array_equal(out, golden[k + "/out"])


@pytest.mark.parametrize("t", [0, 2, 3])
@pytest.mark.parametrize("sym", [0, 1])
def test_sor_golden(golden, oracle, t, sym):
    name = "lap2d_9_upper" if sym else "lap2d_9"
    ptr, ind, val, m, n = _mat(golden, name)
    k = f"sor/t{t}_s{sym}"
    out = oracle.sor(ptr, ind, val, golden[k + "/x0"], golden[k + "/b"], float(golden[k + "/omega"]),
                     int(golden[k + "/it"]), t, sym=bool(sym))
    assert np.array_equal(out, golden[k + "/out"])


def _solve_keys(g):
    return sorted({k.split("/")[1] for k in g.files if k.startswith("solve/")})


def test_solvers_golden(golden, oracle):
    keys = _solve_keys(golden)
    assert len(keys) >= 12
    for key in keys:
        which, rest = key.split("_", 1)
        mname, pc, sym = rest.rsplit("_", 2)
        pc, sym = int(pc[1:]), int(sym[1:])
        ptr, ind, val, m, n = _mat(golden, mname)
        A = matgen.upper(ptr, ind, val) if sym else (ptr, ind, val)
        k = f"solve/{key}"
        x, code, nb, _, _ = oracle.solve(which, *A, golden[k + "/b"], sym=bool(sym), precond=pc,
                                         omega=float(golden[k + "/omega"]),
                                         tol=float(golden[k + "/tol"]),
                                         max_iter=int(golden[k + "/max_iter"]),
                                         restart=int(golden[k + "/restart"]))
        assert code == int(golden[k + "/code"]), key
        assert nb == int(golden[k + "/nb"]), key
        assert np.array_equal(x, golden[k + "/x"]), key


def test_genrot_golden(golden, oracle):
    for a, b, r, z, c, s in golden["genrot/table"]:
        assert oracle.genrot(a, b) == (r, z, c, s)


# ---------------------------------------------------------------- live reference

@pytest.mark.parametrize("seed", range(6))
def test_mltadd_live(reference, oracle, seed):
    rng = np.random.default_rng(seed)
    m, n = int(rng.integers(1, 80)), int(rng.integers(1, 80))
    ptr, ind, val = matgen.random_csr(m, n, float(rng.uniform(0.02, 0.4)), seed=seed,
                                      empty_rows=0.2)
    x, y = rng.standard_normal(n), rng.standard_normal(m)
    a, b = float(rng.standard_normal()), float(rng.standard_normal())
    assert np.array_equal(oracle.mltadd(m, n, ptr, ind, val, a, x, b, y),
                          reference.mltadd(m, n, ptr, ind, val, a, x, b, y))
    xt, yt = rng.standard_normal(m), rng.standard_normal(n)
    assert np.array_equal(oracle.mltadd(m, n, ptr, ind, val, a, xt, b, yt, trans=True),
                          reference.mltadd(m, n, ptr, ind, val, a, xt, b, yt, trans=True))


@pytest.mark.parametrize("which", ["cg", "bicgstab", "gmres", "cgs", "tfqmr", "minres", "gcr",
                                   "bicgstabl", "qcgs", "bicg", "cgne", "bicgcr", "lsqr",
                                   "qmrsym", "symmlq"])
@pytest.mark.parametrize("pc", [0, 1, 2])
def test_solvers_live(reference, oracle, which, pc):
    ptr, ind, val = (matgen.convdiff3d(5) if which not in ("cg", "minres", "qmrsym", "symmlq")
                     else matgen.lap2d(15))
    m = ptr.size - 1
    rng = np.random.default_rng(7)
    b = matgen.matvec(ptr, ind, val, rng.uniform(-1, 1, m))
    xo, co, no, _, _ = oracle.solve(which, ptr, ind, val, b, precond=pc, tol=1e-10,
                                    max_iter=500, restart=8, omega=1.1)
    xr, cr, nr = reference.solve(which, ptr, ind, val, b, precond=pc, tol=1e-10,
                                 max_iter=500, restart=8, omega=1.1)
    assert (co, no) == (cr, nr)
    assert np.array_equal(xo, xr)


def test_breakdown_and_edge_codes(reference, oracle):
    # zero right-hand side: Init fails, x untouched, code 0 (Iterative.cxx:240-241)
    ptr, ind, val = matgen.lap2d(4)
    b = np.zeros(16)
    x0 = np.arange(16.0)
    for which in ("cg", "bicgstab", "gmres"):
        xo, co, no, _, _ = oracle.solve(which, ptr, ind, val, b, x0=x0)
        xr, cr, nr = reference.solve(which, ptr, ind, val, b, x0=x0)
        assert co == cr
        assert np.array_equal(xo, xr)
    # max_iter reached -> -2
    b = np.ones(16)
    xo, co, no, _, _ = oracle.solve("cg", ptr, ind, val, b, tol=1e-30, max_iter=3)
    xr, cr, nr = reference.solve("cg", ptr, ind, val, b, tol=1e-30, max_iter=3)
    assert co == cr == -2 and no == nr == 3
    # CG on an indefinite matrix with a vanishing p.q -> breakdown #2
    ptr = np.array([0, 1, 2], dtype=np.int32)
    ind = np.array([0, 1], dtype=np.int32)
    val = np.array([1.0, -1.0])
    b = np.array([1.0, 1.0])
    xo, co, no, _, _ = oracle.solve("cg", ptr, ind, val, b)
    xr, cr, nr = reference.solve("cg", ptr, ind, val, b)
    assert co == cr == 2


def _edge_solves():
    """Small cases on the edges of Cgs and TfQmr: a zero right-hand side with
    a nonzero guess, an exact guess (TfQmr's Init sees a zero preconditioned
    residual), iteration limits 0 to 3, and the indefinite 2 x 2 system whose
    first projections vanish."""
    ptr, ind, val = matgen.lap2d(4)
    n = 16
    rng = np.random.default_rng(5)
    xs = rng.uniform(-1, 1, n)
    b = matgen.matvec(ptr, ind, val, xs)
    out = [("zero_b", (ptr, ind, val), np.zeros(n), np.arange(16.0), {}),
           ("exact_x0", (ptr, ind, val), b, xs, {})]
    for k in range(4):
        out.append((f"max_iter_{k}", (ptr, ind, val), b, None, {"tol": 1e-30, "max_iter": k}))
    ind2 = np.array([0, 1], dtype=np.int32)
    out.append(("indefinite", (np.array([0, 1, 2], dtype=np.int32), ind2,
                               np.array([1.0, -1.0])), np.array([1.0, 1.0]), None, {}))
    out.append(("one_by_one", (np.array([0, 1], dtype=np.int32), ind2[:1], np.array([4.0])),
                np.array([2.0]), None, {}))
    return out


@pytest.mark.parametrize("restart", [1, 2, 5, 16, 24])
def test_gcr_restarts_live(reference, oracle, restart):
    ptr, ind, val = matgen.convdiff3d(6)
    b = np.random.default_rng(5).uniform(-1, 1, ptr.size - 1)
    for pc in (0, 1):
        xo, co, no, _, _ = oracle.solve("gcr", ptr, ind, val, b, precond=pc, tol=1e-10,
                                        max_iter=600, restart=restart)
        xr, cr, nr = reference.solve("gcr", ptr, ind, val, b, precond=pc, tol=1e-10,
                                     max_iter=600, restart=restart)
        assert (co, no) == (cr, nr)
        assert np.array_equal(xo, xr)


@pytest.mark.parametrize("l", [1, 2, 4, 10, 16, 20])
def test_bicgstabl_live(reference, oracle, l):
    ptr, ind, val = matgen.convdiff3d(6)
    b = np.random.default_rng(7).uniform(-1, 1, ptr.size - 1)
    for pc in (0, 1, 2):
        xo, co, no, _, _ = oracle.solve("bicgstabl", ptr, ind, val, b, precond=pc, omega=1.1,
                                        tol=1e-10, max_iter=600, restart=l)
        assert co == 0
        xr, cr, nr = reference.solve("bicgstabl", ptr, ind, val, b, precond=pc, omega=1.1,
                                     tol=1e-10, max_iter=600, restart=l)
        assert (co, no) == (cr, nr)
        assert np.array_equal(xo, xr)


def test_bicgstabl_no_progress_stops(oracle):
    """diag(1, -1), b = (1, 1): sigma = (A r, r) vanishes at the first step,
    then rho_0 = 0 at every later cycle, and the reference repeats that
    cycle for ever; the restatement stops after it.  Never run on the
    reference."""
    p, i, v = (np.array([0, 1, 2], dtype=np.int32), np.array([0, 1], dtype=np.int32),
               np.array([1.0, -1.0]))
    _, code, nb, h, _ = oracle.solve("bicgstabl", p, i, v, np.array([1.0, 1.0]), tol=1e-10,
                                     max_iter=100, hist_cap=10)
    assert (code, nb) == (1, 1) and len(h) == 2


@pytest.mark.parametrize("which", ["bicg", "cgne", "lsqr"])
@pytest.mark.parametrize("sor_sym", [True, False])
def test_bicg_transpose_live(reference, oracle, sor_sym, which):
    """BiCg's and Cgne's product by A^T: the reference's Mlt(SeldonTrans, ...)
    runs the generic loop over M(j, i) (Functions_MatVect.cxx:1279-1317) --
    column sums for RowSparse, full symmetric rows for RowSymSparse -- and
    SOR's TransSolve sweeps backward when the preconditioner is not
    symmetric."""
    cases = [(matgen.convdiff3d(5), False), (matgen.upper(*matgen.poisson3d(6)), True),
             (matgen.upper(*matgen.lap2d(12)), True)]
    for A, sym in cases:
        b = np.random.default_rng(9).uniform(-1, 1, A[0].size - 1)
        for pc in (0, 1, 2):
            xo, co, no, _, _ = oracle.solve(which, *A, b, sym=sym, precond=pc, omega=1.1,
                                            sor_sym=sor_sym, tol=1e-10, max_iter=400)
            xr, cr, nr = reference.solve(which, *A, b, sym=sym, precond=pc, omega=1.1,
                                         sor_sym=sor_sym, tol=1e-10, max_iter=400)
            assert (co, no) == (cr, nr)
            assert np.array_equal(xo, xr)


def test_cocg_is_cg_live(reference):
    """The reference's CoCg in real arithmetic gives its Cg's bits (the same
    steps without conjugation), which is why sb2_cocg runs Cg's engines."""
    cases = [(matgen.lap2d(15), False), (matgen.upper(*matgen.lap2d(15)), True),
             (matgen.convdiff3d(6), False)]
    for A, sym in cases:
        b = np.random.default_rng(3).uniform(-1, 1, A[0].size - 1)
        for pc in (0, 1, 2):
            x1, c1, n1 = reference.solve("cg", *A, b, sym=sym, precond=pc, omega=1.1,
                                         tol=1e-10, max_iter=500)
            x2, c2, n2 = reference.solve("cocg", *A, b, sym=sym, precond=pc, omega=1.1,
                                         tol=1e-10, max_iter=500)
            assert (c1, n1) == (c2, n2)
            assert np.array_equal(x1, x2, equal_nan=True)
    for name, (p, i, v), b, x0, kw in _edge_solves():
        for pc in (0, 1, 2):
            x1, c1, n1 = reference.solve("cg", p, i, v, b, x0=x0, precond=pc, **kw)
            x2, c2, n2 = reference.solve("cocg", p, i, v, b, x0=x0, precond=pc, **kw)
            assert (c1, n1) == (c2, n2), name
            assert np.array_equal(x1, x2, equal_nan=True), name


def test_gcr_no_step_stops(oracle):
    """Where the reference's Gcr never returns (a cycle that takes no step:
    a breakdown at its first product, or restart 0), the restatement stops
    after that cycle.  Never run on the reference."""
    one = (np.array([0, 1], dtype=np.int32), np.array([0], dtype=np.int32), np.array([0.0]))
    _, code, nb, _, _ = oracle.solve("gcr", *one, np.array([1.0]), tol=1e-10, max_iter=50)
    assert (code, nb) == (1, 0)
    ptr, ind, val = matgen.lap2d(4)
    x, code, nb, h, _ = oracle.solve("gcr", ptr, ind, val, np.ones(16), tol=1e-10, max_iter=50,
                                     restart=0, hist_cap=10)
    assert (code, nb) == (0, 0) and not x.any() and len(h) == 2


def shifted_laplacian(g, sigma):
    """The g x g Laplacian minus sigma I: symmetric indefinite for sigma
    above its smallest eigenvalue (MinRes's case)."""
    ptr, ind, val = matgen.lap2d(g)
    val = val.copy()
    rows = np.repeat(np.arange(ptr.size - 1), np.diff(ptr))
    val[ind == rows] -= sigma
    return ptr, ind, val


@pytest.mark.parametrize("pc", [0, 1, 2])
@pytest.mark.parametrize("sym", [False, True])
def test_minres_indefinite_live(reference, oracle, pc, sym):
    full = shifted_laplacian(15, 0.5)
    A = matgen.upper(*full) if sym else full
    b = np.random.default_rng(4).uniform(-1, 1, full[0].size - 1)
    xo, co, no, _, _ = oracle.solve("minres", *A, b, sym=sym, precond=pc, omega=1.1,
                                    tol=1e-10, max_iter=500)
    xr, cr, nr = reference.solve("minres", *A, b, sym=sym, precond=pc, omega=1.1, tol=1e-10,
                                 max_iter=500)
    assert (co, no) == (cr, nr)
    assert np.array_equal(xo, xr)


@pytest.mark.parametrize("which", ["cgs", "tfqmr", "minres", "gcr", "bicgstabl", "qcgs", "bicg",
                                   "cgne", "bicgcr", "lsqr", "qmrsym", "symmlq"])
def test_cgs_tfqmr_edges_live(reference, oracle, which):
    for name, (p, i, v), b, x0, kw in _edge_solves():
        for pc in (0, 1, 2):
            xo, co, no, _, _ = oracle.solve(which, p, i, v, b, x0=x0, precond=pc, **kw)
            if which == "bicgstabl" and co in (1, 2):
                # after a breakdown the reference's BiCgStabl may repeat a
                # cycle that counts nothing for ever: never run it there
                continue
            xr, cr, nr = reference.solve(which, p, i, v, b, x0=x0, precond=pc, **kw)
            assert (co, no) == (cr, nr), (name, pc)
            assert np.array_equal(xo, xr, equal_nan=True), (name, pc)


COO_CASES = ["gen_dup_i1", "gen_min", "sym_both", "sym_i1_min", "empty_gen", "empty_sym"]


def _coo(g, name):
    k = f"coo/{name}"
    return (g[k + "/row"], g[k + "/col"], g[k + "/val"], int(g[k + "/index"]),
            int(g[k + "/m_min"]), int(g[k + "/n_min"]), bool(g[k + "/sym"]))


@pytest.mark.parametrize("name", COO_CASES)
def test_coo_to_csr_golden(golden, oracle, name):
    row, col, val, index, m_min, n_min, sym = _coo(golden, name)
    m, n, ptr, ind, out = oracle.coo_to_csr(row, col, val, index, m_min, n_min, sym)
    k = f"coo/{name}"
    assert (m, n) == (int(golden[k + "/m"]), int(golden[k + "/n"]))
    assert np.array_equal(ptr, golden[k + "/ptr"])
    assert np.array_equal(ind, golden[k + "/ind"])
    assert np.array_equal(out, golden[k + "/out"])


def test_coo_to_csr_live_fuzz(oracle, reference):
    """Random triplets (many duplicates, both index bases, both storages,
    current sizes larger and smaller than the entries) against Seldon's own
    ConvertMatrix_from_Coordinates."""
    rng = np.random.default_rng(11)
    for _ in range(200):
        nnz = int(rng.integers(0, 300))
        m, n = int(rng.integers(1, 30)), int(rng.integers(1, 30))
        index, sym = int(rng.integers(0, 2)), bool(rng.integers(0, 2))
        if sym:
            n = m
        row = rng.integers(0, m, nnz) + index
        col = rng.integers(0, n, nnz) + index
        val = rng.standard_normal(nnz)
        m_min, n_min = int(rng.integers(0, 40)), int(rng.integers(0, 40))
        a = oracle.coo_to_csr(row, col, val, index, m_min, n_min, sym)
        b = reference.coo_to_csr(row, col, val, index, m_min, n_min, sym)
        assert a[:2] == b[:2]
        for u, v in zip(a[2:], b[2:]):
            assert np.array_equal(u, v)


ILUT_CASES = ["conv5_ilut", "conv5_perm_piv", "conv5_ilu0", "conv5_iluk2", "lap9_sym"]


def ilut_factor(g, name):
    k = f"ilut/{name}"
    return tuple(g[f"{k}/{a}"] for a in ("fptr", "find", "fval", "prow", "pcol"))


@pytest.mark.parametrize("name", ILUT_CASES)
def test_ilut_solve_golden(golden, oracle, name):
    k = f"ilut/{name}"
    sym = bool(golden[k + "/sym"])
    f = ilut_factor(golden, name)
    assert np.array_equal(oracle.ilut_solve(f, golden[k + "/r"], sym=sym), golden[k + "/z"])
    assert np.array_equal(oracle.ilut_solve(f, golden[k + "/r"], sym=sym, trans=True),
                          golden[k + "/zt"])


def test_ilut_solve_live(oracle, reference):
    """Seldon's factorization of larger and harder systems; the oracle's
    solve equals Seldon's bit for bit."""
    rng = np.random.default_rng(17)
    cases = [(matgen.convdiff3d(9), False, dict(droptol=1e-4)),
             (matgen.convdiff3d(8), False, dict(droptol=1e-5, permtol=0.3)),
             (matgen.upper(*matgen.lap2d(25)), True, dict(droptol=1e-4)),
             (matgen.convdiff3d(8), False, dict(type_ilu=reference.MILU_0))]
    for (p, i, v), sym, kw in cases:
        f = reference.ilut_factor(p, i, v, sym=sym, perm=rng.permutation(p.size - 1), **kw)
        for trans in (False, True):
            r = rng.standard_normal(p.size - 1)
            assert np.array_equal(oracle.ilut_solve(f, r, sym=sym, trans=trans),
                                  reference.ilut_solve(r, trans=trans))


def _nonfinite_cases():
    p, i, v = matgen.lap2d(12)
    n = p.size - 1
    out = {}
    b = np.ones(n)
    b[5] = np.nan
    out["nan_b"] = (p, i, v, b, None)
    b = np.ones(n)
    b[3] = np.inf
    out["inf_b"] = (p, i, v, b, None)
    v2 = v.copy()
    v2[7] = np.nan
    out["nan_A"] = (p, i, v2, np.ones(n), None)
    v3 = v.copy()
    v3[10] = np.inf
    out["inf_A"] = (p, i, v3, np.ones(n), None)
    x0 = np.zeros(n)
    x0[2] = np.nan
    out["nan_x0"] = (p, i, v, np.ones(n), x0)
    return out


@pytest.mark.parametrize("name", list(_nonfinite_cases()))
def test_nonfinite_inputs_live(oracle, reference, name):
    """NaN and Inf in b, A or x0: Seldon's drivers never see the residual
    fall below tol and stop at max_iter with -2; the oracle does the same,
    with the same iterate (NaNs included)."""
    p, i, v, b, x0 = _nonfinite_cases()[name]
    for which in ("cg", "bicgstab", "gmres"):
        for pc in (0, 1, 2):
            xo, co, no, _, _ = oracle.solve(which, p, i, v, b, x0=x0, precond=pc, tol=1e-10,
                                            max_iter=25, restart=5)
            xr, cr, nr = reference.solve(which, p, i, v, b, x0=x0, precond=pc, tol=1e-10,
                                         max_iter=25, restart=5)
            assert (co, no) == (cr, nr) == (-2, 25)
            assert np.array_equal(xo, xr, equal_nan=True)
    # Cgs counts two per loop and TfQmr's scalars may vanish on an infinite
    # product: the codes and counts are the reference's, whatever they are
    for which in ("cgs", "tfqmr", "minres", "gcr", "bicgstabl", "qcgs", "bicg", "cgne",
                  "bicgcr", "lsqr", "qmrsym", "symmlq"):
        for pc in (0, 1, 2):
            xo, co, no, _, _ = oracle.solve(which, p, i, v, b, x0=x0, precond=pc, tol=1e-10,
                                            max_iter=25)
            xr, cr, nr = reference.solve(which, p, i, v, b, x0=x0, precond=pc, tol=1e-10,
                                         max_iter=25)
            assert (co, no) == (cr, nr)
            assert np.array_equal(xo, xr, equal_nan=True)
