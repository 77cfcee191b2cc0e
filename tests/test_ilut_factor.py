"""The host ILUT factorization (sb2_ilut_factor) against Seldon's own
IlutPreconditioning::FactorizeMatrix: the factor's rows, in stored order,
and both permutations, bit for bit.  Host code only: no GPU needed."""
import numpy as np
import pytest

from seldon_b200 import matgen


@pytest.fixture(scope="module")
def api():
    from seldon_b200 import api as a
    return a


def _diag_dominant(n, density, seed, shift=4.0):
    import scipy.sparse as sp
    p, i, v = matgen.random_csr(n, n, density, seed=seed)
    S = sp.csr_matrix((v, i, p), shape=(n, n)) + sp.identity(n) * shift
    S.sort_indices()
    return S.indptr.astype(np.int32), S.indices.astype(np.int32), S.data


def _ours(api, p, i, v, perm, type_ilu, sym=False, **kw):
    M = api.IlutPreconditioning()
    M.SetFactorisationType(type_ilu)
    for key, set_ in (("fill_level", M.SetFillLevel), ("additional_fill", M.SetAdditionalFillNumber),
                      ("mbloc", M.SetPivotBlockInteger), ("alpha", M.SetDiagonalCoefficient),
                      ("droptol", M.SetDroppingThreshold), ("permtol", M.SetPivotThreshold)):
        if key in kw:
            set_(kw[key])
    return M.factor_host(p.size - 1, p, i, v, perm=perm, symmetric=sym)


CASES = [
    # (name, matrix, factorization type, options)
    ("conv6_ilut", lambda: matgen.convdiff3d(6), 0, dict(droptol=1e-3)),
    ("conv6_ilut_lfil", lambda: matgen.convdiff3d(6), 0, dict(droptol=1e-4, fill_level=3)),
    ("conv6_pivot", lambda: matgen.convdiff3d(6), 0, dict(droptol=1e-4, permtol=0.5)),
    ("conv6_pivot_blocks", lambda: matgen.convdiff3d(6), 0,
     dict(droptol=1e-4, permtol=0.9, mbloc=17)),
    ("conv6_ilu_d", lambda: matgen.convdiff3d(6), 1, dict(droptol=1e-2, alpha=0.7)),
    ("conv6_ilut_k", lambda: matgen.convdiff3d(6), 2, dict(droptol=1e-3, additional_fill=2)),
    ("rand_ilut", lambda: _diag_dominant(400, 0.02, 3), 0, dict(droptol=1e-3)),
    ("rand_pivot", lambda: _diag_dominant(400, 0.02, 5, shift=0.5), 0,
     dict(droptol=1e-4, permtol=0.3, fill_level=8)),
    ("rand_pivot_blocks", lambda: _diag_dominant(400, 0.02, 5, shift=0.5), 0,
     dict(droptol=1e-4, permtol=0.3, fill_level=8, mbloc=13)),
    ("rand_ilu_d", lambda: _diag_dominant(300, 0.03, 7), 1, dict(droptol=0.05)),
    ("lap_ilut_k", lambda: matgen.lap2d(20), 2, dict(droptol=1e-2, additional_fill=1)),
]


@pytest.mark.parametrize("name,make,type_ilu,kw", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("ordered", [False, True])
def test_factor_matches_reference(api, reference, name, make, type_ilu, kw, ordered):
    p, i, v = make()
    n = p.size - 1
    perm = np.random.default_rng(n).permutation(n) if ordered else None
    ours = _ours(api, p, i, v, perm, type_ilu, **kw)
    theirs = reference.ilut_factor(p, i, v, perm=perm, type_ilu=type_ilu, **kw)
    for name_, a, b in zip(("fptr", "find", "fval", "perm_row", "perm_col"), ours, theirs):
        assert a.shape == b.shape, name_
        assert np.array_equal(a, b), name_


def test_rejections(api):
    from seldon_b200._lib import SeldonB200Error
    p = np.array([0, 1, 2], dtype=np.int32)
    i = np.array([0, 1], dtype=np.int32)
    M = api.IlutPreconditioning()
    with pytest.raises(SeldonB200Error):  # a row of zeros
        M.factor_host(2, p, i, np.array([1.0, 0.0]))
    with pytest.raises(SeldonB200Error):  # not a permutation
        M.factor_host(2, p, i, np.ones(2), perm=np.array([0, 0]))
    with pytest.raises(SeldonB200Error):  # a repeated column
        M.factor_host(1, np.array([0, 2], dtype=np.int32), np.array([0, 0], dtype=np.int32),
                      np.ones(2))


@pytest.mark.parametrize("sym", [False, True])
def test_fill_below_one_is_refused(api, sym):
    """ILUT with fill level 0, or ILUT_K with additional fill at or below
    minus a row's length, keeps no pivot; the reference then writes past the
    row it resized, so the factorization is refused.  ILU_D ignores the fill
    level and keeps the pivot."""
    from seldon_b200._lib import SeldonB200Error, SB2_ERR_INVALID_VALUE
    A = matgen.upper(*matgen.lap2d(6)) if sym else matgen.convdiff3d(4)
    for type_ilu, kw in ((0, dict(fill_level=0)), (2, dict(additional_fill=-7))):
        with pytest.raises(SeldonB200Error) as e:
            _ours(api, *A, None, type_ilu, sym=sym, droptol=1e-3, **kw)
        assert e.value.status == SB2_ERR_INVALID_VALUE
    fptr, find, fval, prow, pcol = _ours(api, *A, None, 1, sym=sym, droptol=1e-3, fill_level=0)
    assert np.all(np.diff(fptr) >= 1)


SYM_CASES = [
    ("lap_ilut", lambda: matgen.upper(*matgen.lap2d(20)), 0, dict(droptol=1e-3)),
    ("lap_ilut_lfil", lambda: matgen.upper(*matgen.lap2d(20)), 0, dict(droptol=1e-4, fill_level=4)),
    ("lap_ilu_d", lambda: matgen.upper(*matgen.lap2d(20)), 1, dict(droptol=1e-2, alpha=0.5)),
    ("lap_ilut_k", lambda: matgen.upper(*matgen.lap2d(20)), 2, dict(droptol=1e-3, additional_fill=2)),
    ("poisson_ilut", lambda: matgen.upper(*matgen.poisson3d(7)), 0, dict(droptol=1e-3)),
    ("spd_rand", lambda: _spd_upper(300, 0.02, 9), 0, dict(droptol=1e-3, fill_level=10)),
]


def _spd_upper(n, density, seed):
    import scipy.sparse as sp
    p, i, v = matgen.random_csr(n, n, density, seed=seed)
    S = sp.csr_matrix((v, i, p), shape=(n, n))
    S = (S + S.T) * 0.5 + sp.identity(n) * 8.0
    U = sp.triu(S).tocsr()
    U.sort_indices()
    return U.indptr.astype(np.int32), U.indices.astype(np.int32), U.data


@pytest.mark.parametrize("name,make,type_ilu,kw", SYM_CASES, ids=[c[0] for c in SYM_CASES])
@pytest.mark.parametrize("ordered", [False, True])
def test_symmetric_factor_matches_reference(api, reference, name, make, type_ilu, kw, ordered):
    p, i, v = make()
    n = p.size - 1
    perm = np.random.default_rng(n + 1).permutation(n) if ordered else None
    ours = _ours(api, p, i, v, perm, type_ilu, sym=True, **kw)
    theirs = reference.ilut_factor(p, i, v, sym=True, perm=perm, type_ilu=type_ilu, **kw)
    for name_, a, b in zip(("fptr", "find", "fval", "perm_row", "perm_col"), ours, theirs):
        assert a.shape == b.shape, name_
        assert np.array_equal(a, b), name_


class _HostMatrix:
    """Stands in for RowSparse / RowSymSparse on the host: the factorization
    only downloads the arrays (and clears the matrix unless asked to keep it)."""

    def __init__(self, p, i, v, symmetric=False):
        self.m = p.size - 1
        self.symmetric = symmetric
        self._arrays = (p, i, v)
        self.cleared = False

    def download(self):
        return self._arrays

    def Clear(self):
        self.cleared = True
        self.m = 0


def test_interface_matches_reference(api):
    """Defaults and accessors of IlutPreconditioning (IlutPreconditioning.cxx:
    27-168), and FactorizeMatrix in both call forms: (A, perm=None) keeps A,
    the reference's (perm, A, keep_matrix=False) clears it unless asked."""
    M = api.IlutPreconditioning()
    assert (M.GetFactorisationType(), M.GetFillLevel(), M.GetAdditionalFillNumber(),
            M.GetPivotBlockInteger(), M.GetPrintLevel()) == (M.ILUT, 1000000, 1000000, 1000000, 0)
    assert (M.GetDiagonalCoefficient(), M.GetDroppingThreshold(), M.GetPivotThreshold()) == \
        (1.0, 0.01, 0.1)
    M.SetFillLevel(7)
    M.SetAdditionalFillNumber(3)
    M.SetPivotBlockInteger(11)
    M.SetPrintLevel(2)
    M.SetDiagonalCoefficient(0.5)
    M.SetDroppingThreshold(1e-3)
    M.SetPivotThreshold(0.4)
    assert (M.GetFillLevel(), M.GetAdditionalFillNumber(), M.GetPivotBlockInteger(),
            M.GetPrintLevel(), M.GetDiagonalCoefficient(), M.GetDroppingThreshold(),
            M.GetPivotThreshold()) == (7, 3, 11, 2, 0.5, 1e-3, 0.4)
    p, i, v = matgen.convdiff3d(5)
    n = p.size - 1
    perm = np.random.default_rng(1).permutation(n).astype(np.int32)
    want = M.factor_host(n, p, i, v, perm=perm)
    for args, kw, cleared in (((None,), dict(perm=perm), False), ((perm, None), {}, True),
                              ((perm, None, True), {}, False), ((perm, None, False), {}, True)):
        A = _HostMatrix(p, i, v)
        args = tuple(A if a is None else a for a in args)
        M.FactorizeMatrix(*args, **kw)
        assert A.cleared == cleared
        got = M._factor
        for a, b in zip(got[1:6], want):
            assert np.array_equal(a, b)
    M.Clear()
    assert M._factor is None
    with pytest.raises(ValueError):  # the reference aborts on a wrong-size ordering
        M.FactorizeMatrix(perm[:-1], _HostMatrix(p, i, v))
    with pytest.raises(NotImplementedError):
        M.FactorizeSymMatrix(perm, _HostMatrix(p, i, v))
    up = matgen.upper(*matgen.lap2d(5))
    S = _HostMatrix(*up, symmetric=True)
    with pytest.raises(NotImplementedError):
        M.FactorizeUnsymMatrix(np.arange(25), S)
    M.FactorizeSymMatrix(np.arange(25), S, True)
    assert not S.cleared and M._factor[6]
