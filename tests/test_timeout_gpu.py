"""The bounded waits of the fused persistent solvers, made to run out.

Every grid barrier of the cooperative CG, BiCGSTAB and GMRES kernels (both
orthogonalizations) polls
its release flag for at most the wait limit (%globaltimer).  With the limit
set to one microsecond, a CTA that reaches a barrier before the slowest CTA
stops waiting, records the timeout and leaves; the others leave at their next
barrier.  The call must return SB2_ERR_TIMEOUT (no hang, no fault), the
context must stay usable, and the same handle must then solve to the
oracle's result once the default limit is back.  Nothing here waits on a flag
that stays unset: each wait ends by the clock."""
import numpy as np
import pytest

from seldon_b200 import matgen

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("which", ["cg", "bicgstab", "gmres", "gmres_cgs2"])
def test_wait_limit_runs_out_then_solves(cuda, oracle, which):
    import torch
    from seldon_b200 import _lib, api
    L = _lib.load()
    ptr, ind, val = matgen.poisson3d(48)  # 110,592 rows: a grid of ~108 CTAs
    n = ptr.size - 1
    b = matgen.matvec(ptr, ind, val, np.random.default_rng(3).uniform(-1, 1, n))
    A = api.RowSparse(n, n, ptr, ind, val)
    B = torch.as_tensor(b, device="cuda")
    solver = {"cg": api.Cg, "bicgstab": api.BiCgStab, "gmres": api.Gmres,
              "gmres_cgs2": lambda *a: api.Gmres(*a, orthogonalization="cgs2")}[which]

    def run():
        X = torch.zeros(n, dtype=torch.float64, device="cuda")
        it = api.Iteration(5000, 1e-10)
        it.HideMessages()
        it.SetRestart(20)
        solver(A, X, B, api.Preconditioner_Base(), it)
        return X, it

    old_cluster = L.sb2_krylov_set_cluster(0)  # the cooperative kernel, not the cluster one
    try:
        X0, it0 = run()  # before: the default limit
        old_us = L.sb2_set_wait_limit_us(1)
        try:
            with pytest.raises(_lib.SeldonB200Error) as err:
                run()
            assert err.value.status == _lib.SB2_ERR_TIMEOUT
        finally:
            assert L.sb2_set_wait_limit_us(old_us) == 1
        torch.cuda.synchronize()  # the context is intact
        X, it = run()
    finally:
        L.sb2_krylov_set_cluster(old_cluster)
    # the same handle solves as before the timeout, bit for bit (the
    # reductions have a fixed order), and meets the oracle
    assert torch.equal(X, X0) and it.GetNumberIteration() == it0.GetNumberIteration()
    xo, co, no, _, _ = oracle.solve(which.split("_")[0], ptr, ind, val, b, tol=1e-10,
                                    max_iter=5000, restart=20)
    x = X.cpu().numpy()
    assert it.ErrorCode() == co == 0
    # BiCGSTAB's iteration count follows rounding more closely than CG's
    slack = max(2, no // (10 if which == "bicgstab" else 20))
    assert abs(it.GetNumberIteration() - no) <= slack, (it.GetNumberIteration(), no)
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) < 1e-7
