"""Calls from several host threads at once, each on its own CUDA stream,
sharing one matrix handle.  The matrix's lazily built members (the diagonal
Jacobi reads, the cluster-resident CG plan) are built under the handle's
lock; every stream has its own reduction scratch and takes its solver work
vectors from the stream-ordered pool.  So each thread gets exactly what a
lone call on another handle of the same matrix gives, bit for bit.  (ctypes
releases the interpreter lock for the call, so the threads do overlap.)"""
import threading

import numpy as np
import pytest

from seldon_b200 import matgen

pytestmark = pytest.mark.gpu

N_THREADS = 4


def _work(api, torch, A, x, b, stream):
    """MltAdd, DotProd, Norm2 and a Jacobi-preconditioned Cg (the
    cluster-resident path at this size) on one stream."""
    n = x.size
    sp = stream.cuda_stream
    with torch.cuda.stream(stream):
        X = torch.as_tensor(x).cuda()
        Y = torch.zeros(n, dtype=torch.float64, device="cuda")
        api.MltAdd(2.0, A, X, 0.0, Y, stream=sp)
        dot = api.DotProd(X, Y, stream=sp)
        nrm = api.Norm2(Y, stream=sp)
        S = torch.zeros(n, dtype=torch.float64, device="cuda")
        B = torch.as_tensor(b).cuda()
        it = api.Iteration(3000, 1e-10)
        it.HideMessages()
        code = api.Cg(A, S, B, api.JacobiPreconditioner(), it, stream=sp)
        stream.synchronize()
        return (Y.cpu().numpy(), dot, nrm, S.cpu().numpy(), code, it.GetNumberIteration())


@pytest.mark.parametrize("sym", [False, True])
def test_threads_share_a_matrix(cuda, sym):
    import torch
    from seldon_b200 import api
    p, i, v = matgen.lap2d(60)
    n = p.size - 1
    rng = np.random.default_rng(11)
    xs = [rng.uniform(-1, 1, n) for _ in range(N_THREADS)]
    bs = [matgen.matvec(p, i, v, x) for x in xs]

    def make():
        return api.RowSymSparse(n, *matgen.upper(p, i, v)) if sym else api.RowSparse(n, n, p, i, v)

    lone = [_work(api, torch, make(), xs[k], bs[k], torch.cuda.Stream()) for k in range(N_THREADS)]
    for _ in range(3):  # a fresh shared handle each round: its lazy members race
        A = make()
        streams = [torch.cuda.Stream() for _ in range(N_THREADS)]
        start = threading.Barrier(N_THREADS)
        out, err = [None] * N_THREADS, []

        def run(k):
            try:
                start.wait()
                out[k] = _work(api, torch, A, xs[k], bs[k], streams[k])
            except Exception as e:  # reported below, on the main thread
                err.append(e)

        ts = [threading.Thread(target=run, args=(k,)) for k in range(N_THREADS)]
        for t in ts:
            t.start()
        for t in ts:
            t.join(timeout=120)
        assert not any(t.is_alive() for t in ts)
        assert not err, err
        for k in range(N_THREADS):
            y, dot, nrm, s, code, nb = out[k]
            y0, dot0, nrm0, s0, code0, nb0 = lone[k]
            assert code == code0 == 0
            assert nb == nb0
            assert np.array_equal(y, y0) and dot == dot0 and nrm == nrm0
            assert np.array_equal(s, s0)
            assert np.linalg.norm(s - xs[k]) / np.linalg.norm(xs[k]) < 1e-6
