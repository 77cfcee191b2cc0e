"""Hand-written adjoint of x = A^{-1} b (torch.autograd wrappers): gradients
against an FP64 dense reference and central finite differences."""
import numpy as np
import pytest

from seldon_b200 import matgen

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ag(cuda):
    from seldon_b200 import autograd
    return autograd


def _dense(ptr, ind, val, n):
    A = np.zeros((n, n))
    rows = np.repeat(np.arange(n), np.diff(ptr))
    np.add.at(A, (rows, ind), val)
    return A


def test_graph_laplacian_gradients(ag):
    import torch
    g = 24
    n = g * g
    rng = np.random.default_rng(0)
    edges = matgen.grid_edges(g)
    theta = rng.lognormal(0.0, 1.0, edges.shape[0])
    xt = rng.standard_normal(n)
    b = rng.standard_normal(n)
    lap = ag.GraphLaplacian(n, edges, 1e-3)
    T = torch.tensor(theta, device="cuda", requires_grad=True)
    B = torch.tensor(b, device="cuda", requires_grad=True)
    XT = torch.tensor(xt, device="cuda")
    x = ag.graph_laplacian_solve(T, B, lap, 1e-13)
    loss = 0.5 * ((x - XT) ** 2).sum()
    loss.backward()
    gt, gb = T.grad.cpu().numpy(), B.grad.cpu().numpy()
    # FP64 dense reference gradient
    ptr, ind, val, _ = matgen.aniso2d(g, theta, 1e-3)
    A = _dense(ptr, ind, val, n)
    xr = np.linalg.solve(A, b)
    lam = np.linalg.solve(A.T, xr - xt)
    gref = -(lam[edges[:, 0]] - lam[edges[:, 1]]) * (xr[edges[:, 0]] - xr[edges[:, 1]])
    assert np.linalg.norm(x.detach().cpu().numpy() - xr) / np.linalg.norm(xr) < 1e-9
    assert np.linalg.norm(gt - gref) / np.linalg.norm(gref) < 1e-8
    assert np.linalg.norm(gb - lam) / np.linalg.norm(lam) < 1e-8
    # central finite differences, h = 1e-6, on random edges.  L(theta +- h e)
    # is formed from the perturbation dx = x(theta +- h e) - x, which solves
    # (A +- h E_e) dx = -+ h E_e x with E_e = (e_i - e_j)(e_i - e_j)^T, so the
    # difference is not lost to cancellation in L ~ 1e2:
    #   L(theta +- h e) - L(theta) = dx . (x - x_t) + |dx|^2 / 2
    h = 1e-6
    xg = x.detach()
    res = (xg - XT)

    def dL(th, i, j, sign):
        rhs = torch.zeros(n, dtype=torch.float64, device="cuda")
        d = float(xg[i] - xg[j])
        rhs[i] = -sign * h * d
        rhs[j] = sign * h * d
        with torch.no_grad():
            dx = ag.graph_laplacian_solve(torch.tensor(th, device="cuda"), rhs, lap, 1e-13)
        return float(dx @ res) + 0.5 * float(dx @ dx)
    for e in rng.choice(edges.shape[0], 16, replace=False):
        i, j = edges[e]
        tp, tm = theta.copy(), theta.copy()
        tp[e] += h
        tm[e] -= h
        fd = (dL(tp, i, j, 1.0) - dL(tm, i, j, -1.0)) / (2 * h)
        assert abs(fd - gt[e]) <= 1e-5 * abs(gt[e]) + 1e-9, (e, fd, gt[e])


def test_general_pattern_gradient(ag):
    import torch
    ptr, ind, val = matgen.convdiff3d(6)
    n = ptr.size - 1
    rng = np.random.default_rng(1)
    P = ag.SparsePattern(n, ptr, ind)
    V = torch.tensor(val, device="cuda", requires_grad=True)
    b = torch.tensor(rng.standard_normal(n), device="cuda", requires_grad=True)
    xt = torch.tensor(rng.standard_normal(n), device="cuda")
    x = ag.sparse_solve(V, b, P, 1e-13)
    loss = 0.5 * ((x - xt) ** 2).sum()
    loss.backward()
    A = _dense(ptr, ind, val, n)
    xr = np.linalg.solve(A, b.detach().cpu().numpy())
    lam = np.linalg.solve(A.T, xr - xt.cpu().numpy())
    rows = np.repeat(np.arange(n), np.diff(ptr))
    gref = -lam[rows] * xr[ind]
    assert np.linalg.norm(V.grad.cpu().numpy() - gref) / np.linalg.norm(gref) < 1e-8
    assert np.linalg.norm(b.grad.cpu().numpy() - lam) / np.linalg.norm(lam) < 1e-8
