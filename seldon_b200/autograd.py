"""torch.autograd.Function wrappers of the sparse solve x = A^{-1} b.

The backward pass is the hand-written adjoint, run entirely in
libseldon_b200.so:

    A^T lambda = dL/dx          (the library's CG for symmetric A,
                                 BiCGSTAB on A^T otherwise)
    dL/db      = lambda
    dL/dA_ij   = -lambda_i x_j  on the stored pattern      (sb2_grad_pattern)
    dL/dtheta_e = -(lambda_i - lambda_j)(x_i - x_j)         (sb2_grad_edges,
                                 graph Laplacian A = L(theta) + shift I)

torch supplies device memory and the autograd graph; no solve runs in torch.
"""
import ctypes

import numpy as np
import torch

from . import _lib, api
from ._lib import check

_L = _lib.load()


def _vp(t):
    return ctypes.c_void_p(t.data_ptr())


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


class SparsePattern:
    """A fixed CSR pattern on the device whose values change per call."""

    def __init__(self, n, ptr, ind, symmetric_values=False):
        self.n = int(n)
        self.ptr = np.ascontiguousarray(ptr, dtype=np.int32)
        self.ind = np.ascontiguousarray(ind, dtype=np.int32)
        self.nnz = self.ind.size
        self.symmetric_values = bool(symmetric_values)
        self.A = api.RowSparse(self.n, self.n, self.ptr, self.ind, np.zeros(self.nnz))
        self._current = None
        rows = np.repeat(np.arange(self.n), np.diff(self.ptr))
        self.rows = torch.as_tensor(rows.astype(np.int64)).cuda()
        self.cols = torch.as_tensor(self.ind.astype(np.int64)).cuda()
        if not symmetric_values:
            # A^T on the same pattern: position of (j, i) for every entry (i, j)
            key = rows.astype(np.int64) * self.n + self.ind
            tkey = self.ind.astype(np.int64) * self.n + rows
            order = np.argsort(key)
            tpos = order[np.searchsorted(key[order], tkey)]
            if not np.array_equal(key[tpos], tkey):
                raise ValueError("the pattern must be structurally symmetric for the adjoint")
            self.tpos = torch.as_tensor(tpos).cuda()
            self.AT = api.RowSparse(self.n, self.n, self.ptr, self.ind, np.zeros(self.nnz))

    def set_values(self, values):
        v = values.detach().contiguous()
        check(_L.sb2_csr_set_values(self.A.handle, _vp(v), 1, _stream()), "sb2_csr_set_values")
        self._current = v
        if not self.symmetric_values:
            vt = v[self.tpos].contiguous()
            check(_L.sb2_csr_set_values(self.AT.handle, _vp(vt), 1, _stream()),
                  "sb2_csr_set_values")


def _solve(A, b, tol, max_iter, symmetric):
    x = torch.zeros_like(b)
    it = api.Iteration(max_iter, tol)
    it.HideMessages()
    if symmetric:
        code = api.Cg(A, x, b.contiguous(), api.Preconditioner_Base(), it)
    else:
        code = api.BiCgStab(A, x, b.contiguous(), api.Preconditioner_Base(), it)
    if code != 0:
        raise RuntimeError(f"sparse solve did not converge (Iteration::ErrorCode {code}, "
                           f"{it.GetNumberIteration()} iterations)")
    return x


class SparseSolve(torch.autograd.Function):
    """x = A(values)^{-1} b on a fixed pattern; gradients for values and b."""

    @staticmethod
    def forward(ctx, values, b, pattern, tol=1e-12, max_iter=100000):
        pattern.set_values(values)
        x = _solve(pattern.A, b, tol, max_iter, pattern.symmetric_values)
        ctx.pattern, ctx.tol, ctx.max_iter = pattern, tol, max_iter
        ctx.save_for_backward(values, x)
        return x

    @staticmethod
    def backward(ctx, gx):
        values, x = ctx.saved_tensors
        P = ctx.pattern
        if P._current is None or P._current.data_ptr() != values.data_ptr():
            P.set_values(values)
        AT = P.A if P.symmetric_values else P.AT
        lam = _solve(AT, gx.contiguous().double(), ctx.tol, ctx.max_iter, P.symmetric_values)
        gv = None
        if ctx.needs_input_grad[0]:
            gv = torch.empty(P.nnz, dtype=torch.float64, device=x.device)
            check(_L.sb2_grad_pattern(P.A.handle, -1.0, _vp(lam), _vp(x), _vp(gv), _stream()),
                  "sb2_grad_pattern")
        gb = lam if ctx.needs_input_grad[1] else None
        return gv, gb, None, None, None


class GraphLaplacian:
    """A(theta) = sum_e theta_e (e_i - e_j)(e_i - e_j)^T + shift I on fixed edges."""

    def __init__(self, n, edges, shift):
        edges = np.asarray(edges, dtype=np.int64)
        if edges.size == 0:
            edges = edges.reshape(0, 2)
        if edges.ndim != 2 or edges.shape[1] != 2:
            raise ValueError("WrongDim: edges must be an (E, 2) array of vertex pairs")
        if edges.size and (edges.min() < 0 or edges.max() >= n):
            # sb2_grad_edges reads lambda and x through these indices unchecked
            raise ValueError(f"WrongRow: an edge index lies outside [0, {n})")
        self.n, self.shift = int(n), float(shift)
        self.E = edges.shape[0]
        rows = np.concatenate([edges[:, 0], edges[:, 1], np.arange(n)])
        cols = np.concatenate([edges[:, 1], edges[:, 0], np.arange(n)])
        order = np.argsort(rows * n + cols, kind="stable")
        ptr = np.zeros(n + 1, dtype=np.int64)
        np.cumsum(np.bincount(rows, minlength=n), out=ptr[1:])
        inv = np.empty_like(order)
        inv[order] = np.arange(order.size)
        self.pos_ij = torch.as_tensor(inv[:self.E]).cuda()
        self.pos_ji = torch.as_tensor(inv[self.E:2 * self.E]).cuda()
        self.pos_d = torch.as_tensor(inv[2 * self.E:]).cuda()
        self.ei = torch.as_tensor(edges[:, 0].astype(np.int32)).cuda()
        self.ej = torch.as_tensor(edges[:, 1].astype(np.int32)).cuda()
        self.ei64 = self.ei.long()
        self.ej64 = self.ej.long()
        self.pattern = SparsePattern(n, ptr, cols[order], symmetric_values=True)

    def values(self, theta):
        v = torch.zeros(self.pattern.nnz, dtype=torch.float64, device=theta.device)
        v[self.pos_ij] = -theta
        v[self.pos_ji] = -theta
        deg = torch.zeros(self.n, dtype=torch.float64, device=theta.device)
        deg.index_add_(0, self.ei64, theta)
        deg.index_add_(0, self.ej64, theta)
        v[self.pos_d] = deg + self.shift
        return v


class GraphLaplacianSolve(torch.autograd.Function):
    """x = (L(theta) + shift I)^{-1} b with dL/dtheta_e = -(lambda_i - lambda_j)(x_i - x_j)."""

    @staticmethod
    def forward(ctx, theta, b, lap, tol=1e-12, max_iter=100000):
        lap.pattern.set_values(lap.values(theta.detach()))
        x = _solve(lap.pattern.A, b, tol, max_iter, True)
        ctx.lap, ctx.tol, ctx.max_iter = lap, tol, max_iter
        ctx.save_for_backward(theta, x)
        return x

    @staticmethod
    def backward(ctx, gx):
        theta, x = ctx.saved_tensors
        lap = ctx.lap
        lap.pattern.set_values(lap.values(theta.detach()))
        lam = _solve(lap.pattern.A, gx.contiguous().double(), ctx.tol, ctx.max_iter, True)
        gt = None
        if ctx.needs_input_grad[0]:
            gt = torch.empty(lap.E, dtype=torch.float64, device=x.device)
            check(_L.sb2_grad_edges(lap.E, _vp(lap.ei), _vp(lap.ej), _vp(lam), _vp(x), _vp(gt),
                                    _stream()), "sb2_grad_edges")
        gb = lam if ctx.needs_input_grad[1] else None
        return gt, gb, None, None, None


def sparse_solve(values, b, pattern, tol=1e-12, max_iter=100000):
    return SparseSolve.apply(values, b, pattern, tol, max_iter)


def graph_laplacian_solve(theta, b, lap, tol=1e-12, max_iter=100000):
    return GraphLaplacianSolve.apply(theta, b, lap, tol, max_iter)
