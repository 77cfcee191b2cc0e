"""Shared helpers for the test-suite (parity criteria and device transfers)."""
import numpy as np

# FP64 SpMV parity bar: normwise relative error and an elementwise bound
# scaled by sum_j |a_ij x_j| (Laplacian outputs cancel to ~0, so a pure
# elementwise relative test would be meaningless).
SPMV_RTOL = 1e-12


def to_dev(a):
    import torch
    return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64)).cuda()


def to_host(t):
    return t.detach().cpu().numpy()


def abs_matvec(ptr, ind, val, x):
    ptr = np.asarray(ptr, dtype=np.int64)
    rows = np.repeat(np.arange(ptr.size - 1), np.diff(ptr))
    return np.bincount(rows, weights=np.abs(val * x[ind]), minlength=ptr.size - 1)


def assert_spmv_close(y, y_ref, scale, rtol=SPMV_RTOL):
    """Normwise and scaled elementwise FP64 SpMV agreement."""
    y = np.asarray(y)
    y_ref = np.asarray(y_ref)
    both_nan = np.isnan(y) & np.isnan(y_ref)
    assert np.array_equal(np.isnan(y), np.isnan(y_ref)), "NaN pattern differs"
    y = np.where(both_nan, 0.0, y)
    y_ref = np.where(both_nan, 0.0, y_ref)
    nrm = np.linalg.norm(y_ref)
    err = np.linalg.norm(y - y_ref)
    assert err <= rtol * max(nrm, 1e-300) or err == 0.0, f"normwise {err / max(nrm, 1e-300):.3e}"
    bound = rtol * (np.asarray(scale) + np.abs(y_ref)) + 1e-300
    bad = np.abs(y - y_ref) > bound
    assert not bad.any(), f"{bad.sum()} entries beyond the elementwise bound"
