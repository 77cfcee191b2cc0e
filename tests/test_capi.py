"""The C ABI library loads and exports every symbol include/*.h declares
(no device call is made: these run without a GPU)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = set()
    inc = os.path.join(ROOT, "include")
    for f in os.listdir(inc):
        if f.endswith(".h"):
            src = open(os.path.join(inc, f)).read()
            src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
            names |= set(re.findall(r"\b(sb2_\w+)\s*\(", src))
    return names


def test_library_exports_every_declared_symbol():
    from seldon_b200 import _lib
    lib = _lib.load()
    declared = _declared()
    assert len(declared) >= 25
    missing = [n for n in sorted(declared) if not hasattr(lib, n)]
    assert not missing, missing


def test_python_prototypes_cover_header():
    from seldon_b200 import _lib
    assert _declared() <= set(_lib.exported_names())


def test_status_strings_without_gpu():
    from seldon_b200 import _lib
    lib = _lib.load()
    assert lib.sb2_status_string(0) == b"ok"
    assert b"CSR" in lib.sb2_status_string(_lib.SB2_ERR_INVALID_CSR)
    assert lib.sb2_version() >= 10000
    assert lib.sb2_status_string(_lib.SB2_ERR_HOST) == b"host-side failure"


def test_wait_limit_setters_round_trip():
    """ms and us setters share one limit; values <= 0 leave it unchanged."""
    from seldon_b200 import _lib
    L = _lib.load()
    old = L.sb2_set_wait_limit_us(2500)
    try:
        assert L.sb2_set_wait_limit_us(0) == 2500
        assert L.sb2_set_wait_limit_ms(-1) == 3  # 2500 us, rounded up
        assert L.sb2_set_wait_limit_ms(7) == 3
        assert L.sb2_set_wait_limit_us(-5) == 7000
    finally:
        L.sb2_set_wait_limit_us(old)


_OOM_CHILD = r"""
import ctypes, re, resource, sys
import numpy as np
from seldon_b200 import _lib
lib = _lib.load()
n = 4_000_000
ptr = np.arange(n + 1, dtype=np.int32)
ind = np.arange(n, dtype=np.int32)
val = np.ones(n)
perm = np.arange(n, dtype=np.int32)
prm = _lib.IlutParams(0, 10, 0, 100, 1.0, 1e-3, 0.0)
h = ctypes.c_void_p()
vm = int(re.search(r"VmSize:\s+(\d+)", open("/proc/self/status").read()).group(1)) * 1024
resource.setrlimit(resource.RLIMIT_AS, (vm + (96 << 20), resource.RLIM_INFINITY))
p = lambda a: a.ctypes.data_as(ctypes.c_void_p)
st = lib.sb2_ilut_factor(n, p(ptr), p(ind), p(val), p(perm), ctypes.byref(prm), ctypes.byref(h))
print("status", st, h.value)
"""


def test_host_allocation_failure_is_a_status():
    """No C++ exception crosses the C ABI: a host allocation that fails
    inside an entry point (here the ILUT factorization of a 4M-row matrix
    under a 96 MB address-space allowance) returns SB2_ERR_NO_MEMORY and the
    caller's process goes on."""
    import subprocess
    import sys
    from seldon_b200 import _lib
    out = subprocess.run([sys.executable, "-c", _OOM_CHILD], cwd=ROOT, capture_output=True,
                         text=True, timeout=300)
    assert out.returncode == 0, out.stderr[-2000:]
    assert out.stdout.split() == ["status", str(_lib.SB2_ERR_NO_MEMORY), "None"], out.stdout


def test_iteration_loop_interface(capsys):
    """Iteration's loop interface for hand-written drivers (Iterative.cxx:
    236-354): First, Finished on a residual norm (with the reference's
    printed lines), Fail, ++ (as +=) and ErrorCode's rule."""
    from seldon_b200 import api
    it = api.Iteration(250, 1e-8)
    assert it.First() and it.ErrorCode() == 0 and it.GetTypeSolver() == 0
    it.SetSolver(3, 30, 1)
    assert (it.GetTypeSolver(), it.GetRestart()) == (3, 30)
    it.facteur_reste = 0.5
    assert not it.Finished(1.0)
    assert capsys.readouterr().out == "Residu at iteration number 0  0.5\n"
    it += 1
    assert not it.First()
    assert it.Finished(1e-8) and not it.Finished(2e-8)
    assert capsys.readouterr().out == ""          # print level 1: every 100th only
    it.ShowFullHistory()
    it.Finished(3e-8)
    assert capsys.readouterr().out == "Residu at iteration number 1  1.5e-08\n"
    it.Fail(3, "breakdown")
    assert it.ErrorCode() == 3
    c = it.copy()
    assert (c.GetNumberIteration(), c.GetFactor(), c.GetRestart()) == (0, 0.5, 30)
    it.SetNumberIteration(250)
    assert it.Finished(1.0) and it.ErrorCode() == -2   # max_iter outranks a failure


def test_element_lookup_rule():
    """RowSparse(i, j) and Print use the reference's lookup: the scan stops
    at the first column >= j, so with unsorted rows an entry after a larger
    column is not found, and a repeated column gives its first copy."""
    import numpy as np
    from seldon_b200.api import lookup
    ptr = np.array([0, 3, 3, 5])
    ind = np.array([2, 0, 1, 1, 1])
    val = np.array([5.0, 6.0, 7.0, 8.0, 9.0])
    assert lookup(ptr, ind, val, 0, 2) == 5.0
    assert lookup(ptr, ind, val, 0, 0) == 0.0   # stored after column 2: not reached
    assert lookup(ptr, ind, val, 0, 1) == 0.0
    assert lookup(ptr, ind, val, 1, 0) == 0.0   # empty row
    assert lookup(ptr, ind, val, 2, 1) == 8.0   # first of the repeated column
    rng = np.random.default_rng(3)
    for _ in range(200):                          # sorted, unique rows: the dense value
        n = int(rng.integers(1, 9))
        dense = np.where(rng.random((n, n)) < 0.4, rng.standard_normal((n, n)), 0.0)
        rows = [np.nonzero(dense[i])[0] for i in range(n)]
        p = np.concatenate([[0], np.cumsum([r.size for r in rows])])
        c = np.concatenate(rows) if p[-1] else np.zeros(0, dtype=int)
        v = dense[dense != 0]
        for i in range(n):
            for j in range(n):
                assert lookup(p, c, v, i, j) == dense[i, j]
        up = np.triu(dense)
        rows = [np.nonzero(up[i])[0] for i in range(n)]
        p = np.concatenate([[0], np.cumsum([r.size for r in rows])])
        c = np.concatenate(rows) if p[-1] else np.zeros(0, dtype=int)
        v = up[up != 0]
        for i in range(n):
            for j in range(n):
                assert lookup(p, c, v, i, j, True) == up[min(i, j), max(i, j)]


def test_preconditioner_handle_cache(monkeypatch):
    """The Python preconditioners create one library handle per (matrix,
    matrix handle, settings): repeated solves reuse it, a matrix whose handle
    was replaced (Clear) gets a new one, changed settings rebuild it and free
    the old one, and Clear / destruction free them all.  The library calls
    are replaced by a recorder, so no device is needed."""
    import numpy as np
    from seldon_b200 import api
    calls = {"create": 0, "destroy": 0}

    class Recorder:
        def _new(self, out, base):
            calls["create"] += 1
            ctypes.cast(out, ctypes.POINTER(ctypes.c_void_p))[0] = base + calls["create"]
            return 0

        def sb2_precond_create(self, A, kind, omega, nb, sym, out):
            return self._new(out, 1000)

        def sb2_precond_create_ilut(self, A, n, *rest):
            return self._new(rest[-1], 2000)

        def sb2_precond_destroy(self, h):
            calls["destroy"] += 1
            return 0

    class Matrix:
        symmetric = False
        m = 4

        def __init__(self, h):
            self.handle = ctypes.c_void_p(h)

    monkeypatch.setattr(api, "_L", Recorder())
    A = Matrix(77)
    J = api.JacobiPreconditioner()
    assert J.handle_for(A).value == J.handle_for(A).value and calls["create"] == 1
    A.handle = ctypes.c_void_p(78)
    J.handle_for(A)
    assert calls["create"] == 2
    S = api.SorPreconditioner()
    S.handle_for(A)
    S.SetParameterRelaxation(1.3)
    S.handle_for(A)
    assert (calls["create"], calls["destroy"]) == (4, 1)
    M = api.IlutPreconditioning()
    M.SetFactor(np.array([0, 1, 2, 3, 4]), np.arange(4), np.ones(4), np.arange(4))
    a, b, c = M.handle_for(A), M.handle_for(A), M.handle_for(None)
    assert a.value == b.value != c.value and calls["create"] == 6
    M.Clear()
    assert calls["destroy"] == 3
    del J, S
    import gc
    gc.collect()
    assert calls["destroy"] == 6


def test_graph_edges_checked_before_the_device():
    """GraphLaplacian refuses malformed or out-of-range edges on the host
    (the gradient kernel reads through them unchecked)."""
    from seldon_b200.autograd import GraphLaplacian
    for edges in ([[0, 3]], [[-1, 1]], [[0, 1, 2]]):
        with pytest.raises(ValueError):
            GraphLaplacian(3, edges, 0.1)
