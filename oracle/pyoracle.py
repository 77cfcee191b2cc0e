"""ctypes access to the checkers -- TEST INFRASTRUCTURE ONLY.

* ``Oracle``: the plain-C restatement (oracle/liboracle.so).
* ``Reference``: the reference itself (oracle/_ref/libseldon_ref.so, built
  from the Seldon headers by oracle/Makefile), present only where it was
  built; ``Reference.available()`` says so.

Only the tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
bench.py use this module; the product path never does.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libseldon_ref.so")
# the `which` numbers of orc_solve / ref_solve
_SOLVERS = {"cg": 0, "bicgstab": 1, "gmres": 2, "cgs": 3, "tfqmr": 4, "minres": 5, "gcr": 6,
            "bicgstabl": 7, "qcgs": 8, "bicg": 9, "cocg": 10, "cgne": 11,
            "bicgcr": 12, "lsqr": 13, "qmrsym": 14, "symmlq": 15}
REF_FAST_SO = os.path.join(HERE, "_ref", "libseldon_ref_fast.so")

_vp = ctypes.c_void_p
_i = ctypes.c_int
_d = ctypes.c_double


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


def _coo_args(row, col, val):
    return (np.ascontiguousarray(row, dtype=np.int32), np.ascontiguousarray(col, dtype=np.int32),
            np.ascontiguousarray(val, dtype=np.float64))


def _csr_args(ptr, ind, val):
    ptr = np.ascontiguousarray(ptr, dtype=np.int32)
    ind = np.ascontiguousarray(ind, dtype=np.int32)
    val = np.ascontiguousarray(val, dtype=np.float64)
    return ptr, ind, val


class _Base:
    def __init__(self, path):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} is missing: run `make -C oracle`")
        self.lib = ctypes.CDLL(path)


class Oracle(_Base):
    """The plain-C restatement of Seldon's path (seldon_oracle.c)."""

    def __init__(self, path=ORACLE_SO):
        super().__init__(path)
        L = self.lib
        L.orc_mltadd.argtypes = [_i, _i, _vp, _vp, _vp, _i, _i, _d, _vp, _d, _vp]
        L.orc_mltadd.restype = None
        L.orc_dot.argtypes = [_i, _vp, _vp]
        L.orc_dot.restype = _d
        L.orc_nrm2.argtypes = [_i, _vp]
        L.orc_nrm2.restype = _d
        L.orc_genrot.argtypes = [_vp, _vp, _vp, _vp]
        L.orc_genrot.restype = None
        L.orc_trsv_upper.argtypes = [_i, _vp, _i, _vp]
        L.orc_trsv_upper.restype = None
        L.orc_sor.argtypes = [_i, _vp, _vp, _vp, _i, _vp, _vp, _d, _i, _i]
        L.orc_sor.restype = None
        L.orc_solve.argtypes = [_i, _i, _i, _vp, _vp, _vp, _i, _i, _d, _i, _i, _vp, _vp,
                                _d, _i, _i, _i, _vp, _vp, _vp, _i, _vp]
        L.orc_solve.restype = _i
        L.orc_coo_sizes.argtypes = [_i, _vp, _vp, _i, _i, _i, _i, _vp, _vp, _vp]
        L.orc_coo_sizes.restype = _i
        L.orc_coo_to_csr.argtypes = [_i, _vp, _vp, _vp, _i, _i, _i, _vp, _vp, _vp]
        L.orc_coo_to_csr.restype = None
        L.orc_ilut_solve.argtypes = [_i, _vp, _vp, _vp, _i, _vp, _vp, _i, _vp, _vp]
        L.orc_ilut_solve.restype = None

    def ilut_solve(self, factor, r, sym=False, trans=False):
        """z = M^{-1} r (or M^{-T} r) with factor = (fptr, find, fval,
        perm_row, perm_col) as the reference returns it."""
        fp, fi, fv, pr, pc = (np.ascontiguousarray(a) for a in factor)
        r = np.ascontiguousarray(r, dtype=np.float64)
        z = np.zeros_like(r)
        self.lib.orc_ilut_solve(r.size, _p(fp.astype(np.int32)), _p(fi.astype(np.int32)),
                                _p(fv.astype(np.float64)), int(sym), _p(pr.astype(np.int32)),
                                _p(pc.astype(np.int32)), int(trans), _p(r), _p(z))
        return z

    def coo_to_csr(self, row, col, val, index=0, m_min=0, n_min=0, sym=False):
        """ConvertMatrix_from_Coordinates restated: (m, n, ptr, ind, val)."""
        row, col, val = _coo_args(row, col, val)
        m, n, nz = (ctypes.c_int() for _ in range(3))
        if self.lib.orc_coo_sizes(row.size, _p(row), _p(col), index, m_min, n_min, int(sym),
                                  ctypes.byref(m), ctypes.byref(n), ctypes.byref(nz)) != 0:
            raise ValueError("coordinate below the index base")
        ptr = np.zeros(m.value + 1, dtype=np.int32)
        ind = np.zeros(nz.value, dtype=np.int32)
        out = np.zeros(nz.value)
        self.lib.orc_coo_to_csr(row.size, _p(row), _p(col), _p(val), index, m.value, int(sym),
                                _p(ptr), _p(ind), _p(out))
        return m.value, n.value, ptr, ind, out

    def mltadd(self, m, n, ptr, ind, val, alpha, x, beta, y, sym=False, trans=False):
        """Returns a new y = beta*y + alpha*op(A)*x (MltAdd)."""
        ptr, ind, val = _csr_args(ptr, ind, val)
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.array(y, dtype=np.float64, copy=True)
        self.lib.orc_mltadd(m, n, _p(ptr), _p(ind), _p(val), int(sym), int(trans),
                            float(alpha), _p(x), float(beta), _p(y))
        return y

    def dot(self, x, y):
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.ascontiguousarray(y, dtype=np.float64)
        return self.lib.orc_dot(x.size, _p(x), _p(y))

    def nrm2(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        return self.lib.orc_nrm2(x.size, _p(x))

    def genrot(self, a, b):
        v = np.array([a, b, 0.0, 0.0])
        base = v.ctypes.data
        self.lib.orc_genrot(base, base + 8, base + 16, base + 24)
        return tuple(v)  # (r, z, c, s)

    def sor(self, ptr, ind, val, x, b, omega, it, type_ssor, sym=False):
        ptr, ind, val = _csr_args(ptr, ind, val)
        x = np.array(x, dtype=np.float64, copy=True)
        b = np.ascontiguousarray(b, dtype=np.float64)
        self.lib.orc_sor(ptr.size - 1, _p(ptr), _p(ind), _p(val), int(sym), _p(x), _p(b),
                         float(omega), int(it), int(type_ssor))
        return x

    def solve(self, which, ptr, ind, val, b, x0=None, sym=False, precond=0, omega=1.0,
              sor_iter=1, sor_sym=True, tol=1e-6, max_iter=100, restart=10,
              hist_cap=0):
        """which: 'cg' | 'bicgstab' | 'gmres' | 'cgs' | 'tfqmr' | 'minres' | 'gcr' |
        'bicgstabl' | 'qcgs' | 'bicg'.  precond: 0 identity, 1 Jacobi, 2 SOR.
        Returns (x, error_code, nb_iter, hist, hist_it)."""
        w = _SOLVERS[which]
        ptr, ind, val = _csr_args(ptr, ind, val)
        m = ptr.size - 1
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.zeros(m) if x0 is None else np.array(x0, dtype=np.float64, copy=True)
        nb = ctypes.c_int(0)
        hl = ctypes.c_int(0)
        hist = np.zeros(max(hist_cap, 1))
        hist_it = np.zeros(max(hist_cap, 1), dtype=np.int32)
        code = self.lib.orc_solve(
            w, m, ind.size, _p(ptr), _p(ind), _p(val), int(sym), int(precond), float(omega),
            int(sor_iter), int(sor_sym), _p(x), _p(b), float(tol), int(max_iter), int(restart),
            int(x0 is None), ctypes.byref(nb), _p(hist) if hist_cap else None,
            _p(hist_it) if hist_cap else None, int(hist_cap), ctypes.byref(hl))
        return x, code, nb.value, hist[:hl.value].copy(), hist_it[:hl.value].copy()


class Reference(_Base):
    """The reference compiled from its own headers (oracle/_ref)."""

    @staticmethod
    def available(path=REF_SO):
        return os.path.exists(path)

    def __init__(self, path=REF_SO):
        super().__init__(path)
        L = self.lib
        L.ref_mltadd.argtypes = [_i, _i, _i, _vp, _vp, _vp, _i, _i, _d, _vp, _d, _vp]
        L.ref_mltadd.restype = _i
        L.ref_sor.argtypes = [_i, _i, _vp, _vp, _vp, _i, _vp, _vp, _d, _i, _i]
        L.ref_sor.restype = _i
        L.ref_solve.argtypes = [_i, _i, _i, _vp, _vp, _vp, _i, _i, _d, _i, _i, _vp, _vp, _d,
                                _i, _i, _i, _i, _vp]
        L.ref_solve.restype = _i
        L.ref_dot.argtypes = [_i, _vp, _vp]
        L.ref_dot.restype = _d
        L.ref_norm2.argtypes = [_i, _vp]
        L.ref_norm2.restype = _d
        L.ref_genrot.argtypes = [_vp, _vp, _vp, _vp]
        L.ref_genrot.restype = None
        L.ref_write_csr.argtypes = [ctypes.c_char_p, _i, _i, _i, _vp, _vp, _vp, _i]
        L.ref_write_csr.restype = _i
        L.ref_read_csr_sizes.argtypes = [ctypes.c_char_p, _i, _vp, _vp, _vp]
        L.ref_read_csr_sizes.restype = _i
        L.ref_read_csr.argtypes = [ctypes.c_char_p, _i, _vp, _vp, _vp]
        L.ref_read_csr.restype = _i
        L.ref_write_vector.argtypes = [ctypes.c_char_p, _i, _vp, _i]
        L.ref_write_vector.restype = _i
        L.ref_coo_to_csr.argtypes = [_i, _vp, _vp, _vp, _i, _i, _i, _i, _i, _vp, _vp, _vp,
                                     _vp, _vp, _vp]
        L.ref_coo_to_csr.restype = _i
        L.ref_write_text.argtypes = [ctypes.c_char_p, _i, _i, _i, _vp, _vp, _vp, _i]
        L.ref_write_text.restype = _i
        L.ref_read_text_sizes.argtypes = [ctypes.c_char_p, _i, _vp, _vp, _vp]
        L.ref_read_text_sizes.restype = _i
        L.ref_read_text.argtypes = [ctypes.c_char_p, _i, _vp, _vp, _vp]
        L.ref_read_text.restype = _i
        L.ref_ilut_factor.argtypes = [_i, _i, _vp, _vp, _vp, _i, _vp, _i, _i, _i, _i, _d, _d, _d,
                                      _vp]
        L.ref_ilut_factor.restype = _i
        L.ref_ilut_get.argtypes = [_i, _vp, _vp, _vp, _vp, _vp]
        L.ref_ilut_get.restype = _i
        L.ref_ilut_solve.argtypes = [_i, _i, _vp, _vp]
        L.ref_ilut_solve.restype = _i
        L.ref_solve_ilut.argtypes = [_i, _i, _i, _vp, _vp, _vp, _i, _vp, _vp, _d, _i, _i, _i, _vp]
        L.ref_solve_ilut.restype = _i

    ILUT, ILU_D, ILUT_K, ILU_0, MILU_0, ILU_K = range(6)

    def write_hb(self, path, m, n, ptr, ind, val):
        """Seldon's WriteHarwellBoeing of a RowSparse matrix."""
        ptr, ind, val = _csr_args(ptr, ind, val)
        self.lib.ref_write_hb.argtypes = [ctypes.c_char_p, _i, _i, _i, _vp, _vp, _vp]
        self.lib.ref_write_hb(str(path).encode(), m, n, ind.size, _p(ptr), _p(ind), _p(val))

    def read_hb(self, path, cap_cols=1 << 20, cap_nnz=1 << 24):
        """Seldon's ReadHarwellBoeing into ColSparse: (m, n, colptr, rowind,
        val), or raises RuntimeError with Seldon's message."""
        L = self.lib
        L.ref_read_hb.argtypes = [ctypes.c_char_p, _vp, _vp, _vp, _i, _i, _vp, _vp, _vp,
                                  ctypes.c_char_p, _i]
        m, n, nz = (ctypes.c_int() for _ in range(3))
        cp = np.zeros(cap_cols + 1, dtype=np.int32)
        ri = np.zeros(cap_nnz, dtype=np.int32)
        v = np.zeros(cap_nnz)
        msg = ctypes.create_string_buffer(512)
        st = L.ref_read_hb(str(path).encode(), ctypes.byref(m), ctypes.byref(n), ctypes.byref(nz),
                           cap_cols, cap_nnz, _p(cp), _p(ri), _p(v), msg, 512)
        if st != 0:
            raise RuntimeError(msg.value.decode() or f"ref_read_hb status {st}")
        return m.value, n.value, cp[:n.value + 1].copy(), ri[:nz.value].copy(), v[:nz.value].copy()

    def ilut_factor(self, ptr, ind, val, sym=False, perm=None, type_ilu=0, fill_level=1000000,
                    additional_fill=1000000, mbloc=1000000, alpha=1.0, droptol=0.01,
                    permtol=0.1):
        """Seldon's IlutPreconditioning factorization (held for ilut_solve and
        solve_ilut): returns (fptr, find, fval, perm_row, perm_col)."""
        ptr, ind, val = _csr_args(ptr, ind, val)
        n = ptr.size - 1
        pm = None if perm is None else np.ascontiguousarray(perm, dtype=np.int32)
        nz = ctypes.c_int()
        self.lib.ref_ilut_factor(n, ind.size, _p(ptr), _p(ind), _p(val), int(sym), _p(pm),
                                 type_ilu, fill_level, additional_fill, mbloc, alpha, droptol,
                                 permtol, ctypes.byref(nz))
        fptr = np.zeros(n + 1, dtype=np.int32)
        find = np.zeros(max(nz.value, 1), dtype=np.int32)
        fval = np.zeros(max(nz.value, 1))
        pr = np.zeros(max(n, 1), dtype=np.int32)
        pc = np.zeros(max(n, 1), dtype=np.int32)
        self.lib.ref_ilut_get(n, _p(fptr), _p(find), _p(fval), _p(pr), _p(pc))
        return fptr, find[:nz.value], fval[:nz.value], pr[:n], pc[:n]

    def ilut_solve(self, r, trans=False):
        r = np.ascontiguousarray(r, dtype=np.float64)
        z = np.zeros_like(r)
        self.lib.ref_ilut_solve(int(trans), r.size, _p(r), _p(z))
        return z

    def solve_ilut(self, which, ptr, ind, val, b, sym=False, x0=None, tol=1e-10,
                   max_iter=400, restart=10):
        """Cg/BiCgStab/Gmres preconditioned by the held ILUT factor."""
        ptr, ind, val = _csr_args(ptr, ind, val)
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.zeros_like(b) if x0 is None else np.array(x0, dtype=np.float64)
        nb = ctypes.c_int()
        w = _SOLVERS[which]
        code = self.lib.ref_solve_ilut(w, ptr.size - 1, ind.size, _p(ptr), _p(ind), _p(val),
                                       int(sym), _p(x), _p(b), tol, max_iter, restart,
                                       int(x0 is None), ctypes.byref(nb))
        return x, code, nb.value

    def write_text(self, path, m, n, ptr, ind, val, sym=False):
        ptr, ind, val = _csr_args(ptr, ind, val)
        self.lib.ref_write_text(str(path).encode(), m, n, ind.size, _p(ptr), _p(ind), _p(val),
                                int(sym))

    def read_text(self, path, sym=False):
        m, n, nz = (ctypes.c_int() for _ in range(3))
        self.lib.ref_read_text_sizes(str(path).encode(), int(sym), ctypes.byref(m),
                                     ctypes.byref(n), ctypes.byref(nz))
        ptr = np.zeros(m.value + 1, dtype=np.int32)
        ind = np.zeros(max(nz.value, 1), dtype=np.int32)
        val = np.zeros(max(nz.value, 1))
        self.lib.ref_read_text(str(path).encode(), int(sym), _p(ptr), _p(ind), _p(val))
        return m.value, n.value, ptr, ind[:nz.value], val[:nz.value]

    def coo_to_csr(self, row, col, val, index=0, m_min=0, n_min=0, sym=False):
        """Seldon's own ConvertMatrix_from_Coordinates: (m, n, ptr, ind, val)."""
        row, col, val = _coo_args(row, col, val)
        cap = max(m_min, n_min, 1, int(row.max(initial=0)) + 2, int(col.max(initial=0)) + 2)
        ptr = np.zeros(cap + 1, dtype=np.int32)
        ind = np.zeros(max(row.size, 1), dtype=np.int32)
        out = np.zeros(max(row.size, 1))
        m, n, nz = (ctypes.c_int() for _ in range(3))
        if self.lib.ref_coo_to_csr(row.size, _p(row), _p(col), _p(val), index, m_min, n_min,
                                   int(sym), cap, ctypes.byref(m), ctypes.byref(n),
                                   ctypes.byref(nz), _p(ptr), _p(ind), _p(out)) != 0:
            raise RuntimeError("ref_coo_to_csr: result larger than the buffers")
        return (m.value, n.value, ptr[:m.value + 1].copy(), ind[:nz.value].copy(),
                out[:nz.value].copy())

    def write_csr(self, path, m, n, ptr, ind, val, sym=False):
        ptr, ind, val = _csr_args(ptr, ind, val)
        self.lib.ref_write_csr(str(path).encode(), m, n, ind.size, _p(ptr), _p(ind), _p(val),
                               int(sym))

    def read_csr(self, path, sym=False):
        m, n, nz = (ctypes.c_int() for _ in range(3))
        self.lib.ref_read_csr_sizes(str(path).encode(), int(sym), ctypes.byref(m),
                                    ctypes.byref(n), ctypes.byref(nz))
        ptr = np.zeros(m.value + 1, dtype=np.int32)
        ind = np.zeros(nz.value, dtype=np.int32)
        val = np.zeros(nz.value)
        self.lib.ref_read_csr(str(path).encode(), int(sym), _p(ptr), _p(ind), _p(val))
        return m.value, n.value, ptr, ind, val

    def write_vector(self, path, x, with_size=True):
        x = np.ascontiguousarray(x, dtype=np.float64)
        self.lib.ref_write_vector(str(path).encode(), x.size, _p(x), int(with_size))

    def mltadd(self, m, n, ptr, ind, val, alpha, x, beta, y, sym=False, trans=False):
        ptr, ind, val = _csr_args(ptr, ind, val)
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.array(y, dtype=np.float64, copy=True)
        self.lib.ref_mltadd(m, n, ind.size, _p(ptr), _p(ind), _p(val), int(sym), int(trans),
                            float(alpha), _p(x), float(beta), _p(y))
        return y

    def dot(self, x, y):
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.ascontiguousarray(y, dtype=np.float64)
        return self.lib.ref_dot(x.size, _p(x), _p(y))

    def nrm2(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        return self.lib.ref_norm2(x.size, _p(x))

    def genrot(self, a, b):
        v = np.array([a, b, 0.0, 0.0])
        base = v.ctypes.data
        self.lib.ref_genrot(base, base + 8, base + 16, base + 24)
        return tuple(v)

    def sor(self, ptr, ind, val, x, b, omega, it, type_ssor, sym=False):
        ptr, ind, val = _csr_args(ptr, ind, val)
        x = np.array(x, dtype=np.float64, copy=True)
        b = np.ascontiguousarray(b, dtype=np.float64)
        self.lib.ref_sor(ptr.size - 1, ind.size, _p(ptr), _p(ind), _p(val), int(sym), _p(x),
                         _p(b), float(omega), int(it), int(type_ssor))
        return x

    def solve(self, which, ptr, ind, val, b, x0=None, sym=False, precond=0, omega=1.0,
              sor_iter=1, sor_sym=True, tol=1e-6, max_iter=100, restart=10,
              print_level=0):
        """Returns (x, error_code, nb_iter)."""
        w = _SOLVERS[which]
        ptr, ind, val = _csr_args(ptr, ind, val)
        m = ptr.size - 1
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.zeros(m) if x0 is None else np.array(x0, dtype=np.float64, copy=True)
        nb = ctypes.c_int(0)
        code = self.lib.ref_solve(w, m, ind.size, _p(ptr), _p(ind), _p(val), int(sym),
                                  int(precond), float(omega), int(sor_iter), int(sor_sym),
                                  _p(x), _p(b), float(tol), int(max_iter), int(restart),
                                  int(x0 is None), int(print_level), ctypes.byref(nb))
        return x, code, nb.value
