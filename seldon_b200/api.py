"""Python mirror of Seldon's interface for the sparse Krylov path.

Names, argument order and error behaviour follow the reference's free
functions, so code written against Seldon reads the same here:

    A = RowSparse(m, n, ptr, ind, val)            # Matrix<double, General, RowSparse>
    S = RowSymSparse(m, ptr, ind, val)            # Matrix<double, Symmetric, RowSymSparse>
    MltAdd(alpha, A, X, beta, Y)                  # Functions_MatVect.cxx:398-431
    Mlt(A, X, Y); Mlt(alpha, X)                   # :72-130; Functions_Vector.cxx:69-74
    DotProd(X, Y); Norm2(X); Add(alpha, X, Y); Copy(X, Y)
    it = Iteration(max_iter, tol); Cg(A, x, b, M, it)   # Cg.cxx:45-116

Vectors are device tensors (torch, float64, contiguous) -- torch is used only
for device memory and streams; every operation runs in libseldon_b200.so.
"""
import ctypes

from . import _lib
from ._lib import IrParams, IrResult, IterParams, IterResult, check

_L = _lib.load()


def _stream(stream=None):
    if stream is not None:
        return ctypes.c_void_p(int(stream))
    import torch
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _dev_ptr(t, n=None, name="vector"):
    import torch
    if not isinstance(t, torch.Tensor) or not t.is_cuda or t.dtype != torch.float64:
        raise TypeError(f"{name}: expected a CUDA float64 tensor")
    if not t.is_contiguous():
        raise ValueError(f"{name}: expected a contiguous tensor")
    if n is not None and t.numel() != n:
        raise ValueError(f"{name}: length {t.numel()} != {n} (WrongDim)")
    return ctypes.c_void_p(t.data_ptr())


def _np_ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


class _DeviceArray:
    """A device array allocated by the library (released with
    sb2_device_free when the last tensor viewing it goes away)."""

    def __init__(self, ptr, n, typestr):
        self._p = ptr
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": typestr,
                                         "data": (ptr or 0, False), "version": 2,
                                         "strides": None}

    def __del__(self):
        if self._p:
            _L.sb2_device_free(ctypes.c_void_p(self._p))
            self._p = None


def _as_tensor(ptr, n, typestr, dtype):
    import torch
    if n == 0:
        if ptr:
            _L.sb2_device_free(ctypes.c_void_p(ptr))
        return torch.zeros(0, dtype=dtype, device="cuda")
    return torch.as_tensor(_DeviceArray(ptr, n, typestr), device="cuda")


def _int_dev_ptr(t, name):
    import torch
    if not isinstance(t, torch.Tensor) or not t.is_cuda or t.dtype != torch.int32:
        raise TypeError(f"{name}: expected a CUDA int32 tensor")
    if not t.is_contiguous():
        raise ValueError(f"{name}: expected a contiguous tensor")
    return ctypes.c_void_p(t.data_ptr())


def ConvertMatrix_from_Coordinates(IndRow, IndCol, Val, index=0, m=0, n=0, symmetric=False,
                                   stream=None):
    """Assemble CSR arrays on the device from coordinate triplets
    (Matrix_Conversions.cxx:1291-1334 RowSparse, 1397-1467 RowSymSparse).

    IndRow/IndCol: CUDA int32 tensors, Val: CUDA float64 tensor, indices from
    `index`; (m, n) is the target matrix's current size.  Returns
    (m, n, ptr, ind, val) with device tensors in Seldon's stable (row, column)
    order, duplicates kept.  symmetric=True drops the entries below the
    diagonal (RowSymSparse)."""
    nnz = IndRow.numel()
    if IndCol.numel() != nnz or Val.numel() != nnz:
        raise ValueError("WrongDim: IndRow, IndCol and Val must have the same length")
    rp = _int_dev_ptr(IndRow, "IndRow") if nnz else None
    cp = _int_dev_ptr(IndCol, "IndCol") if nnz else None
    vp = _dev_ptr(Val, nnz, "Val") if nnz else None
    mo, no, zo = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    dp, di, dv = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p()
    check(_L.sb2_coo_to_csr(int(nnz), rp, cp, vp, int(index), int(m), int(n), int(symmetric),
                            _stream(stream), ctypes.byref(mo), ctypes.byref(no),
                            ctypes.byref(zo), ctypes.byref(dp), ctypes.byref(di),
                            ctypes.byref(dv)), "sb2_coo_to_csr")
    import torch
    ptr = _as_tensor(dp.value, mo.value + 1, "<i4", torch.int32)
    ind = _as_tensor(di.value, zo.value, "<i4", torch.int32)
    val = _as_tensor(dv.value, zo.value, "<f8", torch.float64)
    return mo.value, no.value, ptr, ind, val


def lookup(ptr, ind, val, i, j, symmetric=False):
    """The reference's element lookup on CSR arrays: scan row i while k < b-1
    and ind[k] < j, then test ind[k] == j (Matrix_Sparse.cxx:1054-1083); the
    symmetric storage looks up (min(i, j), max(i, j))."""
    if symmetric and i > j:
        i, j = j, i
    a, b = int(ptr[i]), int(ptr[i + 1])
    if a == b:
        return 0.0
    k = a
    while k < b - 1 and ind[k] < j:
        k += 1
    return float(val[k]) if ind[k] == j else 0.0


class RowSparse:
    """Matrix<double, General, RowSparse> held on the device.

    ptr/ind/val are host arrays in Seldon's layout (ptr_, ind_, data_); they
    are copied, the caller keeps them."""

    symmetric = False

    def __init__(self, m, n, ptr, ind, val, validate=True):
        import numpy as np
        if hasattr(ptr, "is_cuda") and ptr.is_cuda:  # device arrays (e.g. assembled)
            nz = int(ind.numel())
            if ptr.numel() != m + 1 or val.numel() != nz:
                raise ValueError("WrongDim: ptr must hold m+1 entries and ind/val nnz entries")
            args = (_int_dev_ptr(ptr, "ptr"), _int_dev_ptr(ind, "ind") if nz else None,
                    _dev_ptr(val, nz, "val") if nz else None)
        else:
            ptr = np.ascontiguousarray(ptr, dtype=np.int32)
            ind = np.ascontiguousarray(ind, dtype=np.int32)
            val = np.ascontiguousarray(val, dtype=np.float64)
            if ptr.size != m + 1 or ind.size != val.size:
                raise ValueError("WrongDim: ptr must hold m+1 entries and ind/val nnz entries")
            nz = int(ind.size)
            args = (_np_ptr(ptr), _np_ptr(ind), _np_ptr(val))
        h = ctypes.c_void_p()
        st = _L.sb2_csr_create(int(m), int(n), nz, *args, int(self.symmetric), int(validate),
                               ctypes.byref(h))
        check(st, "sb2_csr_create")
        self._h = h
        self.m, self.n = int(m), int(n)
        self.nnz_stored = nz
        full = ctypes.c_int()
        _L.sb2_csr_info(h, None, None, None, ctypes.byref(full))
        self.nnz_full = full.value

    @property
    def handle(self):
        return self._h

    def GetM(self):
        return self.m

    def GetN(self):
        return self.n

    def GetNonZeros(self):
        return self.nnz_stored

    def GetDataSize(self):
        return self.nnz_stored

    def GetPtrSize(self):
        return self.m + 1

    def GetIndSize(self):
        return self.nnz_stored

    def __call__(self, i, j):
        """Element (i, j) by the reference's lookup (Matrix_Sparse.cxx:
        1054-1083; RowSymSparse reads (min, max), Matrix_SymSparse.cxx:
        1013-1053).  Each call downloads the matrix: for inspection."""
        if not (0 <= i < self.m and 0 <= j < self.n):
            raise IndexError("WrongRow/WrongCol: index out of range")
        return lookup(*self.download(), i, j, self.symmetric)

    def Print(self):
        """The dense matrix, row by row, tab-separated (Matrix_Sparse::Print,
        Matrix_Sparse.cxx:1491-1499), from one download."""
        ptr, ind, val = self.download()
        for i in range(self.m):
            print("".join(f"{lookup(ptr, ind, val, i, j, self.symmetric):g}\t"
                          for j in range(self.n)))

    def download(self):
        """The stored arrays (ptr, ind, val) copied back to the host."""
        import numpy as np
        ptr = np.zeros(self.m + 1, dtype=np.int32)
        ind = np.zeros(self.nnz_stored, dtype=np.int32)
        val = np.zeros(self.nnz_stored)
        check(_L.sb2_csr_download(self._h, _np_ptr(ptr), _np_ptr(ind), _np_ptr(val)),
              "sb2_csr_download")
        return ptr, ind, val

    def Write(self, path):
        """Save in Seldon's binary format (Matrix_Sparse::Write)."""
        from seldon_b200 import io
        io.write_csr(path, self.m, self.m if self.symmetric else self.n, *self.download())

    @classmethod
    def Read(cls, path, validate=True):
        """Load a file in Seldon's binary format (Matrix_Sparse::Read)."""
        from seldon_b200 import io
        m, n, ptr, ind, val = io.read_csr(path)
        if cls.symmetric:
            return cls(m, ptr, ind, val, validate)
        return cls(m, n, ptr, ind, val, validate)

    def WriteText(self, path):
        """Save as "row column value" lines (Matrix_Sparse::WriteText)."""
        from seldon_b200 import io
        io.write_text(path, *self.download(), sym=self.symmetric)

    @classmethod
    def ReadText(cls, path, validate=True):
        """Load "row column value" lines (Matrix_Sparse::ReadText): the
        triplets are parsed on the host and assembled on the device."""
        import torch
        from seldon_b200 import io
        r, c, v = io.read_text(path)
        if r.size == 0:  # ReadCoordinateMatrix leaves the cleared 0 x 0 matrix
            if cls.symmetric:
                return cls(0, [0], [], [], validate)
            return cls(0, 0, [0], [], [], validate)
        dev = [torch.as_tensor(a, device="cuda") for a in (r, c, v)]
        return cls.from_coordinates(*dev, index=1, validate=validate)

    def WriteHarwellBoeing(self, path):
        """WriteHarwellBoeing (IOMatrixMarket.cxx:394-511): the file
        Seldon's writer produces for this matrix."""
        if self.symmetric:
            raise NotImplementedError("Harwell-Boeing files of RowSparse matrices only")
        from seldon_b200 import io
        io.write_harwell_boeing(path, self.m, self.n, *self.download())

    @classmethod
    def ReadHarwellBoeing(cls, path, validate=True):
        """ReadHarwellBoeing (IOMatrixMarket.cxx:45-329): the file's
        compressed columns, assembled into rows on the device."""
        if cls.symmetric:
            raise NotImplementedError("the reference reads unsymmetric Harwell-Boeing files only")
        import numpy as np
        import torch
        from seldon_b200 import io
        m, n, colptr, rowind, val = io.read_harwell_boeing(path)
        cols = np.repeat(np.arange(n, dtype=np.int32), np.diff(colptr))
        if rowind.size == 0:
            return cls(m, n, np.zeros(m + 1, dtype=np.int32), [], [], validate)
        dev = [torch.as_tensor(a, device="cuda") for a in (rowind, cols, val)]
        return cls.from_coordinates(*dev, index=0, m=m, n=n, validate=validate)

    @classmethod
    def from_coordinates(cls, IndRow, IndCol, Val, index=0, m=0, n=0, validate=True):
        """Matrix built from coordinate triplets on the device, as
        ConvertMatrix_from_Coordinates fills an m x n matrix."""
        m, n, ptr, ind, val = ConvertMatrix_from_Coordinates(
            IndRow, IndCol, Val, index, m, n, cls.symmetric)
        if cls.symmetric:
            return cls(m, ptr, ind, val, validate)
        return cls(m, n, ptr, ind, val, validate)

    def close(self):
        if getattr(self, "_h", None):
            _L.sb2_csr_destroy(self._h)
            self._h = None

    def Clear(self):
        """Matrix_Sparse::Clear (Matrix_Sparse.cxx:278-281): the device
        arrays are released and the matrix becomes 0 x 0."""
        import numpy as np
        h = ctypes.c_void_p()
        check(_L.sb2_csr_create(0, 0, 0, _np_ptr(np.zeros(1, dtype=np.int32)), None, None,
                                int(self.symmetric), 1, ctypes.byref(h)), "sb2_csr_create")
        self.close()
        self._h = h
        self.m = self.n = self.nnz_stored = self.nnz_full = 0

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class RowSymSparse(RowSparse):
    """Matrix<double, Symmetric, RowSymSparse>: only the upper triangle
    (diagonal included) is given (Matrix_SymSparse.cxx:1031-1032)."""

    symmetric = True

    def __init__(self, m, ptr, ind, val, validate=True):
        super().__init__(m, m, ptr, ind, val, validate)


SeldonNoTrans = 0
SeldonTrans = 1


def MltAdd(alpha, A, X, beta, Y, trans=SeldonNoTrans, stream=None):
    """Y = beta*Y + alpha*op(A)*X (Y scaled by beta even when beta == 0)."""
    nx, ny = (A.m, A.n) if trans else (A.n, A.m)
    check(_L.sb2_spmv(A.handle, int(trans), float(alpha), _dev_ptr(X, nx, "X"), float(beta),
                      _dev_ptr(Y, ny, "Y"), _stream(stream)), "MltAdd")


def Mlt(*args, trans=SeldonNoTrans, stream=None):
    """Mlt(A, X, Y): Y = A*X;  Mlt(alpha, A, X, Y): Y = alpha*A*X;
    Mlt(alpha, X): X *= alpha."""
    if len(args) == 2:
        alpha, X = args
        check(_L.sb2_scal(X.numel(), float(alpha), _dev_ptr(X), _stream(stream)), "Mlt")
        return
    if len(args) == 3:
        alpha, (A, X, Y) = 1.0, args
    else:
        alpha, A, X, Y = args
    nx, ny = (A.m, A.n) if trans else (A.n, A.m)
    check(_L.sb2_mlt(A.handle, int(trans), float(alpha), _dev_ptr(X, nx, "X"),
                     _dev_ptr(Y, ny, "Y"), _stream(stream)), "Mlt")


def MltHostBatch(A, X, Y, alpha=1.0, trans=SeldonNoTrans, stream=None):
    """Y[i] = alpha*op(A)*X[i] for host arrays X (count x cols of op(A)) and
    Y (count x rows), C-contiguous float64 (numpy arrays or CPU tensors;
    pinned memory lets the copies overlap the products).  Each Y[i] is the
    same bits as Mlt on X[i]."""
    import numpy as np
    nx, ny = (A.m, A.n) if trans else (A.n, A.m)

    def host_ptr(a, cols, name):
        if hasattr(a, "data_ptr"):
            if a.is_cuda or a.dtype.itemsize != 8 or not a.is_contiguous():
                raise ValueError(f"{name}: a contiguous CPU float64 tensor is required")
            count = a.numel() // max(cols, 1) if cols else a.shape[0]
            return ctypes.c_void_p(a.data_ptr()), a.numel(), count
        if not (isinstance(a, np.ndarray) and a.dtype == np.float64 and a.flags.c_contiguous):
            raise ValueError(f"{name}: a C-contiguous float64 array is required")
        count = a.size // max(cols, 1) if cols else a.shape[0]
        return ctypes.c_void_p(a.ctypes.data), a.size, count
    px, sx, count = host_ptr(X, nx, "X")
    py, sy, _ = host_ptr(Y, ny, "Y")
    if sx != count * nx or sy != count * ny:
        raise ValueError("X and Y must hold the same number of vectors of op(A)'s sizes")
    check(_L.sb2_mlt_host_batch(A.handle, int(trans), float(alpha), count, px, py,
                                _stream(stream)), "MltHostBatch")


def DotProd(X, Y, stream=None):
    out = ctypes.c_double()
    check(_L.sb2_dot(X.numel(), _dev_ptr(X), _dev_ptr(Y, X.numel(), "Y"), ctypes.byref(out),
                     _stream(stream)), "DotProd")
    return out.value


DotProdConj = DotProd


def Norm2(X, stream=None):
    out = ctypes.c_double()
    check(_L.sb2_nrm2(X.numel(), _dev_ptr(X), ctypes.byref(out), _stream(stream)), "Norm2")
    return out.value


def Add(alpha, X, Y, stream=None):
    """Y += alpha*X (no-op when alpha == 0)."""
    check(_L.sb2_axpy(X.numel(), float(alpha), _dev_ptr(X), _dev_ptr(Y, X.numel(), "Y"),
                      _stream(stream)), "Add")


def Copy(X, Y, stream=None):
    check(_L.sb2_copy(X.numel(), _dev_ptr(X), _dev_ptr(Y, X.numel(), "Y"), _stream(stream)),
          "Copy")


def Fill(X, value, stream=None):
    check(_L.sb2_fill(X.numel(), float(value), _dev_ptr(X), _stream(stream)), "Fill")


# ------------------------------------------------------------------ preconditioners

class Preconditioner_Base:
    """Identity preconditioner (Iterative.cxx:50-77)."""

    kind = _lib.PRECOND_IDENTITY

    def handle_for(self, A):
        return None

    def Solve(self, A, r, z, stream=None):
        """z = r (Copy)."""
        Copy(r, z, stream=stream)

    def TransSolve(self, A, r, z, stream=None):
        Copy(r, z, stream=stream)


class _DevicePrecond:
    kind = None

    def __init__(self):
        self._cache = {}

    def _params(self):
        return 1.0, 1, 1

    def handle_for(self, A):
        # keyed on the matrix object and its current library handle (Clear
        # replaces the handle)
        key = (id(A), getattr(A.handle, "value", None))
        ent = self._cache.get(key)
        if ent is None or ent[0] is not A or ent[2] != self._params():
            omega, nb, sym = self._params()
            h = ctypes.c_void_p()
            check(_L.sb2_precond_create(A.handle, self.kind, float(omega), int(nb), int(sym),
                                        ctypes.byref(h)), "sb2_precond_create")
            if ent is not None:
                _L.sb2_precond_destroy(ent[1])
            ent = (A, h, self._params())
            self._cache[key] = ent
        return ent[1]

    def Solve(self, A, r, z, stream=None):
        check(_L.sb2_precond_solve(self.handle_for(A), _dev_ptr(r, A.m, "r"),
                                   _dev_ptr(z, A.m, "z"), _stream(stream)), "Solve")

    def TransSolve(self, A, r, z, stream=None):
        check(_L.sb2_precond_trans_solve(self.handle_for(A), _dev_ptr(r, A.m, "r"),
                                         _dev_ptr(z, A.m, "z"), _stream(stream)), "TransSolve")

    def __del__(self):
        try:
            for _, h, _p in self._cache.values():
                _L.sb2_precond_destroy(h)
        except Exception:
            pass


class JacobiPreconditioner(_DevicePrecond):
    """z_i = r_i / A(i,i).  The reference has no Jacobi preconditioner; this
    one has the shape of Preconditioner_Base (Iterative.hxx:24-39)."""

    kind = _lib.PRECOND_JACOBI


class SorPreconditioner(_DevicePrecond):
    """SorPreconditioner<double> (Precond_Ssor.cxx:24-90): omega 1, one
    sweep, symmetric by default."""

    kind = _lib.PRECOND_SOR

    def __init__(self):
        super().__init__()
        self.omega, self.nb_iter, self.symmetric = 1.0, 1, True

    def InitSymmetricPreconditioning(self):
        self.symmetric = True

    def InitUnSymmetricPreconditioning(self):
        self.symmetric = False

    def SetParameterRelaxation(self, omega):
        self.omega = float(omega)

    def SetNumberIterations(self, n):
        self.nb_iter = int(n)

    def _params(self):
        return self.omega, self.nb_iter, int(self.symmetric)


class IlutPreconditioning(_DevicePrecond):
    """IlutPreconditioning's Solve / TransSolve (IlutPreconditioning.cxx:
    329-374) on the device, from a factor computed on the host by Seldon's
    GetIlut (FactorizeMatrix / FactorizeSymMatrix).  SetFactor takes the
    factor's rows in stored order as flat CSR arrays and the permutations;
    the sweeps reproduce SolveLU bit for bit."""

    kind = _lib.PRECOND_ILUT

    def __init__(self):
        super().__init__()
        self._factor = None
        self._device_handle = None
        self._serial = 0
        # IlutPreconditioning's defaults (IlutPreconditioning.cxx:27-40)
        self.type_ilu = self.ILUT
        self.fill_level = 1000000
        self.additional_fill = 1000000
        self.mbloc = 1000000
        self.alpha = 1.0
        self.droptol = 0.01
        self.permtol = 0.1
        self.symmetric_algorithm = False
        self.print_level = 0

    def Clear(self):
        """Releases the factor and its device sweeps (IlutPreconditioning.cxx:
        43-50); the settings stay."""
        for _, h, _s in self._cache.values():
            _L.sb2_precond_destroy(h)
        if self._device_handle is not None:
            _L.sb2_precond_destroy(self._device_handle)
        self._cache = {}
        self._device_handle = None
        self._factor = None
        self._serial += 1

    def SetSymmetricAlgorithm(self):
        self.symmetric_algorithm = True

    def SetUnsymmetricAlgorithm(self):
        self.symmetric_algorithm = False

    def SetFactorisationType(self, t):
        self.type_ilu = int(t)

    def GetFactorisationType(self):
        return self.type_ilu

    def SetFillLevel(self, k):
        self.fill_level = int(k)

    def SetAdditionalFillNumber(self, k):
        self.additional_fill = int(k)

    def SetPivotBlockInteger(self, k):
        self.mbloc = int(k)

    def SetDiagonalCoefficient(self, a):
        self.alpha = float(a)

    def SetDroppingThreshold(self, t):
        self.droptol = float(t)

    def SetPivotThreshold(self, t):
        self.permtol = float(t)

    def SetPrintLevel(self, k):
        """Kept for the interface; the factorization prints nothing."""
        self.print_level = int(k)

    def GetFillLevel(self):
        return self.fill_level

    def GetAdditionalFillNumber(self):
        return self.additional_fill

    def GetPrintLevel(self):
        return self.print_level

    def GetPivotBlockInteger(self):
        return self.mbloc

    def GetDroppingThreshold(self):
        return self.droptol

    def GetDiagonalCoefficient(self):
        return self.alpha

    def GetPivotThreshold(self):
        return self.permtol

    def factor_host(self, n, ptr, ind, val, perm=None, symmetric=False):
        """The ILUT / ILU_D / ILUT_K factor of host CSR arrays, computed on
        the host in the reference's order (sb2_ilut_factor, or with
        `symmetric` sb2_ilut_factor_sym on the upper triangle): (fptr, find,
        fval, perm_row, perm_col)."""
        import numpy as np
        ptr = np.ascontiguousarray(ptr, dtype=np.int32)
        ind = np.ascontiguousarray(ind, dtype=np.int32)
        val = np.ascontiguousarray(val, dtype=np.float64)
        perm = (np.arange(n, dtype=np.int32) if perm is None
                else np.ascontiguousarray(perm, dtype=np.int32))
        types = {self.ILUT: 0, self.ILU_D: 1, self.ILUT_K: 2}
        if self.type_ilu not in types:
            raise NotImplementedError("host factorization of ILUT, ILU_D and ILUT_K")
        prm = _lib.IlutParams(types[self.type_ilu], self.fill_level, self.additional_fill,
                              self.mbloc, self.alpha, self.droptol, self.permtol)
        h = ctypes.c_void_p()
        fn = _L.sb2_ilut_factor_sym if symmetric else _L.sb2_ilut_factor
        check(fn(int(n), _np_ptr(ptr), _np_ptr(ind), _np_ptr(val), _np_ptr(perm),
                 ctypes.byref(prm), ctypes.byref(h)), "sb2_ilut_factor")
        try:
            nn, nz = ctypes.c_int(), ctypes.c_int()
            _L.sb2_ilut_size(h, ctypes.byref(nn), ctypes.byref(nz))
            fptr = np.zeros(n + 1, dtype=np.int32)
            find = np.zeros(max(nz.value, 1), dtype=np.int32)
            fval = np.zeros(max(nz.value, 1))
            prow = np.zeros(max(n, 1), dtype=np.int32)
            pcol = np.zeros(max(n, 1), dtype=np.int32)
            _L.sb2_ilut_arrays(h, _np_ptr(fptr), _np_ptr(find), _np_ptr(fval), _np_ptr(prow),
                               _np_ptr(pcol))
        finally:
            _L.sb2_ilut_destroy(h)
        return fptr, find[:nz.value], fval[:nz.value], prow[:n], pcol[:n]

    def SetFactor(self, fptr, find, fval, perm_row, perm_col=None, symmetric=False):
        import numpy as np
        fptr = np.ascontiguousarray(fptr, dtype=np.int32)
        n = fptr.size - 1
        find = np.ascontiguousarray(find, dtype=np.int32)
        fval = np.ascontiguousarray(fval, dtype=np.float64)
        prow = np.ascontiguousarray(perm_row, dtype=np.int32)
        pcol = prow if perm_col is None else np.ascontiguousarray(perm_col, dtype=np.int32)
        if find.size != fval.size or find.size < fptr[-1] or prow.size != n or pcol.size != n:
            raise ValueError("WrongDim: factor arrays and permutations do not match")
        self._factor = (n, fptr, find, fval, prow, pcol, bool(symmetric))
        self._serial += 1

    ILUT, ILU_D, ILUT_K, ILU_0, MILU_0, ILU_K = range(6)

    @staticmethod
    def _factorize_args(args, perm):
        """(A, perm, keep_matrix) from FactorizeMatrix(A, perm=None), which
        keeps A, or from the reference's FactorizeMatrix(perm, A,
        keep_matrix=False), which clears A afterwards unless keep_matrix."""
        if len(args) == 1:
            return args[0], perm, True
        if len(args) in (2, 3) and perm is None:
            return args[1], args[0], bool(args[2]) if len(args) == 3 else False
        raise TypeError("FactorizeMatrix(A, perm=None) or FactorizeMatrix(perm, A[, keep_matrix])")

    def FactorizeSymMatrix(self, *args, perm=None, stream=None):
        """The symmetric algorithm on a RowSymSparse matrix, whatever
        SetSymmetricAlgorithm says (IlutPreconditioning.cxx:216-263)."""
        A, perm, keep = self._factorize_args(args, perm)
        if not A.symmetric:
            raise NotImplementedError("FactorizeSymMatrix takes a RowSymSparse matrix here")
        self._factorize(A, perm, keep, stream)

    def FactorizeUnsymMatrix(self, *args, perm=None, stream=None):
        """The unsymmetric algorithm on a RowSparse matrix, whatever
        SetSymmetricAlgorithm says (IlutPreconditioning.cxx:266-323)."""
        A, perm, keep = self._factorize_args(args, perm)
        if A.symmetric:
            # the reference's unsymmetric algorithm on symmetric storage
            # does not compile
            raise NotImplementedError("FactorizeUnsymMatrix takes a RowSparse matrix")
        self._factorize(A, perm, keep, stream)

    def FactorizeMatrix(self, *args, perm=None, stream=None):
        """FactorizeMatrix (IlutPreconditioning.cxx:186-213), called as
        FactorizeMatrix(A, perm=None) or as the reference's
        FactorizeMatrix(perm, A, keep_matrix=False).  ILU_0 / MILU_0
        (identity ordering) are factored on the device, as GetIlu0 / GetMilu0
        do; ILUT, ILU_D and ILUT_K on the host in GetIlut's order, with the
        unsymmetric algorithm on RowSparse and the symmetric one on
        RowSymSparse.  ILU_K comes from Seldon through SetFactor."""
        A, perm, keep = self._factorize_args(args, perm)
        if A.symmetric != self.symmetric_algorithm:
            # the reference factors symmetric storage with the symmetric
            # algorithm only (its other path does not compile) and aborts on
            # the symmetric algorithm with general storage
            raise NotImplementedError(
                "RowSymSparse takes SetSymmetricAlgorithm(), RowSparse the unsymmetric one")
        self._factorize(A, perm, keep, stream)

    def _factorize(self, A, perm, keep, stream):
        if perm is not None and len(perm) != A.m:
            # the reference aborts: "Numbering array should have the same
            # size as matrix."
            raise ValueError("WrongDim: the ordering must have one entry per row")
        self._factorize_kept(A, perm, stream)
        if not keep:
            A.Clear()

    def _factorize_kept(self, A, perm, stream):
        if self.type_ilu in (self.ILUT, self.ILU_D, self.ILUT_K):
            f = self.factor_host(A.m, *A.download(), perm=perm, symmetric=A.symmetric)
            self.SetFactor(*f, symmetric=A.symmetric)
            return
        if A.symmetric:
            raise NotImplementedError("the reference has no symmetric ILU(0) or ILU(k) here")
        if self.type_ilu not in (self.ILU_0, self.MILU_0):
            raise NotImplementedError(
                "ILU_K is not factored here: factor it with Seldon "
                "(IlutPreconditioning::FactorizeMatrix) and pass it to SetFactor")
        import numpy as np
        if perm is not None and not np.array_equal(np.asarray(perm), np.arange(A.m)):
            raise NotImplementedError("the device ILU(0) uses the identity ordering")
        h = ctypes.c_void_p()
        check(_L.sb2_precond_create_ilu0(A.handle, int(self.type_ilu == self.MILU_0),
                                         _stream(stream), ctypes.byref(h)),
              "sb2_precond_create_ilu0")
        self.Clear()
        self._factor = ("device", A.m)
        self._device_handle = h

    def _params(self):
        return self._serial

    def Solve(self, *args, stream=None):
        """Solve(A, r, z), or in place Solve(z) and Solve(trans, z)
        (IlutPreconditioning.cxx:329-374)."""
        if len(args) == 3:
            return super().Solve(*args, stream=stream)
        if len(args) == 1:
            return self._in_place(args[0], False, stream)
        if len(args) == 2:
            return self._in_place(args[1], args[0] == SeldonTrans, stream)
        raise TypeError("Solve(A, r, z), Solve(z) or Solve(trans, z)")

    def TransSolve(self, *args, stream=None):
        """TransSolve(A, r, z), or in place TransSolve(z)."""
        if len(args) == 3:
            return super().TransSolve(*args, stream=stream)
        if len(args) == 1:
            return self._in_place(args[0], True, stream)
        raise TypeError("TransSolve(A, r, z) or TransSolve(z)")

    def _in_place(self, z, trans, stream):
        h = self.handle_for(None)
        n = self._factor[1] if self._factor[0] == "device" else self._factor[0]
        r = z.clone()
        fn = _L.sb2_precond_trans_solve if trans else _L.sb2_precond_solve
        check(fn(h, _dev_ptr(r, n, "z"), _dev_ptr(z, n, "z"), _stream(stream)),
              "TransSolve" if trans else "Solve")

    def __del__(self):
        try:
            self.Clear()
        except Exception:
            pass

    def handle_for(self, A):
        if self._factor is None:
            raise RuntimeError("IlutPreconditioning: no factor (call SetFactor first)")
        if self._factor[0] == "device":
            # the device factor keeps no reference to the matrix it came from
            if A is not None and A.m != self._factor[1]:
                raise ValueError("WrongDim: the factor's order differs from the matrix's")
            return self._device_handle
        key = (id(A), None if A is None else getattr(A.handle, "value", None))
        ent = self._cache.get(key)
        if ent is None or ent[0] is not A or ent[2] != self._serial:
            n, fptr, find, fval, prow, pcol, sym = self._factor
            h = ctypes.c_void_p()
            check(_L.sb2_precond_create_ilut(None if A is None else A.handle, n, _np_ptr(fptr), _np_ptr(find),
                                             _np_ptr(fval), _np_ptr(prow), _np_ptr(pcol),
                                             int(sym), ctypes.byref(h)),
                  "sb2_precond_create_ilut")
            if ent is not None:
                _L.sb2_precond_destroy(ent[1])
            ent = (A, h, self._serial)
            self._cache[key] = ent
        return ent[1]


def SOR(A, X, B, omega, iter, type_ssor=2, stream=None):
    """In-place relaxation (Relaxation_MatVect.cxx:41-95, :176-298)."""
    check(_L.sb2_sor(A.handle, _dev_ptr(X, A.m, "X"), _dev_ptr(B, A.m, "B"), float(omega),
                     int(iter), int(type_ssor), _stream(stream)), "SOR")


# ------------------------------------------------------------------ Iteration

class Iteration:
    """Iteration<double> (Iterative.hxx:47-108): defaults tol 1e-6,
    max_iter 100, restart 10, print level 1, null initial guess."""

    def __init__(self, max_iteration=100, tol=1e-6):
        self.tolerance = float(tol)
        self.max_iter = int(max_iteration)
        self.parameter_restart = 10
        self.print_level = 1
        self.init_guess_null = True
        self.nb_iter = 0
        self.error_code = 0
        self.facteur_reste = 0.0
        self.history = []      # (iteration, relative residual) of each Finished() test
        self.init_failed = False
        self.fail_convergence = False
        self.type_solver = 0
        self.type_preconditioning = 0

    def copy(self):
        """The copy constructor (Iterative.cxx:110-122): settings, factor and
        error code carried over, iteration count reset, null initial guess."""
        it = Iteration(self.max_iter, self.tolerance)
        it.facteur_reste = self.facteur_reste
        it.print_level = self.print_level
        it.error_code = self.error_code
        it.type_solver = self.type_solver
        it.parameter_restart = self.parameter_restart
        it.type_preconditioning = self.type_preconditioning
        return it

    def GetTypeSolver(self):
        return self.type_solver

    def SetSolver(self, type_resolution, param_restart, type_prec):
        self.type_solver = int(type_resolution)
        self.parameter_restart = int(param_restart)
        self.type_preconditioning = int(type_prec)

    def Init(self, r):
        """Iteration::Init (Iterative.cxx:236-251) on a device vector: -1 for
        a zero right-hand side, otherwise 1/Norm2(r) becomes the factor of
        the relative residual and the count restarts."""
        norm = Norm2(r)
        if norm == 0.0:
            return -1
        self.facteur_reste = 1.0 / norm
        self.nb_iter = 0
        return 0

    def First(self):
        return self.nb_iter == 0

    def Finished(self, r):
        """Iteration::Finished (Iterative.cxx:272-321) on a residual vector
        (its Norm2 on the device) or on a residual norm: true once the
        relative residual is below the tolerance or the count reaches
        max_iter, printing the reference's lines at its print levels."""
        reste = self.facteur_reste * (float(r) if isinstance(r, (int, float)) else Norm2(r))
        if (self.print_level >= 1 and self.nb_iter % 100 == 0) or self.print_level >= 6:
            print(f"Residu at iteration number {self.nb_iter}  {reste:g}")
        return reste < self.tolerance or self.nb_iter >= self.max_iter

    def Fail(self, i, s):
        """Iteration::Fail (Iterative.cxx:324-333)."""
        self.fail_convergence = True
        self.error_code = int(i)
        if self.print_level >= 1 and self.nb_iter % 100 == 0:
            print(f"Error during resolution : {s}")

    def __iadd__(self, k):
        """`it += 1` for the reference's ++iter."""
        self.nb_iter += int(k)
        return self

    def SetRestart(self, m):
        self.parameter_restart = int(m)

    def GetRestart(self):
        return self.parameter_restart

    def SetTolerance(self, tol):
        self.tolerance = float(tol)

    def GetTolerance(self):
        return self.tolerance

    def SetMaxNumberIteration(self, n):
        self.max_iter = int(n)

    def GetNumberIteration(self):
        return self.nb_iter

    def SetNumberIteration(self, n):
        self.nb_iter = int(n)

    def GetFactor(self):
        return self.facteur_reste

    def ShowMessages(self):
        self.print_level = 1

    def ShowFullHistory(self):
        self.print_level = 6

    def HideMessages(self):
        self.print_level = 0

    def SetInitGuess(self, null):
        self.init_guess_null = bool(null)

    def IsInitGuess_Null(self):
        return self.init_guess_null

    def ErrorCode(self):
        """Iteration::ErrorCode (Iterative.cxx:345-354)."""
        if self.nb_iter >= self.max_iter:
            return -2
        if self.fail_convergence:
            return self.error_code
        return 0

    def _replay(self):
        # the lines Iteration::Finished prints (Iterative.cxx:282-287)
        for it, res in self.history:
            if (self.print_level >= 1 and it % 100 == 0) or self.print_level >= 6:
                print(f"Residu at iteration number {it}  {res:g}")


def _solve(fn, A, x, b, M, iteration, hist_cap, stream):
    import numpy as np
    params = IterParams(iteration.tolerance, iteration.max_iter, iteration.parameter_restart,
                        iteration.print_level, int(iteration.init_guess_null))
    res = IterResult()
    cap = int(hist_cap if hist_cap is not None else max(iteration.max_iter * 2 + 8, 16))
    hist = np.zeros(cap)
    hist_it = np.zeros(cap, dtype=np.int32)
    Mh = None if M is None else M.handle_for(A)
    st = fn(A.handle, Mh, _dev_ptr(x, A.m, "x"), _dev_ptr(b, A.m, "b"), ctypes.byref(params),
            ctypes.byref(res), _np_ptr(hist), _np_ptr(hist_it), cap, _stream(stream))
    check(st, fn.__name__)
    iteration.nb_iter = res.nb_iter
    iteration.error_code = res.error_code
    iteration.fail_convergence = res.error_code not in (0, -2)
    iteration.facteur_reste = res.facteur_reste
    iteration.init_failed = bool(res.init_failed)
    iteration.history = list(zip(hist_it[:res.hist_len].tolist(), hist[:res.hist_len].tolist()))
    iteration._replay()
    return res.error_code


def Cg(A, x, b, M, iteration, hist_cap=None, stream=None):
    """Preconditioned CG (Cg.cxx:45-116); returns Iteration::ErrorCode()."""
    return _solve(_L.sb2_cg, A, x, b, M, iteration, hist_cap, stream)


def BiCgStab(A, x, b, M, iteration, hist_cap=None, stream=None):
    """BiCGSTAB (BiCgStab.cxx:43-145); returns Iteration::ErrorCode()."""
    return _solve(_L.sb2_bicgstab, A, x, b, M, iteration, hist_cap, stream)


def Cgs(A, x, b, M, iteration, hist_cap=None, stream=None):
    """Conjugate gradient squared (Cgs.cxx:45-132), right preconditioned;
    returns Iteration::ErrorCode()."""
    return _solve(_L.sb2_cgs, A, x, b, M, iteration, hist_cap, stream)


def TfQmr(A, x, b, M, iteration, hist_cap=None, stream=None):
    """Transpose-free QMR (TfQmr.cxx:44-243), left preconditioned; the
    stopping test is on the quasi-residual bound; returns
    Iteration::ErrorCode()."""
    return _solve(_L.sb2_tfqmr, A, x, b, M, iteration, hist_cap, stream)


def MinRes(A, x, b, M, iteration, hist_cap=None, stream=None):
    """MINRES for symmetric (possibly indefinite) systems (MinRes.cxx:46-153);
    the stopping test is on the recurrence's residual estimate; returns
    Iteration::ErrorCode()."""
    return _solve(_L.sb2_minres, A, x, b, M, iteration, hist_cap, stream)


def Gcr(A, x, b, M, iteration, hist_cap=None, stream=None):
    """Restarted generalized conjugate residuals (Gcr.cxx:45-141), left
    preconditioned, restart iteration.GetRestart(); returns
    Iteration::ErrorCode()."""
    return _solve(_L.sb2_gcr, A, x, b, M, iteration, hist_cap, stream)


def Symmlq(A, x, b, M, iteration, hist_cap=None, stream=None):
    """Symmlq (Symmlq.cxx:45-161); returns Iteration::ErrorCode()."""
    return _solve(_L.sb2_symmlq, A, x, b, M, iteration, hist_cap, stream)


def QmrSym(A, x, b, M, iteration, hist_cap=None, stream=None):
    """QMR for symmetric systems (QmrSym.cxx:41-165); returns
    Iteration::ErrorCode()."""
    return _solve(_L.sb2_qmrsym, A, x, b, M, iteration, hist_cap, stream)


def Lsqr(A, x, b, M, iteration, hist_cap=None, stream=None):
    """Lsqr (Lsqr.cxx:40-135); M is not used, as in the reference; returns
    Iteration::ErrorCode()."""
    return _solve(_L.sb2_lsqr, A, x, b, M, iteration, hist_cap, stream)


def BiCgcr(A, x, b, M, iteration, hist_cap=None, stream=None):
    """Biconjugate conjugate residuals (BiCgcr.cxx:44-118); returns
    Iteration::ErrorCode()."""
    return _solve(_L.sb2_bicgcr, A, x, b, M, iteration, hist_cap, stream)


def Cgne(A, x, b, M, iteration, hist_cap=None, stream=None):
    """CG on the normal equations A^T A x = A^T b (Cgne.cxx:40-127);
    returns Iteration::ErrorCode()."""
    return _solve(_L.sb2_cgne, A, x, b, M, iteration, hist_cap, stream)


def CoCg(A, x, b, M, iteration, hist_cap=None, stream=None):
    """CoCg (CoCg.cxx:45-116): in real arithmetic Cg's steps and results;
    returns Iteration::ErrorCode()."""
    return _solve(_L.sb2_cocg, A, x, b, M, iteration, hist_cap, stream)


def BiCg(A, x, b, M, iteration, hist_cap=None, stream=None):
    """Biconjugate gradients (BiCg.cxx:46-134), one product by A and one by
    A^T per loop; returns Iteration::ErrorCode()."""
    return _solve(_L.sb2_bicg, A, x, b, M, iteration, hist_cap, stream)


def QCgs(A, x, b, M, iteration, hist_cap=None, stream=None):
    """Cgs with a quasi-minimal smoothing step (QCgs.cxx:46-165), right
    preconditioned; returns Iteration::ErrorCode()."""
    return _solve(_L.sb2_qcgs, A, x, b, M, iteration, hist_cap, stream)


def BiCgStabl(A, x, b, M, iteration, hist_cap=None, stream=None):
    """BiCGSTAB(l) with l = iteration.GetRestart() >= 1 (BiCgStabl.cxx:43-180),
    right preconditioned; returns Iteration::ErrorCode()."""
    return _solve(_L.sb2_bicgstabl, A, x, b, M, iteration, hist_cap, stream)


def Gmres(A, x, b, M, iteration, hist_cap=None, stream=None, orthogonalization="mgs"):
    """Restarted left-preconditioned GMRES(m) (Gmres.cxx:44-183).

    orthogonalization="mgs" runs the reference's modified Gram-Schmidt loop
    (Gmres.cxx:127-132); "cgs2" the labelled variant that projects on the
    whole basis at once, twice (three grid reductions per step instead of
    i + 2; identity or Jacobi preconditioner, restart <= 32)."""
    if orthogonalization not in ("mgs", "cgs2"):
        raise ValueError(f"orthogonalization must be 'mgs' or 'cgs2', not {orthogonalization!r}")
    fn = _L.sb2_gmres if orthogonalization == "mgs" else _L.sb2_gmres_cgs2
    return _solve(fn, A, x, b, M, iteration, hist_cap, stream)


# ------------------------------------------------------------------ mixed precision

def IterativeRefinement(A, x, b, M=None, tol=1e-10, inner_tol=None, max_outer=None,
                        max_inner=20000, init_guess_null=True, restarted=False, stream=None,
                        solver="cg", restart=30):
    """FP32-inner / FP64-outer iterative refinement with CG or GMRES.

    solver="gmres": restarted GMRES(restart) whose restarts are the FP64
    refinement steps (FP32 Arnoldi basis, FP64 Hessenberg, update and
    residual); a cycle also ends once its residual estimate has dropped by
    inner_tol (default 1e-6); max_outer bounds the cycles (default 1000;
    50 refinement steps for CG), max_inner the Arnoldi steps; `restarted` is
    not read.

    restarted=False: reliable updates -- one FP32 CG run whose residual is
    replaced by the FP64 true residual each time it has dropped by inner_tol
    (default 1e-2); True: a fresh FP32 CG solve of A d = r to inner_tol
    (default 1e-5) per outer step.  Returns (error_code, info) with the FP64
    corrections, FP32 iterations, final FP64 relative residual and the
    residual history."""
    import numpy as np
    if solver not in ("cg", "gmres"):
        raise ValueError(f"solver must be 'cg' or 'gmres', not {solver!r}")
    gm = solver == "gmres"
    if inner_tol is None:
        inner_tol = 1e-6 if gm else (1e-5 if restarted else 1e-2)
    if max_outer is None:
        max_outer = 1000 if gm else 50
    prm = IrParams(tol, inner_tol, max_outer, max_inner, 1 if gm else 0, int(restart) if gm else 0,
                   int(init_guess_null), 1 if restarted else 0)
    res = IrResult()
    hist = np.zeros(max_outer + 2)
    Mh = None if (M is None or M.kind == _lib.PRECOND_IDENTITY) else M.handle_for(A)
    check(_L.sb2_ir_solve(A.handle, Mh, _dev_ptr(x, A.m, "x"), _dev_ptr(b, A.m, "b"),
                          ctypes.byref(prm), ctypes.byref(res), _np_ptr(hist), hist.size,
                          _stream(stream)), "sb2_ir_solve")
    info = {"outer_iter": res.outer_iter, "inner_iter": res.inner_iter,
            "rel_residual": res.rel_residual, "init_failed": bool(res.init_failed),
            "history": hist[:res.hist_len].tolist()}
    return res.error_code, info


# ------------------------------------------------------------------ batched solves

class Batch:
    """Independent systems solved together (block-diagonal CSR + row ranges).

    systems: list of (ptr, ind, val) CSR triples with local indices."""

    def __init__(self, systems):
        import numpy as np
        sizes = [len(p) - 1 for p, _, _ in systems]
        sys_row = np.zeros(len(systems) + 1, dtype=np.int32)
        np.cumsum(sizes, out=sys_row[1:])
        ptrs, inds, vals, off, base = [], [], [], 0, 0
        for (p, i, v), r0 in zip(systems, sys_row[:-1]):
            p = np.asarray(p, dtype=np.int64)
            ptrs.append(p[:-1] + base)
            inds.append(np.asarray(i, dtype=np.int64) + r0)
            vals.append(np.asarray(v, dtype=np.float64))
            base += int(p[-1])
        ptr = np.concatenate(ptrs + [np.array([base])]).astype(np.int32)
        ind = np.ascontiguousarray(np.concatenate(inds).astype(np.int32))
        val = np.ascontiguousarray(np.concatenate(vals))
        self.sys_row = sys_row
        self.m = int(sys_row[-1])
        self.nsys = len(systems)
        h = ctypes.c_void_p()
        check(_L.sb2_batch_create(self.nsys, _np_ptr(sys_row), _np_ptr(ptr), _np_ptr(ind),
                                  _np_ptr(val), ctypes.byref(h)), "sb2_batch_create")
        self._h = h

    @property
    def handle(self):
        return self._h

    def params(self, tol=1e-9, update_ratio=1e-2, max_iter=10000, mixed=True, init_guess_null=True):
        return _lib.BatchParams(tol, update_ratio, max_iter, 0 if mixed else 1, int(init_guess_null))

    def solve(self, x, b, iters=None, relres=None, summary=True, stream=None, **kw):
        """Solve all systems; iters/relres: optional device tensors (int32/float64)."""
        import torch
        prm = self.params(**kw)
        if summary and (iters is None or relres is None):
            iters = torch.zeros(self.nsys, dtype=torch.int32, device=x.device)
            relres = torch.zeros(self.nsys, dtype=torch.float64, device=x.device)
        res = _lib.BatchResult()
        check(_L.sb2_batch_solve(self._h, _dev_ptr(x, self.m, "x"), _dev_ptr(b, self.m, "b"),
                                 ctypes.byref(prm),
                                 ctypes.c_void_p(iters.data_ptr()) if iters is not None else None,
                                 ctypes.c_void_p(relres.data_ptr()) if relres is not None else None,
                                 ctypes.byref(res) if summary else None, _stream(stream)),
              "sb2_batch_solve")
        return res if summary else None

    def autotune(self, x, b, stream=None, **kw):
        """Times the candidate plans on this batch (x is overwritten) and keeps
        the fastest; a batch with the same size histogram reuses the cached
        choice.  Returns the CTA size (see plan())."""
        prm = self.params(**kw)
        check(_L.sb2_batch_autotune(self._h, _dev_ptr(x, self.m, "x"), _dev_ptr(b, self.m, "b"),
                                    ctypes.byref(prm), _stream(stream)), "sb2_batch_autotune")
        return _L.sb2_batch_get_threads(self._h)

    def plan(self):
        """(threads per CTA, largest system one warp solves; 0: none)."""
        t, w = ctypes.c_int(0), ctypes.c_int(0)
        check(_L.sb2_batch_get_plan(self._h, ctypes.byref(t), ctypes.byref(w)), "sb2_batch_get_plan")
        return t.value, w.value

    def set_plan(self, threads, warp_max=0, cluster=0, cluster_min=0):
        """Fixes the plan: CTA size, largest system one warp solves, and the
        cluster part (CTAs per cluster, 0: none; systems of more than
        cluster_min rows each take a whole cluster)."""
        check(_L.sb2_batch_set_plan(self._h, int(threads), int(warp_max)), "sb2_batch_set_plan")
        if cluster:
            check(_L.sb2_batch_set_cluster_plan(self._h, int(cluster), int(cluster_min)),
                  "sb2_batch_set_cluster_plan")

    def cluster_plan(self):
        """(CTAs per cluster, 0: none; systems of more rows take a whole cluster)."""
        c, m = ctypes.c_int(0), ctypes.c_int(0)
        check(_L.sb2_batch_get_cluster_plan(self._h, ctypes.byref(c), ctypes.byref(m)),
              "sb2_batch_get_cluster_plan")
        return c.value, m.value

    @classmethod
    def from_coordinates(cls, IndRow, IndCol, Val, index=0, m=0, n=0, validate=True):
        """Matrix built from coordinate triplets on the device, as
        ConvertMatrix_from_Coordinates fills an m x n matrix."""
        m, n, ptr, ind, val = ConvertMatrix_from_Coordinates(
            IndRow, IndCol, Val, index, m, n, cls.symmetric)
        if cls.symmetric:
            return cls(m, ptr, ind, val, validate)
        return cls(m, n, ptr, ind, val, validate)

    def close(self):
        if getattr(self, "_h", None):
            _L.sb2_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
