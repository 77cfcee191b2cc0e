"""ctypes binding of libseldon_b200.so (the C ABI in include/seldon_b200.h).

The shared library is built in-tree (seldon_b200/libseldon_b200.so) by
``seldon_b200.build.build_library()``.  There is no fallback: if the library
is missing or fails to load, importing this module raises.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libseldon_b200.so")

SB2_OK = 0
SB2_ERR_INVALID_VALUE = -1
SB2_ERR_NO_MEMORY = -2
SB2_ERR_CUDA = -3
SB2_ERR_TIMEOUT = -4
SB2_ERR_INVALID_CSR = -5
SB2_ERR_NOT_SUPPORTED = -6
SB2_ERR_HOST = -7

SPMV_SELL = 0
SPMV_STREAM = 1
SPMV_TMA = 2

PRECOND_IDENTITY = 0
PRECOND_JACOBI = 1
PRECOND_SOR = 2
PRECOND_ILUT = 3

c_int_p = ctypes.POINTER(ctypes.c_int)
c_double_p = ctypes.POINTER(ctypes.c_double)
c_void_p = ctypes.c_void_p


class IlutParams(ctypes.Structure):
    """sb2_ilut_params: IlutPreconditioning's settings."""

    _fields_ = [
        ("type", ctypes.c_int),
        ("fill_level", ctypes.c_int),
        ("additional_fill", ctypes.c_int),
        ("mbloc", ctypes.c_int),
        ("alpha", ctypes.c_double),
        ("droptol", ctypes.c_double),
        ("permtol", ctypes.c_double),
    ]


class IterParams(ctypes.Structure):
    """sb2_iter_params: Seldon's Iteration<double> settings."""

    _fields_ = [
        ("tol", ctypes.c_double),
        ("max_iter", ctypes.c_int),
        ("restart", ctypes.c_int),
        ("print_level", ctypes.c_int),
        ("init_guess_null", ctypes.c_int),
    ]


class IterResult(ctypes.Structure):
    """sb2_iter_result: what a Krylov driver reports back."""

    _fields_ = [
        ("nb_iter", ctypes.c_int),
        ("error_code", ctypes.c_int),
        ("init_failed", ctypes.c_int),
        ("hist_len", ctypes.c_int),
        ("facteur_reste", ctypes.c_double),
        ("last_residual", ctypes.c_double),
    ]


class IrParams(ctypes.Structure):
    """sb2_ir_params: mixed-precision iterative refinement settings."""

    _fields_ = [
        ("tol", ctypes.c_double),
        ("inner_tol", ctypes.c_double),
        ("max_outer", ctypes.c_int),
        ("max_inner", ctypes.c_int),
        ("solver", ctypes.c_int),
        ("restart", ctypes.c_int),
        ("init_guess_null", ctypes.c_int),
        ("mode", ctypes.c_int),
    ]


class IrResult(ctypes.Structure):
    """sb2_ir_result."""

    _fields_ = [
        ("outer_iter", ctypes.c_int),
        ("inner_iter", ctypes.c_int),
        ("error_code", ctypes.c_int),
        ("init_failed", ctypes.c_int),
        ("hist_len", ctypes.c_int),
        ("rel_residual", ctypes.c_double),
    ]


class BatchParams(ctypes.Structure):
    """sb2_batch_params."""

    _fields_ = [
        ("tol", ctypes.c_double),
        ("update_ratio", ctypes.c_double),
        ("max_iter", ctypes.c_int),
        ("mode", ctypes.c_int),
        ("init_guess_null", ctypes.c_int),
    ]


class BatchResult(ctypes.Structure):
    """sb2_batch_result."""

    _fields_ = [
        ("converged", ctypes.c_int),
        ("max_iter", ctypes.c_int),
        ("total_iter", ctypes.c_longlong),
        ("max_rel_residual", ctypes.c_double),
    ]


class SeldonB200Error(RuntimeError):
    def __init__(self, status, where):
        self.status = status
        msg = _lib.sb2_status_string(status).decode() if _lib else str(status)
        super().__init__(f"{where}: status {status} ({msg})")


# (name, restype, argtypes) of every exported entry point
_PROTOS = [
    ("sb2_status_string", ctypes.c_char_p, [ctypes.c_int]),
    ("sb2_version", ctypes.c_int, []),
    ("sb2_device_alloc", ctypes.c_int, [ctypes.c_size_t, c_void_p]),
    ("sb2_device_free", ctypes.c_int, [c_void_p]),
    ("sb2_memcpy", ctypes.c_int, [c_void_p, c_void_p, ctypes.c_size_t, c_void_p]),
    ("sb2_stream_sync", ctypes.c_int, [c_void_p]),
    ("sb2_set_wait_limit_ms", ctypes.c_int, [ctypes.c_int]),
    ("sb2_set_wait_limit_us", ctypes.c_int, [ctypes.c_int]),
    ("sb2_krylov_set_pcg", ctypes.c_int, [ctypes.c_int]),
    ("sb2_spmv_status", ctypes.c_int, [c_void_p, c_int_p]),
    ("sb2_probe_gather", ctypes.c_int,
     [ctypes.c_longlong, c_void_p, c_void_p, c_void_p, c_void_p, ctypes.c_int, c_int_p, c_void_p]),
    ("sb2_csr_create", ctypes.c_int,
     [ctypes.c_int, ctypes.c_int, ctypes.c_int, c_void_p, c_void_p, c_void_p,
      ctypes.c_int, ctypes.c_int, ctypes.POINTER(c_void_p)]),
    ("sb2_csr_destroy", ctypes.c_int, [c_void_p]),
    ("sb2_csr_info", ctypes.c_int, [c_void_p, c_int_p, c_int_p, c_int_p, c_int_p]),
    ("sb2_csr_download", ctypes.c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
    ("sb2_precond_create_ilut", ctypes.c_int,
     [c_void_p, ctypes.c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, ctypes.c_int,
      ctypes.POINTER(c_void_p)]),
    ("sb2_ilut_factor", ctypes.c_int,
     [ctypes.c_int, c_void_p, c_void_p, c_void_p, c_void_p, ctypes.POINTER(IlutParams),
      ctypes.POINTER(c_void_p)]),
    ("sb2_ilut_factor_sym", ctypes.c_int,
     [ctypes.c_int, c_void_p, c_void_p, c_void_p, c_void_p, ctypes.POINTER(IlutParams),
      ctypes.POINTER(c_void_p)]),
    ("sb2_ilut_size", ctypes.c_int, [c_void_p, c_int_p, c_int_p]),
    ("sb2_ilut_arrays", ctypes.c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    ("sb2_ilut_destroy", ctypes.c_int, [c_void_p]),
    ("sb2_precond_create_ilu0", ctypes.c_int,
     [c_void_p, ctypes.c_int, c_void_p, ctypes.POINTER(c_void_p)]),
    ("sb2_coo_to_csr", ctypes.c_int,
     [ctypes.c_int, c_void_p, c_void_p, c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
      ctypes.c_int, c_void_p, c_int_p, c_int_p, c_int_p, ctypes.POINTER(c_void_p),
      ctypes.POINTER(c_void_p), ctypes.POINTER(c_void_p)]),
    ("sb2_spmv", ctypes.c_int,
     [c_void_p, ctypes.c_int, ctypes.c_double, c_void_p, ctypes.c_double, c_void_p, c_void_p]),
    ("sb2_mlt", ctypes.c_int,
     [c_void_p, ctypes.c_int, ctypes.c_double, c_void_p, c_void_p, c_void_p]),
    ("sb2_spmv_host", ctypes.c_int,
     [c_void_p, ctypes.c_int, ctypes.c_double, c_void_p, ctypes.c_double, c_void_p, c_void_p]),
    ("sb2_mlt_host", ctypes.c_int,
     [c_void_p, ctypes.c_int, ctypes.c_double, c_void_p, c_void_p, c_void_p]),
    ("sb2_mlt_host_batch", ctypes.c_int,
     [c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_int, c_void_p, c_void_p, c_void_p]),
    ("sb2_spmv_set_config", ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    ("sb2_krylov_set_config", ctypes.c_int, [ctypes.c_int]),
    ("sb2_krylov_set_cluster", ctypes.c_int, [ctypes.c_int]),
    ("sb2_dot", ctypes.c_int, [ctypes.c_int, c_void_p, c_void_p, c_double_p, c_void_p]),
    ("sb2_nrm2", ctypes.c_int, [ctypes.c_int, c_void_p, c_double_p, c_void_p]),
    ("sb2_dot_device", ctypes.c_int, [ctypes.c_int, c_void_p, c_void_p, c_void_p, c_void_p]),
    ("sb2_nrm2_device", ctypes.c_int, [ctypes.c_int, c_void_p, c_void_p, c_void_p]),
    ("sb2_axpy", ctypes.c_int, [ctypes.c_int, ctypes.c_double, c_void_p, c_void_p, c_void_p]),
    ("sb2_scal", ctypes.c_int, [ctypes.c_int, ctypes.c_double, c_void_p, c_void_p]),
    ("sb2_copy", ctypes.c_int, [ctypes.c_int, c_void_p, c_void_p, c_void_p]),
    ("sb2_fill", ctypes.c_int, [ctypes.c_int, ctypes.c_double, c_void_p, c_void_p]),
    ("sb2_precond_create", ctypes.c_int,
     [c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_int,
      ctypes.POINTER(c_void_p)]),
    ("sb2_precond_destroy", ctypes.c_int, [c_void_p]),
    ("sb2_precond_solve", ctypes.c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
    ("sb2_precond_trans_solve", ctypes.c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
    ("sb2_sor", ctypes.c_int,
     [c_void_p, c_void_p, c_void_p, ctypes.c_double, ctypes.c_int, ctypes.c_int, c_void_p]),
]

_SOLVER_ARGS = [c_void_p, c_void_p, c_void_p, c_void_p, ctypes.POINTER(IterParams),
                ctypes.POINTER(IterResult), c_void_p, c_void_p, ctypes.c_int, c_void_p]
for _name in ("sb2_cg", "sb2_bicgstab", "sb2_gmres", "sb2_gmres_cgs2", "sb2_cgs", "sb2_tfqmr",
              "sb2_minres", "sb2_gcr", "sb2_bicgstabl", "sb2_qcgs", "sb2_bicg", "sb2_cocg",
              "sb2_cgne", "sb2_bicgcr", "sb2_lsqr", "sb2_qmrsym", "sb2_symmlq"):
    _PROTOS.append((_name, ctypes.c_int, _SOLVER_ARGS))
_PROTOS.append(("sb2_ir_solve", ctypes.c_int,
                [c_void_p, c_void_p, c_void_p, c_void_p, ctypes.POINTER(IrParams),
                 ctypes.POINTER(IrResult), c_void_p, ctypes.c_int, c_void_p]))
_PROTOS += [
    ("sb2_batch_create", ctypes.c_int,
     [ctypes.c_int, c_void_p, c_void_p, c_void_p, c_void_p, ctypes.POINTER(c_void_p)]),
    ("sb2_batch_destroy", ctypes.c_int, [c_void_p]),
    ("sb2_batch_solve", ctypes.c_int,
     [c_void_p, c_void_p, c_void_p, ctypes.POINTER(BatchParams), c_void_p, c_void_p,
      ctypes.POINTER(BatchResult), c_void_p]),
    ("sb2_batch_autotune", ctypes.c_int,
     [c_void_p, c_void_p, c_void_p, ctypes.POINTER(BatchParams), c_void_p]),
    ("sb2_batch_set_threads", ctypes.c_int, [c_void_p, ctypes.c_int]),
    ("sb2_batch_get_threads", ctypes.c_int, [c_void_p]),
    ("sb2_batch_set_plan", ctypes.c_int, [c_void_p, ctypes.c_int, ctypes.c_int]),
    ("sb2_batch_get_plan", ctypes.c_int, [c_void_p, c_int_p, c_int_p]),
    ("sb2_batch_set_cluster_plan", ctypes.c_int, [c_void_p, ctypes.c_int, ctypes.c_int]),
    ("sb2_batch_get_cluster_plan", ctypes.c_int, [c_void_p, c_int_p, c_int_p]),
]
_PROTOS += [
    ("sb2_csr_set_values", ctypes.c_int, [c_void_p, c_void_p, ctypes.c_int, c_void_p]),
    ("sb2_grad_pattern", ctypes.c_int,
     [c_void_p, ctypes.c_double, c_void_p, c_void_p, c_void_p, c_void_p]),
    ("sb2_grad_edges", ctypes.c_int,
     [ctypes.c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
]
_PROTOS.append(("sb2_cg_noalloc", ctypes.c_int,
                [c_void_p, c_void_p, c_void_p, ctypes.POINTER(IterParams),
                 ctypes.POINTER(IterResult), c_void_p]))

_lib = None


def load():
    """Load the library (once) and attach prototypes.  Raises if absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with seldon_b200.build.build_library() "
            "(there is no CPU fallback)")
    lib = ctypes.CDLL(LIB_PATH)
    for name, res, args in _PROTOS:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def exported_names():
    return [p[0] for p in _PROTOS]


def check(status, where):
    if status != SB2_OK:
        raise SeldonB200Error(status, where)
