"""C++ drop-in: Seldon user code templated on the allocator runs on Seldon's
host types and on the CudaAlloc device types of include/SeldonB200.hxx, and
every result is compared (tests/cpp/dropin_test.cpp): SpMV, BLAS-1, the fused
Cg/BiCgStab/Gmres, and all of Seldon's other Krylov drivers."""
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "tests", "cpp", "_bin", "dropin_test")


def test_cpp_dropin(cuda, tmp_path):
    if not os.path.exists(BIN):
        pytest.skip("dropin_test not built (needs the reference headers: make -C tests/cpp)")
    p = subprocess.run([BIN], capture_output=True, text=True, timeout=600, cwd=str(tmp_path))
    print(p.stdout)
    lines = [ln for ln in p.stdout.splitlines() if ln.startswith(("PASS", "FAIL"))]
    fails = [ln for ln in lines if ln.startswith("FAIL")]
    assert p.returncode == 0 and not fails, (p.returncode, fails, p.stderr[-2000:])
    names = {ln.split()[1] for ln in lines}
    for must in ("spmv_general", "spmv_symmetric", "blas1", "cg_identity", "cg_ssor",
                 "gmres20_jacobi", "bicgstab_identity", "cg_user_preconditioner",
                 "cg_zero_rhs", "invalid_csr_throws", "binary_files",
                 "coordinate_assembly", "text_files", "ilut_apply", "ilut_gmres",
                 "ilut_bicgstab", "ilut_sym_apply", "ilut_cg", "harwell_boeing", "array_row_sparse"):
        assert must in names, must
    # Seldon's other Krylov drivers, its generic templates on device types
    for drv in ("bicg", "bicgstabl", "bicgcr", "cgne", "cgs", "cocg", "gcr", "lsqr", "minres",
                "qcgs", "qmr", "qmrsym", "symmlq", "tfqmr"):
        assert "generic_" + drv in names, drv
