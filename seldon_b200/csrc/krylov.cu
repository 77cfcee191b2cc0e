// Krylov drivers (placeholder entry points).
#include "sb2_internal.cuh"

extern "C" {
int sb2_cg(const sb2_csr*, const sb2_precond*, double*, const double*, const sb2_iter_params*, sb2_iter_result*, double*, int*, int, void*) { return SB2_ERR_NOT_SUPPORTED; }
int sb2_bicgstab(const sb2_csr*, const sb2_precond*, double*, const double*, const sb2_iter_params*, sb2_iter_result*, double*, int*, int, void*) { return SB2_ERR_NOT_SUPPORTED; }
int sb2_gmres(const sb2_csr*, const sb2_precond*, double*, const double*, const sb2_iter_params*, sb2_iter_result*, double*, int*, int, void*) { return SB2_ERR_NOT_SUPPORTED; }
}
