// Preconditioners (placeholder entry points; filled in by the solver work).
#include "sb2_internal.cuh"

struct sb2_precond {
  int kind;
};

extern "C" {
int sb2_precond_create(const sb2_csr*, int, double, int, int, sb2_precond** out) {
  if (out) *out = nullptr;
  return SB2_ERR_NOT_SUPPORTED;
}
int sb2_precond_destroy(sb2_precond* M) { delete M; return SB2_OK; }
int sb2_precond_solve(const sb2_precond*, const double*, double*, void*) { return SB2_ERR_NOT_SUPPORTED; }
int sb2_precond_trans_solve(const sb2_precond*, const double*, double*, void*) { return SB2_ERR_NOT_SUPPORTED; }
int sb2_sor(const sb2_csr*, double*, const double*, double, int, int, void*) { return SB2_ERR_NOT_SUPPORTED; }
}
