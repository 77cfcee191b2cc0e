// Givens rotations of the GMRES drivers, on the device: Seldon's GenRot and
// ApplyRot, with every product and sum rounded separately so the rotations
// equal the reference's bit for bit.
#pragma once

#include "sb2_internal.cuh"

namespace sb2 {

#ifdef __CUDACC__

// Givens rotation, Functions_Vector.cxx:612-649 (old BLAS drotg semantics).
__device__ __forceinline__ void gen_rot(double& a_in, double& b_in, double& c_, double& s_) {
  const double a = a_in, b = b_in;
  const double roe = (fabs(a) > fabs(b)) ? a : b;
  const double scal = fabs(a) + fabs(b);
  double r, z;
  if (scal != 0.0) {
    const double a_scl = a / scal, b_scl = b / scal;
    r = mul_rn(scal, sqrt(add_rn(mul_rn(a_scl, a_scl), mul_rn(b_scl, b_scl))));
    if (roe < 0.0) r = mul_rn(r, -1.0);
    c_ = a / r;
    s_ = b / r;
    z = 1.0;
    if (fabs(a) > fabs(b)) z = s_;
    else if (fabs(b) >= fabs(a) && c_ != 0.0) z = 1.0 / c_;
  } else {
    c_ = 1.0;
    s_ = 0.0;
    r = 0.0;
    z = 0.0;
  }
  a_in = r;
  b_in = z;
}

// Functions_Vector.cxx:681-687
__device__ __forceinline__ void apply_rot(double& x, double& y, double c, double s) {
  const double temp = add_rn(mul_rn(c, x), mul_rn(s, y));
  y = __dsub_rn(mul_rn(c, y), mul_rn(s, x));
  x = temp;
}

#endif  // __CUDACC__

}  // namespace sb2
