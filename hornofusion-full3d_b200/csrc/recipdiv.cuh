// Correctly rounded t / m from a precomputed y = RN(1/m), by one correction
// step (Markstein, "Computation of elementary functions on the IBM RISC
// System/6000 processor", IBM J. Res. Dev. 34(1), 1990, Theorem 1): with
// q = RN(t*y) within one ulp of t/m, the residual r = t - m*q is exact in an
// FMA and RN(q + r*y) is the correctly rounded quotient -- the value `/`
// returns. The theorem needs the operands away from overflow and underflow:
// both exponents in [-500, 500] (then q, r and r*y are normal); anything else
// -- zeros, subnormals, huge values, infinities, NaN -- takes `/` itself.
// Used where one divisor serves several quotients (one reciprocal, then a
// multiply and two FMAs each) or where the reciprocal can leave a dependent
// chain. eaf_diag_div_check compares it with `/` bit for bit on the device.
#pragma once

#include <cuda_runtime.h>

namespace eaf {

__device__ __forceinline__ bool exp_in_safe_range(double v) {
  const unsigned e = (unsigned)((unsigned long long)__double_as_longlong(v) >> 52) & 0x7ffu;
  return e - 523u <= 1000u;  // biased exponent 523..1523
}

__device__ __forceinline__ double div_by_recip(double t, double m, double y, bool m_ok) {
  if (m_ok && (t == 0.0 || exp_in_safe_range(t))) {
    const double q = t * y;
    const double c = __fma_rn(__fma_rn(-q, m, t), y, q);
    return t == 0.0 ? q : c;
  }
  return t / m;
}

}  // namespace eaf
