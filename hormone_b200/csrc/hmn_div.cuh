// hmn_div.cuh -- correctly rounded FP64 division without branches, for
// quotients that share a denominator.
//
// Method: P. Markstein, "Computation of elementary functions on the IBM
// RISC System/6000 processor", IBM J. Res. Develop. 34(1), 1990, and its
// statement in J.-M. Muller et al., "Handbook of Floating-Point Arithmetic"
// (2nd ed., 2018), section 4.7 (Newton-Raphson division with an FMA):
//
//  * reciprocal: from an approximation y0 of 1/b, Newton-Raphson steps
//    y <- y + y (1 - b y) (each residual with one FMA) until y is within
//    one ulp of 1/b; one more such step then gives RN(1/b) exactly, unless
//    the significand of b is 1.11...1 (Markstein's theorem for the
//    reciprocal);
//  * quotient: with y = RN(1/b), q0 = RN(a y) is within 1.5 ulp of a/b;
//    q1 = RN(q0 + r0 y), r0 = RN(a - b q0), is within one ulp; and with q1
//    within one ulp, q2 = RN(q1 + r1 y), r1 = a - b q1 (exact), is RN(a/b)
//    (Markstein's theorem for the quotient).
//
// Both theorems assume that no intermediate overflows or underflows.  The
// operations here check the operands' exponents instead of branching: a
// denominator or numerator outside [2^-500, 2^500] in magnitude (and every
// zero, infinity or NaN denominator, and b with an all-ones significand)
// sets `bad`, and the caller then recomputes with IEEE division.  A zero
// numerator is exact and keeps its sign (q = a * y).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace hmn {

// |x| in [2^-500, 2^500]: biased exponent in [523, 1523].  The high word
// shifted left by one drops the sign and puts the exponent in bits 21..31,
// so the test is one shift-add and one unsigned compare.
__device__ __forceinline__ bool fin_range(double x) {
  const unsigned t = (unsigned)__double2hiint(x) << 1;
  return t - (523u << 21) < (1001u << 21);
}

// approximate reciprocal (relative error below 2^-22 or so; refined below)
__device__ __forceinline__ double rcp_approx(double b) {
  double y;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(b));
  return y;
}

// 1/b within about one ulp, without branches (two Newton-Raphson steps from
// the approximation); for the mixed-precision form, which is not bound to
// IEEE quotients.  A zero b gives NaN where IEEE gives infinity.
__device__ __forceinline__ double rcp_nr(double b) {
  double y = rcp_approx(b);
  double e = __fma_rn(-b, y, 1.0);
  y = __fma_rn(y, e, y);
  e = __fma_rn(-b, y, 1.0);
  return __fma_rn(y, e, y);
}

// RN(1/b); sets bad where b is out of range or has an all-ones significand
__device__ __forceinline__ double recip_rn(double b, bool& bad) {
  const unsigned lo = (unsigned)__double2loint(b), hi = (unsigned)__double2hiint(b);
  // all-ones significand: the low word and the 20 significand bits of the
  // high word are all ones
  bad = bad || !fin_range(b) || ((hi | 0xfff00000u) & lo) == 0xffffffffu;
  double y = rcp_approx(b);
  double e = __fma_rn(-b, y, 1.0);
  y = __fma_rn(y, e, y);
  e = __fma_rn(-b, y, 1.0);
  y = __fma_rn(y, e, y);  // within one ulp of 1/b
  e = __fma_rn(-b, y, 1.0);
  return __fma_rn(y, e, y);  // RN(1/b)
}

// RN(a/b) from y = RN(1/b); sets bad where a is out of range (zero excepted)
__device__ __forceinline__ double div_rn(double a, double b, double y, bool& bad) {
  bad = bad || !(fin_range(a) || a == 0.0);
  const double q0 = a * y;
  const double r0 = __fma_rn(-b, q0, a);
  const double q1 = __fma_rn(r0, y, q0);
  const double r1 = __fma_rn(-b, q1, a);
  const double q2 = __fma_rn(r1, y, q1);
  return a == 0.0 ? q0 : q2;
}

}  // namespace hmn

namespace hmn {

// Division policy of hmn_math.cuh with the operations above: `bad` records
// whether any quotient since construction may differ from IEEE division,
// in which case the caller recomputes the whole expression with PlainDiv.
struct FastDiv {
  bool bad = false;
  __device__ __forceinline__ double rec(double b) { return recip_rn(b, bad); }
  __device__ __forceinline__ double div(double a, double b, double y) { return div_rn(a, b, y, bad); }
};

}  // namespace hmn
