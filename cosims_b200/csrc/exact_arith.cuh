// exact_arith.cuh -- correctly rounded FP64 division and square root without
// branches, for operands in a stated range.
//
// The plain FP64 form must reproduce the reference's IEEE results bit for bit,
// and its force loops evaluate three divisions and a square root per atom.
// The library routines for IEEE division and square root contain a branch to
// a slow path for operands near the ends of the exponent range; the branch
// ends a basic block, so the instruction scheduler cannot overlap the
// dependent chains of one division with the work around it, and a thread
// runs its per-atom chains one after another.  The routines here give the same
// correctly rounded results with straight-line code, for the operands the
// force loops see (the caller checks the range once per evaluation and falls
// back to the IEEE operators outside it).
//
// Method (round to nearest, ties impossible -- see below):
//  1. A hardware approximation of 1/b (or 1/sqrt(x)) is refined by
//     Newton-Raphson iterations with fused multiply-adds (P. Markstein,
//     "Computation of elementary functions on the IBM RISC System/6000
//     processor", IBM J. Res. Dev. 34(1), 1990).
//  2. One correction step, q = q0 + (a - b q0) y, gives a faithful quotient
//     (within one ulp of a/b); likewise s = s0 + (x - s0^2) y / 2 for the root.
//  3. The remainder of a faithful result is exactly representable and one FMA
//     computes it exactly (S. Boldo, M. Daumas, "Representable correcting
//     terms for possibly underflowing floating point operations", ARITH 16,
//     2003).  It decides between the faithful result and its neighbours by an
//     exact comparison with the distance to the midpoint:
//       division:  a/b > q + u/2  <=>  a - b q > b u / 2    (u = ulp above q)
//       root:      sqrt(x) > s + u/2  <=>  (x - s^2) - s u > 0
//     (x - s^2 and s u are integer multiples of u^2, so the u^2/4 of the
//     exact midpoint condition drops out).  A quotient or root of binary
//     floating-point numbers never lies exactly on a midpoint, so there are no
//     ties to break.
// Round to nearest is symmetric, so a quotient is formed on magnitudes and
// takes the sign of the dividend (the divisor is positive here).
//
// Valid range: divisor b in [2^-300, 2^300], dividend |a| <= 2^600 or zero,
// root argument x in [2^-300, 2^300].  Inside it every intermediate is a
// normal number and the results equal CUDA's IEEE `/` and `sqrt` bit for bit
// (tests/test_gpu_exact_arith.py compares them on many operands).
#pragma once
#include <cuda_runtime.h>

namespace cosims {

__device__ __forceinline__ double rcp_approx(double b) {
  double y;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(b));
  return y;
}

__device__ __forceinline__ double rsqrt_approx(double x) {
  double y;
  asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
  return y;
}

__device__ __forceinline__ double next_up_pos(double v) {
  return __longlong_as_double(__double_as_longlong(v) + 1);
}
__device__ __forceinline__ double next_down_pos(double v) {
  return __longlong_as_double(__double_as_longlong(v) - 1);
}

// True when b is a divisor the branch-free division handles.
__device__ __forceinline__ bool div_ok(double b) { return b >= 0x1p-300 && b <= 0x1p300; }
__device__ __forceinline__ bool sqrt_ok(double x) { return x >= 0x1p-300 && x <= 0x1p300; }

// a / b rounded to nearest for b in [2^-300, 2^300] and |a| <= 2^600 (or 0).
__device__ __forceinline__ double div_rn_pos(double a, double b) {
  const double A = fabs(a);
  double y = rcp_approx(b);
  double e = __fma_rn(-b, y, 1.0);
  y = __fma_rn(y, e, y);
  e = __fma_rn(-b, y, 1.0);
  y = __fma_rn(y, e, y);
  e = __fma_rn(-b, y, 1.0);
  y = __fma_rn(y, e, y);
  double q = __dmul_rn(A, y);
  double r = __fma_rn(-b, q, A);
  q = __fma_rn(r, y, q);                         // faithful
  r = __fma_rn(-b, q, A);                        // exact remainder
  const double up = next_up_pos(q), dn = next_down_pos(q);
  const double half_up = __dmul_rn(__dmul_rn(b, __dsub_rn(up, q)), 0.5);
  const double half_dn = __dmul_rn(__dmul_rn(b, __dsub_rn(q, dn)), 0.5);
  q = r > half_up ? up : q;
  q = r < -half_dn ? dn : q;
  q = A == 0.0 ? 0.0 : q;
  return copysign(q, a);
}

// sqrt(x) rounded to nearest for x in [2^-300, 2^300].
__device__ __forceinline__ double sqrt_rn(double x) {
  double y = rsqrt_approx(x);
  const double h = __dmul_rn(0.5, x);
  double e = __fma_rn(-__dmul_rn(h, y), y, 0.5);
  y = __fma_rn(y, e, y);
  e = __fma_rn(-__dmul_rn(h, y), y, 0.5);
  y = __fma_rn(y, e, y);
  e = __fma_rn(-__dmul_rn(h, y), y, 0.5);
  y = __fma_rn(y, e, y);
  double s = __dmul_rn(x, y);
  double r = __fma_rn(-s, s, x);
  s = __fma_rn(r, __dmul_rn(0.5, y), s);         // faithful
  r = __fma_rn(-s, s, x);                        // x - s^2
  const double up = next_up_pos(s), dn = next_down_pos(s);
  const double su = __dmul_rn(s, __dsub_rn(up, s)), sd = __dmul_rn(s, __dsub_rn(s, dn));
  s = __dsub_rn(r, su) > 0.0 ? up : s;
  s = __dadd_rn(r, sd) <= 0.0 && r < 0.0 ? dn : s;
  return s;
}

}  // namespace cosims
