// Double-double ("dd") arithmetic on FP64 hardware, host and device.
//
// The reference keeps the solver scalars xx, scale and xz, and the subspace
// inverse-iteration step, in __float128 (src/config.h:44-51,
// src/wavefunction.h:166-169, src/solver.h:455-538).  A B200 has no quad
// precision, so these values are carried as an unevaluated sum hi + lo of two
// doubles (about 106 significant bits), using the error-free transformations
// of Knuth (TwoSum), Dekker (FastTwoSum) and the FMA form of TwoProduct, and
// the accurate dd add / mul / div / sqrt formulations published by Hida, Li and
// Bailey ("Library for double-double and quad-double arithmetic", 2007).
#pragma once

#include <cmath>

#if defined(__CUDACC__)
#define DD_HD __host__ __device__ __forceinline__
#else
#define DD_HD inline
#endif

namespace mcd {

struct dd {
  double hi, lo;
};

DD_HD dd dd_make(double hi, double lo = 0.0) { return dd{hi, lo}; }

// a + b = s + e exactly (requires |a| >= |b| or a == 0).
DD_HD dd dd_fast_two_sum(double a, double b) {
  double s = a + b;
  double e = b - (s - a);
  return dd{s, e};
}

// a + b = s + e exactly, no ordering requirement.
DD_HD dd dd_two_sum(double a, double b) {
  double s = a + b;
  double bb = s - a;
  double e = (a - (s - bb)) + (b - bb);
  return dd{s, e};
}

// a * b = p + e exactly.
DD_HD dd dd_two_prod(double a, double b) {
  double p = a * b;
#if defined(__CUDA_ARCH__)
  double e = __fma_rn(a, b, -p);
#else
  double e = std::fma(a, b, -p);
#endif
  return dd{p, e};
}

DD_HD dd dd_add(dd a, dd b) {
  dd s = dd_two_sum(a.hi, b.hi);
  dd t = dd_two_sum(a.lo, b.lo);
  s.lo += t.hi;
  s = dd_fast_two_sum(s.hi, s.lo);
  s.lo += t.lo;
  return dd_fast_two_sum(s.hi, s.lo);
}

DD_HD dd dd_add_d(dd a, double b) {
  dd s = dd_two_sum(a.hi, b);
  s.lo += a.lo;
  return dd_fast_two_sum(s.hi, s.lo);
}

DD_HD dd dd_neg(dd a) { return dd{-a.hi, -a.lo}; }

DD_HD dd dd_sub(dd a, dd b) { return dd_add(a, dd_neg(b)); }

DD_HD dd dd_mul(dd a, dd b) {
  dd p = dd_two_prod(a.hi, b.hi);
  p.lo += a.hi * b.lo + a.lo * b.hi;
  return dd_fast_two_sum(p.hi, p.lo);
}

DD_HD dd dd_mul_d(dd a, double b) {
  dd p = dd_two_prod(a.hi, b);
  p.lo += a.lo * b;
  return dd_fast_two_sum(p.hi, p.lo);
}

// Three quotient digits q1 + q2 + q3 from one reciprocal of b.hi: each digit
// is a double estimate of the remaining quotient and the exact remainder
// carries its error to the next one.
DD_HD dd dd_div(dd a, dd b) {
  const double rb = 1.0 / b.hi;
  double q1 = a.hi * rb;
  dd r = dd_sub(a, dd_mul_d(b, q1));
  double q2 = r.hi * rb;
  r = dd_sub(r, dd_mul_d(b, q2));
  double q3 = r.hi * rb;
  dd q = dd_fast_two_sum(q1, q2);
  return dd_add_d(q, q3);
}

DD_HD dd dd_div_d(dd a, double b) { return dd_div(a, dd{b, 0.0}); }

// One Newton step on the double square root (Karp's formulation).
DD_HD dd dd_sqrt(dd a) {
  if (a.hi <= 0.0) return dd{a.hi == 0.0 ? 0.0 : NAN, 0.0};
  double x = 1.0 / sqrt(a.hi);
  double ax = a.hi * x;
  dd ax2 = dd_two_prod(ax, ax);
  dd diff = dd_sub(a, ax2);
  double corr = diff.hi * (x * 0.5);
  return dd_two_sum(ax, corr);
}

DD_HD double dd_to_d(dd a) { return a.hi + a.lo; }

DD_HD dd dd_abs(dd a) { return a.hi < 0.0 ? dd_neg(a) : a; }

// a > b for dd values.
DD_HD bool dd_gt(dd a, dd b) { return a.hi > b.hi || (a.hi == b.hi && a.lo > b.lo); }

}  // namespace mcd
