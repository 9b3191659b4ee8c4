// Correctly rounded FP64 division with the divisor's reciprocal shared between dividends.
//
// The stage kernels divide every tracer of a lane by the same lane quantity (areasvol,
// hnode_new, the QR4C depth gaps, the node-average area, 3, 6). The reciprocal
// r = RN(1/y) is computed once per lane (__drcp_rn, IEEE round-to-nearest) and each
// quotient then costs one multiply and four FMAs:
//
//   q0 = RN(x r);  e0 = x - y q0;  q1 = RN(q0 + e0 r)      (q1 is faithful)
//   e1 = x - y q1 (exact);  q2 = RN(q1 + e1 r) = RN(x / y)
//
// The last step is Markstein's theorem (P. Markstein, "Computation of elementary functions
// on the IBM RISC System/6000 processor", IBM J. Res. Dev. 34(1), 1990; also Muller et
// al., Handbook of Floating-Point Arithmetic, the FMA-based division section): if q is a
// faithful approximation of x/y and r approximates 1/y within a relative error below
// 2^-53, then the remainder x - y q is exactly representable and RN(q + r (x - y q)) is
// the correctly rounded quotient, provided nothing overflows or underflows. So every
// quotient is bit-identical to IEEE x / y. The fast path is taken only when both
// exponents lie in [-500, 500] (so the quotient, the remainders and the products stay
// normal and finite); zero dividends return x * r (a signed zero, as x / y); anything
// else (zero, subnormal, huge, inf or NaN operands) uses the native division.
// fct_div_check (fct_producers.cu) compares this against native division bit for bit.
#pragma once

namespace fct {

__device__ __forceinline__ bool div_exp_ok(double v) {
  const unsigned be = (unsigned(__double2hiint(v)) >> 20) & 0x7ffu;
  return be - 523u <= 1000u;   // unbiased exponent in [-500, 500]
}

struct Rcp {
  double y, r;
  bool ok;
};

__device__ __forceinline__ Rcp rcp(double y) {
  Rcp c;
  c.y = y;
  c.ok = div_exp_ok(y);
  c.r = c.ok ? __drcp_rn(y) : 0.0;
  return c;
}

// The native division for the operands the fast path does not take. Kept out of line so
// that the compiler branches around it instead of evaluating it under a predicate at
// every call site.
static __device__ __noinline__ double div_slow(double x, double y) { return x / y; }

// x / c.y, correctly rounded (IEEE round-to-nearest-even)
__device__ __forceinline__ double divr(double x, const Rcp& c) {
  if (c.ok) {
    if (x == 0.0) return x * c.r;
    if (div_exp_ok(x)) {
      const double q0 = x * c.r;
      const double q1 = fma(fma(-c.y, q0, x), c.r, q0);
      return fma(fma(-c.y, q1, x), c.r, q1);
    }
  }
  return div_slow(x, c.y);
}

}  // namespace fct
