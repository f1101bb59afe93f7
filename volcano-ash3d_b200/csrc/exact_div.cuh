// exact_div.cuh -- correctly rounded double division without a branchy
// library call in the common case.
//
// The transport path needs quotients that are bit-identical to IEEE division
// (the limiter's theta = dqu/dq, src/AdvectionHorz_DCU.f90:204, and the back
// substitution of the tridiagonal solve).  Method: Goldschmidt's iteration
// (R. E. Goldschmidt, "Applications of division by convergence", MIT thesis
// 1964) for the quotient, then Markstein's correction step (Markstein,
// "Computation of elementary functions on the IBM RISC System/6000
// processor", IBM J. R&D 1990; Muller et al., Handbook of Floating-Point
// Arithmetic, ch. 5):
//   y  ~ 1/b from the hardware reciprocal approximation (PTX
//        rcp.approx.ftz.f64), e = 1 - b*y (exact with an FMA);
//   q  = a*y*(1 + e)*(1 + e^2): relative error e^4, the two products and
//        y' = y*(1 + e) formed side by side, so the dependent chain after
//        the estimate is five operations instead of the seven of two
//        sequential Newton-Raphson steps on y;
//   r  = a - b*q (exact with an FMA);  q = q + r*y'.
// The result is then certified exactly: r = a - b*q is computed again with an
// FMA, and q is accepted only if |r| < |b| * ulp(q)/2, i.e. the true quotient
// lies strictly inside the rounding interval of q, and q is not a power of two
// (whose rounding interval is asymmetric).  Everything else -- operands
// outside the fast ranges below, a zero divisor, non-finite values, a residual
// on or beyond the half-ulp bound -- falls back to the IEEE division operator.
// A zero dividend over an in-range divisor returns a*b, the zero whose sign
// IEEE division gives (the signs' exclusive or).  Every path therefore
// returns RN(a/b) exactly.
//
// The fast ranges keep every intermediate normal and the residual exact.
// With q within an ulp or two of a/b, r = a - b*q is a multiple of
// ulp(b)*ulp(q) = 2^(e_b+e_q-104) smaller than |b|*ulp(q) < 2^(e_b+e_q-51), so
// it is a double whenever 2^(e_b+e_q-104) >= 2^-1074, i.e. e_a (which is
// e_b+e_q or one more) >= -969; ulp(q)/2 = 2^(e_q-53) must be normal
// (e_q >= -969), and nothing may overflow.  Both ranges below give e_a and
// e_q in [-951, 951]:
//   div_rn:     |b| in [2^-200, 2^201), |a| in [2^-700, 2^701) or a = 0
//               (the limiter's theta = dqu/dq divides only when |dq| >= the
//               cycle threshold, 1e-10 in the reference);
//   div_rn_rcp: |b| in [2^-50, 2^51), |a| in [2^-900, 2^901) or a = 0
//               (the back substitution's pivots D' are >= 1 on the
//               diagonally dominant Crank-Nicolson matrices, and its
//               dividends run down the diffused tails of a cloud).
#pragma once

namespace a3g {

// The IEEE division operator for the rare operands the fast path does not
// certify, kept out of line so that its code is not repeated at every call
// site (the sweeps inline many divisions).  A translation unit that measured
// faster with it inlined defines A3G_DIV_FALLBACK_INLINE first.
#if defined(A3G_HOST_TEST)
// A host build of this header (the CPU test of the certification) supplies
// its own reciprocal estimates, including deliberately poor ones, and counts
// the quotients that were not certified.
double host_rcp_estimate(double b);
long &host_fallback_count();
static inline double ieee_div(double a, double b) {
  ++host_fallback_count();
  return a / b;
}
#elif defined(A3G_DIV_FALLBACK_INLINE)
static __device__ __forceinline__ double ieee_div(double a, double b) { return a / b; }
#else
static __device__ __noinline__ double ieee_div(double a, double b) { return a / b; }
#endif

__device__ __forceinline__ double rcp_approx(double b) {
#ifdef A3G_HOST_TEST
  return host_rcp_estimate(b);
#else
  double y;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(b));
  return y;
#endif
}

// True when the binary exponent of x lies in [LO, HI] (or x is zero and
// ALLOW_ZERO).
template <int LO, int HI, bool ALLOW_ZERO>
__device__ __forceinline__ bool exp_in(double x) {
  const unsigned e = ((unsigned)__double2hiint(x) >> 20) & 0x7ffu;
  return (e - (unsigned)(1023 + LO)) <= (unsigned)(HI - LO) || (ALLOW_ZERO && x == 0.0);
}

// Certifies q against a/b (see above); returns true if q == RN(a/b).
__device__ __forceinline__ bool certified(double a, double b, double q) {
  const double r = fma(-b, q, a);
  const long long qb = __double_as_longlong(q);
  const long long ex = qb & 0x7ff0000000000000LL;
  const double half_ulp = __longlong_as_double(ex - (53LL << 52));  // 2^(e_q - 53)
  const bool pow2 = (qb & 0x000fffffffffffffLL) == 0;
  return fabs(r) < fabs(b) * half_ulp && !pow2;
}

// RN(a/b).
__device__ __forceinline__ double div_rn(double a, double b) {
  if (!(exp_in<-200, 200, false>(b) && exp_in<-700, 700, true>(a))) return ieee_div(a, b);
  if (a == 0.0) return a * b;  // +-0 with the quotient's sign (b finite, nonzero)
  double y = rcp_approx(b);
  const double e = fma(-b, y, 1.0);
  double q = a * y;
  const double e2 = e * e;
  q = fma(q, e, q);
  y = fma(y, e, y);
  q = fma(q, e2, q);
  const double r = fma(-b, q, a);
  q = fma(r, y, q);
  if (certified(a, b, q)) return q;
  return ieee_div(a, b);
}

// RN(a/b) given y = RN(1/b) (precomputed once for a divisor shared by many
// quotients, e.g. a tridiagonal pivot).
__device__ __forceinline__ double div_rn_rcp(double a, double b, double y) {
  if (!(exp_in<-50, 50, false>(b) && exp_in<-900, 900, true>(a))) return ieee_div(a, b);
  if (a == 0.0) return a * b;  // +-0 with the quotient's sign (b finite, nonzero)
  double q = a * y;
  const double r = fma(-b, q, a);
  q = fma(r, y, q);
  if (certified(a, b, q)) return q;
  return ieee_div(a, b);
}

}  // namespace a3g
