// Correctly rounded exp(x), log(x), x^y and x^(1/4) in FP64, for the
// transport coefficients (zeta/s forms 1-5, src/trancoeff.cpp:19-70),
// EoSChiral's power law, EoSHadron's logarithmic table coordinates and the
// entropy-to-energy inversion of the initial states (src/s95p.cpp:14-40).  The reference
// evaluates them with the host C library, whose exp and pow are accurate to
// about half an ulp; returning the correctly rounded value reproduces the
// library's result except where the exact value lies within ~1e-3 ulp of a
// rounding boundary, while a faithfully rounded device exp (up to 1 ulp)
// differs from it in a sizeable fraction of calls.  Bulk viscosity amplifies
// a last-bit difference by ~1e6 within ten steps near the limiter and the
// vacuum edge, so the last bit matters for parity.
//
// Method (own implementation from the mathematics, double-double arithmetic
// after Dekker (1971) and Knuth's two-sum; constants from
// gen_crmath_consts.py, exact rational arithmetic):
//   exp: k = rint(x / ln 2); r = x - k ln 2 with ln 2 split into three
//        doubles (Cody & Waite 1980); s = r / 2^8; expm1(s) by its Taylor
//        series to s^11 / 11! in double-double (|s| < 1.4e-3, truncation
//        < 2^-125); eight doublings expm1(2a) = 2 expm1(a) + expm1(a)^2;
//        1 + expm1 rounded to nearest once; scaled by 2^k, with the
//        subnormal range rounded to integer multiples of 2^-1074 from the
//        double-double.  Relative error before the final rounding < 2^-98.
//   log: a Newton step on the exp above from a faithful seed (log_cr).
//   x^y: exp of y log(x), both in double-double (pow_cr).
//   x^(1/4): sqrt(x) as a double-double (the correctly rounded square root
//        and its exact residual by fma), its square root the same way, and
//        one rounding of the sum.
// Every operation is an IEEE add, multiply, divide, sqrt or an explicit fma,
// none contracted (the library builds with -fmad=false), so host and device
// compilations of this header give the same bits.
#pragma once

#include <math.h>

#ifdef __CUDACC__
#define VH_CRM __host__ __device__ __forceinline__
#else
#define VH_CRM static inline
#endif

namespace vh {
namespace crm {

struct dd {
  double hi, lo;
};

VH_CRM dd two_sum(double a, double b) {
  const double s = a + b;
  const double bb = s - a;
  const double e = (a - (s - bb)) + (b - bb);
  return {s, e};
}

VH_CRM dd fast_two_sum(double a, double b) {  // |a| >= |b|
  const double s = a + b;
  return {s, b - (s - a)};
}

VH_CRM dd two_prod(double a, double b) {
  const double p = a * b;
  return {p, fma(a, b, -p)};
}

VH_CRM dd add(dd a, dd b) {
  dd s = two_sum(a.hi, b.hi);
  const dd t = two_sum(a.lo, b.lo);
  s.lo += t.hi;
  s = fast_two_sum(s.hi, s.lo);
  s.lo += t.lo;
  return fast_two_sum(s.hi, s.lo);
}

VH_CRM dd mul(dd a, dd b) {
  dd p = two_prod(a.hi, b.hi);
  const double c = a.hi * b.lo;
  const double d = a.lo * b.hi;
  p.lo += c + d;
  return fast_two_sum(p.hi, p.lo);
}

// 2^k for -1022 <= k <= 1023, built from its bit pattern
VH_CRM double pow2i(int k) {
  const long long bits = (long long)(k + 1023) << 52;
#ifdef __CUDA_ARCH__
  return __longlong_as_double(bits);
#else
  double d;
  __builtin_memcpy(&d, &bits, sizeof d);
  return d;
#endif
}

// y * 2^k rounded once, y = hi + lo in [0.7, 1.5), |k| <= 1100
VH_CRM double scale_round(dd y, int k) {
  if (k > 1023) return y.hi * pow2i(1023) * pow2i(k - 1023);  // may overflow to inf
  if (k > -1022) return y.hi * pow2i(k);                        // exact
  // subnormal range: count units of 2^-1074
  const int sh = k + 1074;
  if (sh < -1) return 0.0;  // y 2^k < 2^-1075.4, below half the smallest subnormal
  const double f = sh >= 0 ? pow2i(sh) : 0.5;
  const double zh = y.hi * f, zl = y.lo * f;  // exact
  double n = rint(zh);
  const double rem = (zh - n) + zl;
  if (rem > 0.5) {
    n += 1.0;
  } else if (rem < -0.5) {
    n -= 1.0;
  } else if (rem == 0.5 || rem == -0.5) {  // tie: to even
    const double m = n + (rem > 0 ? 1.0 : -1.0);
    if (fmod(m, 2.0) == 0.0) n = m;
  }
  return n * pow2i(-1022) * pow2i(-52);  // exact: n < 2^53
}

// ln 2 = LN2_1 + LN2_2 + LN2_3 (LN2_1 has 33 significant bits, so k LN2_1
// is exact for |k| < 2^20)
#define VH_CRM_LN2_1 0x1.62e42fef00000p-1
#define VH_CRM_LN2_2 0x1.473de6af278edp-34
#define VH_CRM_LN2_3 -0x1.9ff0342542fc3p-90

// expm1(r) for |r| <= 0.36 as a double-double
VH_CRM dd expm1_dd(dd r) {
  // s = r / 2^8
  const dd s = {r.hi * 0x1p-8, r.lo * 0x1p-8};
  // expm1(s) = s (1 + s/2! + s^2/3! + ... + s^10/11!) by Horner
  const dd c[12] = {{0., 0.},
                    {0x1.0000000000000p+0, 0.},
                    {0x1.0000000000000p-1, 0.},
                    {0x1.5555555555555p-3, 0x1.5555555555555p-57},
                    {0x1.5555555555555p-5, 0x1.5555555555555p-59},
                    {0x1.1111111111111p-7, 0x1.1111111111111p-63},
                    {0x1.6c16c16c16c17p-10, -0x1.f49f49f49f49fp-65},
                    {0x1.a01a01a01a01ap-13, 0x1.a01a01a01a01ap-73},
                    {0x1.a01a01a01a01ap-16, 0x1.a01a01a01a01ap-76},
                    {0x1.71de3a556c734p-19, -0x1.c154f8ddc6c00p-73},
                    {0x1.27e4fb7789f5cp-22, 0x1.cbbc05b4fa99ap-76},
                    {0x1.ae64567f544e4p-26, -0x1.c062e06d1f209p-80}};
  dd p = c[11];
#pragma unroll
  for (int n = 10; n >= 1; n--) p = add(mul(p, s), c[n]);
  dd e = mul(p, s);
  // expm1(2a) = 2 expm1(a) + expm1(a)^2, eight times
#pragma unroll
  for (int j = 0; j < 8; j++) e = add({2. * e.hi, 2. * e.lo}, mul(e, e));
  return e;
}

VH_CRM double exp_cr(double x) {
  if (!(x == x)) return x;  // NaN
  if (x > 709.8) return (double)INFINITY;
  if (x < -746.0) return 0.0;
  const double INV_LN2 = 0x1.71547652b82fep+0;
  const double k = rint(x * INV_LN2);
  // r = x - k ln2 as a double-double
  dd r = two_sum(x, -(k * VH_CRM_LN2_1));  // k * LN2_1 exact
  r = add(r, {-two_prod(k, VH_CRM_LN2_2).hi, -two_prod(k, VH_CRM_LN2_2).lo});
  r = add(r, {-(k * VH_CRM_LN2_3), 0.0});
  const dd y = add({1.0, 0.0}, expm1_dd(r));
  return scale_round(y, (int)k);
}

VH_CRM double from_bits(unsigned long long u) {
#ifdef __CUDA_ARCH__
  return __longlong_as_double((long long)u);
#else
  double d;
  __builtin_memcpy(&d, &u, sizeof d);
  return d;
#endif
}

VH_CRM unsigned long long to_bits(double d) {
#ifdef __CUDA_ARCH__
  return (unsigned long long)__double_as_longlong(d);
#else
  unsigned long long u;
  __builtin_memcpy(&u, &d, sizeof u);
  return u;
#endif
}

// log(x), correctly rounded.  x = m 2^k with m in [0.707, 1.415); the
// platform's log(m) (faithful, on the host or the device) is a seed y0;
// one Newton step on exp, y = y0 + ((m - 1) - expm1(y0)) / exp(y0), with
// m - 1 exact and expm1(y0) a double-double, removes the seed's error (the
// step's own error is of the order of the seed error squared, ~2^-104 |y|);
// then k ln 2 + y in double-double and one rounding.  Seeds that differ by
// an ulp give the same result, so host and device agree.
VH_CRM dd log_dd(double x);

VH_CRM double log_cr(double x) {
  if (!(x > 0.)) return x == 0. ? -(double)INFINITY : (double)NAN;
  if (x == (double)INFINITY) return x;
  return log_dd(x).hi;
}

// log(x) as a double-double for finite x > 0 (relative error ~2^-102):
// the steps of log_cr before its one rounding
VH_CRM dd log_dd(double x) {
  int k = 0;
  if (x < 0x1p-1022) {  // subnormal: scale into the normal range (exact)
    x *= 0x1p54;
    k = -54;
  }
  const unsigned long long u = to_bits(x);
  k += (int)(u >> 52) - 1023;
  double m = from_bits((u & 0x000fffffffffffffull) | 0x3ff0000000000000ull);  // [1, 2)
  if (m > 1.41421356) {
    m *= 0.5;
    k += 1;
  }
  const double y0 = log(m);
  const dd em1 = expm1_dd({y0, 0.});
  const dd d = add({m - 1., 0.}, {-em1.hi, -em1.lo});  // m - 1 exact (Sterbenz)
  const double c = d.hi / (1. + em1.hi);
  const dd y = two_sum(y0, c);
  const double kd = (double)k;
  dd L = add(two_prod(kd, VH_CRM_LN2_2), {kd * VH_CRM_LN2_3, 0.});
  L = add({kd * VH_CRM_LN2_1, 0.}, L);
  return add(L, y);
}

// exp(t.hi + t.lo) for a double-double argument (|t.lo| <= ulp(t.hi)), as
// exp_cr: the low part joins the reduced argument before expm1
VH_CRM double exp_dd_cr(dd t) {
  const double x = t.hi;
  if (!(x == x)) return x;  // NaN
  if (x > 709.8) return (double)INFINITY;
  if (x < -746.0) return 0.0;
  const double INV_LN2 = 0x1.71547652b82fep+0;
  const double k = rint(x * INV_LN2);
  dd r = two_sum(x, -(k * VH_CRM_LN2_1));
  r = add(r, {-two_prod(k, VH_CRM_LN2_2).hi, -two_prod(k, VH_CRM_LN2_2).lo});
  r = add(r, {-(k * VH_CRM_LN2_3), t.lo});
  const dd y = add({1.0, 0.0}, expm1_dd(r));
  return scale_round(y, (int)k);
}

// x^y, correctly rounded but where the exact value lies within ~2^-38 ulp
// of a rounding boundary: exp(y log x) with log x a double-double
// (log_dd), the product y log x a double-double (absolute error below
// 2^-92 while it is in exp's range) and exp_dd_cr.  y = 2 is x * x (one
// rounding of the exact square, which can be a tie).  The C library's
// special values: x^0 = 1 and 1^y = 1 (NaN included), NaN otherwise
// propagates; 0^y = +0 (y > 0) or +inf (y < 0), with -0 kept for odd
// integers y; inf^y = inf or 0; negative x for integer y only (NaN else).
VH_CRM double pow_cr(double x, double y) {
  if (y == 0. || x == 1.) return 1.;
  if (!(x == x) || !(y == y)) return x + y;
  if (y == 2.) return x * x;
  const bool yint = rint(y) == y;
  const bool yodd = yint && fabs(y) < 0x1p53 && fmod(y, 2.0) != 0.;
  if (x == 0.) {
    const double r = y > 0. ? 0. : (double)INFINITY;
    return (yodd && to_bits(x) >> 63) ? -r : r;
  }
  double sgn = 1.;
  if (x < 0.) {
    if (!yint) return (double)NAN;
    if (yodd) sgn = -1.;
    x = -x;
  }
  if (x == (double)INFINITY) return sgn * (y > 0. ? (double)INFINITY : 0.);
  const dd L = log_dd(x);
  const dd t = mul({y, 0.}, L);
  if (t.hi > 709.8) return sgn * (double)INFINITY;
  if (t.hi < -746.0) return sgn * 0.;
  return sgn * exp_dd_cr(t);
}

// x^(1/4) for x >= 0 (x = +0 gives +0, x = inf gives inf)
VH_CRM double root4_cr(double x) {
  if (!(x > 0.) || x == (double)INFINITY) return x < 0. ? (double)NAN : x;
  // a + al = sqrt(x): a correctly rounded, fma(-a, a, x) exact
  const double a = sqrt(x);
  const double al = fma(-a, a, x) / (2. * a);
  // b + bl = sqrt(a + al)
  const double b = sqrt(a);
  const double bl = (fma(-b, b, a) + al) / (2. * b);
  return b + bl;
}

// y / b correctly rounded, from r = RN(1/b), without a divide: the
// quotient q0 = RN(y r) is faithful, the remainder y - b q0 is exact in an
// fma, and RN(q0 + r (y - b q0)) = RN(y / b) (Markstein's theorem, IBM J.
// Res. Dev. 34 (1990); Muller et al., Handbook of Floating-Point
// Arithmetic, the Newton-Raphson division chapter).  It needs nothing to
// underflow or overflow: mk_num_ok(y) (2^-900 <= |y| < 2^900, or y = +-0)
// and mk_den_ok(b) (2^-100 <= b <= 2^100, so b > 0).  Callers test a batch
// of numerators once and divide the IEEE way otherwise, so that a batch of
// quotients is free of branches (a divide is an instruction sequence with a
// branch to a slow path, which keeps independent divides from overlapping).
// Both tests and the sign fix below are bit operations, off the FP64 pipe.
VH_CRM unsigned mk_hi(double y) {
#ifdef __CUDA_ARCH__
  return (unsigned)__double2hiint(y);
#else
  unsigned long long u;
  __builtin_memcpy(&u, &y, sizeof u);
  return (unsigned)(u >> 32);
#endif
}
VH_CRM unsigned mk_lo(double y) {
#ifdef __CUDA_ARCH__
  return (unsigned)__double2loint(y);
#else
  unsigned long long u;
  __builtin_memcpy(&u, &y, sizeof u);
  return (unsigned)u;
#endif
}
// |y| in [2^-900, 2^900): biased exponent in [123, 1922]; or y = +-0
VH_CRM bool mk_num_ok(double y) {
  const unsigned h = mk_hi(y) & 0x7fffffffu;
  return h - (123u << 20) < (1800u << 20) || (h | mk_lo(y)) == 0u;
}
VH_CRM bool mk_den_ok(double b) { return b >= 0x1p-100 && b <= 0x1p100; }
// For y != 0 the quotient has the sign of q0; for y = +-0 (b > 0) the
// divide returns y, which q0 = y r also is, so the sign of q0 is the sign
// of the result in both cases.
VH_CRM double mk_div(double y, double b, double r) {
  const double q0 = y * r;
  const double rem = fma(-q0, b, y);
  return copysign(fma(rem, r, q0), q0);
}

}  // namespace crm
}  // namespace vh

#undef VH_CRM
#undef VH_CRM_LN2_1
#undef VH_CRM_LN2_2
#undef VH_CRM_LN2_3
