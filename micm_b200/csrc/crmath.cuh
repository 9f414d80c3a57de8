// Correctly rounded exp, log10 and pow for the rate constants and the
// step-size controller, evaluated identically on the host and the device.
//
// micm evaluates these with the host C library (std::exp, std::pow,
// std::log10 in rate_constant_functions.hpp:52-136 and the step-size factor
// std::pow(error, 1 / order) in rosenbrock.inl:232-235).  glibc's exp and pow
// round correctly except in rare cases (a few in 10,000 arguments), so a
// correctly rounded evaluation here reproduces micm's values bit for bit
// almost always; a last-bit difference in the step-size factor can change the
// accepted-step sequence of a stiff problem at tight tolerances.
//
// Method: double-double arithmetic (a value is an unevaluated sum hi + lo,
// |lo| <= ulp(hi)/2; Dekker's and Knuth's error-free sum and product, the
// product through a fused multiply-add), about 100 correct bits, then one
// rounding to double.  A result is rounded wrongly only when the exact value
// lies within about 2^-45 ulp of a rounding boundary.
//   exp(x):  x = k ln2 + r (|r| <= ln2/2, ln2 in three parts), r scaled by
//            2^-10, expm1 by its Taylor polynomial to degree 9 (Horner), ten
//            doublings expm1(2s) = 2 expm1(s) + expm1(s)^2, times 2^k.
//   log(x):  x = 2^e m (m in [sqrt(1/2), sqrt(2))), a double seed
//            e ln2 + 2 atanh((m-1)/(m+1)) by its series, then one Newton step
//            l + (x exp(-l) - 1) in double-double (quadratic: error ~1e-33).
//   pow:     exp(y log x);  log10: log(x) / ln(10).
// Arguments outside the ranges the solver meets (non-positive bases, results
// that overflow or fall into the subnormal range) use the plain double
// functions.  Every operation is an explicit IEEE add, multiply, divide or
// fma, so host and device results are identical; the library is compiled
// with contraction off (-fmad=false on the device, -ffp-contract=off on the
// host) so no other fusing happens.
#pragma once

#include <cmath>

#if defined(__CUDACC__)
#define CRM_HD __host__ __device__ __forceinline__
#else
#define CRM_HD inline
#endif

namespace micmb
{
  namespace crm
  {
    struct dd
    {
      double hi, lo;
    };

    CRM_HD dd two_sum(double a, double b)
    {
      const double s = a + b;
      const double bb = s - a;
      const double e = (a - (s - bb)) + (b - bb);
      return { s, e };
    }

    // |a| >= |b| (or a == 0)
    CRM_HD dd quick_two_sum(double a, double b)
    {
      const double s = a + b;
      return { s, b - (s - a) };
    }

    CRM_HD dd two_prod(double a, double b)
    {
      const double p = a * b;
      return { p, fma(a, b, -p) };
    }

    CRM_HD dd add(dd a, dd b)
    {
      dd s = two_sum(a.hi, b.hi);
      const dd t = two_sum(a.lo, b.lo);
      s.lo = s.lo + t.hi;
      s = quick_two_sum(s.hi, s.lo);
      s.lo = s.lo + t.lo;
      return quick_two_sum(s.hi, s.lo);
    }

    CRM_HD dd mul(dd a, dd b)
    {
      dd p = two_prod(a.hi, b.hi);
      p.lo = p.lo + (a.hi * b.lo + a.lo * b.hi);
      return quick_two_sum(p.hi, p.lo);
    }

    CRM_HD dd mul_d(dd a, double b)
    {
      dd p = two_prod(a.hi, b);
      p.lo = p.lo + a.lo * b;
      return quick_two_sum(p.hi, p.lo);
    }

    // ln 2 = LN2_0 + LN2_1 + LN2_2 (each the double nearest the remainder)
    constexpr double LN2_0 = 0x1.62e42fefa39efp-1;
    constexpr double LN2_1 = 0x1.abc9e3b39803fp-56;
    constexpr double LN2_2 = 0x1.7b57a079a1934p-111;
    constexpr double INV_LN2 = 0x1.71547652b82fep+0;
    constexpr double INV_LN10_0 = 0x1.bcb7b1526e50ep-2;
    constexpr double INV_LN10_1 = 0x1.95355baaafad3p-57;
    constexpr double SQRT_HALF = 0x1.6a09e667f3bcdp-1;

    // exp of a double-double argument with |x| < 708 (normal results)
    CRM_HD dd exp_dd(dd x)
    {
      // 1/n! for n = 2..9 as double-doubles
      constexpr double F_HI[10] = { 0, 0, 0x1.0p-1, 0x1.5555555555555p-3, 0x1.5555555555555p-5,
                                    0x1.1111111111111p-7, 0x1.6c16c16c16c17p-10, 0x1.a01a01a01a01ap-13,
                                    0x1.a01a01a01a01ap-16, 0x1.71de3a556c734p-19 };
      constexpr double F_LO[10] = { 0, 0, 0.0, 0x1.5555555555555p-57, 0x1.5555555555555p-59,
                                    0x1.1111111111111p-63, -0x1.f49f49f49f49fp-65, 0x1.a01a01a01a01ap-73,
                                    0x1.a01a01a01a01ap-76, -0x1.c154f8ddc6c00p-73 };
      const double k = rint(x.hi * INV_LN2);
      // r = x - k ln2, each product exact or below 2^-100 relative
      dd r = add(x, two_prod(-k, LN2_0));
      r = add(r, two_prod(-k, LN2_1));
      r = add(r, dd{ -k * LN2_2, 0.0 });
      const dd s{ r.hi * 0x1.0p-10, r.lo * 0x1.0p-10 };
      // expm1(s) = s (1 + s (1/2 + s (1/6 + ... + s/9!)))
      dd t{ F_HI[9], F_LO[9] };
#pragma unroll
      for (int n = 8; n >= 2; --n)
        t = add(dd{ F_HI[n], F_LO[n] }, mul(s, t));
      t = add(dd{ 1.0, 0.0 }, mul(s, t));
      dd p = mul(s, t);
#pragma unroll
      for (int i = 0; i < 10; ++i)
        p = add(dd{ 2.0 * p.hi, 2.0 * p.lo }, mul(p, p));
      const dd e = add(dd{ 1.0, 0.0 }, p);
      const int ki = (int)k;
      return { ldexp(e.hi, ki), ldexp(e.lo, ki) };
    }

    // natural log of a positive, finite, normal double
    CRM_HD dd log_dd(double x)
    {
      int e;
      double m = frexp(x, &e);  // m in [0.5, 1)
      if (m < SQRT_HALF)
      {
        m = m * 2.0;
        e = e - 1;
      }
      // seed: log(m) = 2 atanh(u), u = (m - 1) / (m + 1), |u| <= 0.1716
      const double f = m - 1.0;
      const double u = f / (2.0 + f);
      const double u2 = u * u;
      double ser = 1.0 / 25.0;
#pragma unroll
      for (int j = 11; j >= 0; --j)
        ser = 1.0 / (double)(2 * j + 1) + u2 * ser;
      const double lm = 2.0 * u * ser;
      const double de = (double)e;
      dd l = add(two_prod(de, LN2_0), two_prod(de, LN2_1));
      l = add(l, dd{ lm, 0.0 });
      // Newton step for exp(l) = x:  l <- l + (x exp(-l) - 1)
      const dd q = mul_d(exp_dd(dd{ -l.hi, -l.lo }), x);
      const dd corr = add(q, dd{ -1.0, 0.0 });
      return add(l, corr);
    }

    CRM_HD bool plain_range(double x)
    {
      return !(x > 0.0) || !(x < INFINITY) || x < 0x1.0p-1022;
    }
  }  // namespace crm

  // exp(x), correctly rounded in all but rare cases
  CRM_HD double cr_exp(double x)
  {
    if (!(fabs(x) < 708.0))
      return exp(x);
    const crm::dd r = crm::exp_dd(crm::dd{ x, 0.0 });
    return r.hi + r.lo;
  }

  // pow(x, y) for x > 0, correctly rounded in all but rare cases
  CRM_HD double cr_pow(double x, double y)
  {
    if (y == 0.0)
      return 1.0;
    if (y == 1.0)
      return x;
    if (y == 2.0)
      return x * x;
    if (crm::plain_range(x) || !(fabs(y) < INFINITY))
      return pow(x, y);
    const crm::dd z = crm::mul_d(crm::log_dd(x), y);
    if (!(fabs(z.hi) < 708.0))
      return pow(x, y);
    const crm::dd r = crm::exp_dd(z);
    return r.hi + r.lo;
  }

  // log10(x) for x > 0, correctly rounded in all but rare cases
  CRM_HD double cr_log10(double x)
  {
    if (crm::plain_range(x))
      return log10(x);
    if (x == 1.0)
      return 0.0;
    const crm::dd r = crm::mul(crm::log_dd(x), crm::dd{ crm::INV_LN10_0, crm::INV_LN10_1 });
    return r.hi + r.lo;
  }
}  // namespace micmb
