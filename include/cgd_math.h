/*
 * cgd_math.h - elementary functions used on the hot path (pressure closure
 * and the column Jacobian), written once and compiled for both the host and
 * the device so that every compiler evaluates exactly the same sequence of
 * IEEE-754 double operations.
 *
 * Why this exists: the dry equation of state
 *     p = p0 * exp(log(Rd*rhotheta/p0) / (1 - kappa))
 * (reference: src/Models/Equation.jl:25-38, fast_powGPU at Equation.jl:79)
 * feeds the vertical pressure gradient, where a one-ulp change of p near the
 * surface moves the w tendency by ~1e-13 m/s^2.  Using the same exp/log on
 * both sides keeps the GPU kernels bit-identical to the CPU restatement.
 *
 * Methods (from the mathematics, not from any vendor library):
 *   exp: Cody & Waite argument reduction x = k*ln2 + r, |r| <= ln2/2, with
 *        ln2 split into a 21-bit head (k*head exact) and a tail; exp(r) by
 *        its Taylor series to degree 13 in Horner form; scaling by 2^k.
 *   log: x = m * 2^e with m in [sqrt(1/2), sqrt(2)); log(m) = 2*atanh(s),
 *        s = (m-1)/(m+1), atanh by its Taylor series in s^2 to degree 23;
 *        e*ln2 added in head/tail form.
 *   pow: exp(y*log(x)) (only used for x in (0, 2], |y| < 2 on this path).
 * Accuracy is checked against the C library in tests/test_abi_and_math.py (<= 2 ulp).
 *
 * All arithmetic must be compiled without floating-point contraction
 * (host: -ffp-contract=off; device: -fmad=false) for the bit-exactness claim.
 */
#ifndef CGD_MATH_H
#define CGD_MATH_H

#ifdef __CUDACC__
#define CGD_HD __host__ __device__ __forceinline__
#else
#define CGD_HD static inline
#include <math.h>
#endif

/* ln2 = 0.693147180559945309417232121458... split as head + tail */
#define CGD_LN2_HI 0.6931467056274414        /* 0x3FE62E4200000000, 21 bits */
#define CGD_LN2_LO 4.7493250390316726e-07
#define CGD_INV_LN2 1.4426950408889634
#define CGD_SQRT_HALF 0.7071067811865476

CGD_HD double cgd_exp(double x)
{
  if (x != x) return x;                       /* NaN */
  if (x > 709.782712893384) return 1.0 / 0.0; /* overflow */
  if (x < -745.1332191019412) return 0.0;     /* underflow */
  double kd = rint(x * CGD_INV_LN2);
  double r = (x - kd * CGD_LN2_HI) - kd * CGD_LN2_LO;
  /* Taylor coefficients 1/i!, i = 13 .. 0 */
  double q = 1.6059043836821613e-10;
  q = q * r + 2.08767569878681e-09;
  q = q * r + 2.505210838544172e-08;
  q = q * r + 2.755731922398589e-07;
  q = q * r + 2.7557319223985893e-06;
  q = q * r + 2.48015873015873e-05;
  q = q * r + 0.0001984126984126984;
  q = q * r + 0.001388888888888889;
  q = q * r + 0.008333333333333333;
  q = q * r + 0.041666666666666664;
  q = q * r + 0.16666666666666666;
  q = q * r + 0.5;
  q = q * r;            /* r/2 + r^2/6 + ... */
  q = q * r + r;        /* r + r^2/2 + ... = expm1(r) */
  double e = 1.0 + q;
  return ldexp(e, (int)kd);
}

CGD_HD double cgd_log(double x)
{
  if (x != x) return x;
  if (x < 0.0) return 0.0 / 0.0;
  if (x == 0.0) return -1.0 / 0.0;
  if (x > 1.7976931348623157e308) return x;   /* +inf */
  int e;
  double m = frexp(x, &e);                    /* m in [0.5, 1) */
  if (m < CGD_SQRT_HALF) { m = m * 2.0; e = e - 1; }
  double f = m - 1.0;                          /* exact (Sterbenz) */
  double s = f / (2.0 + f);
  double t = s * s;
  /* atanh(s)/s - 1 = t/3 + t^2/5 + ... + t^11/23 */
  double q = 0.043478260869565216;
  q = q * t + 0.047619047619047616;
  q = q * t + 0.05263157894736842;
  q = q * t + 0.058823529411764705;
  q = q * t + 0.06666666666666667;
  q = q * t + 0.07692307692307693;
  q = q * t + 0.09090909090909091;
  q = q * t + 0.1111111111111111;
  q = q * t + 0.14285714285714285;
  q = q * t + 0.2;
  q = q * t + 0.3333333333333333;
  q = q * t;
  /* log(m) = 2s + 2s*q ; 2s = f - f*s (exact identity 2s = f - s*f) */
  double two_s = f - s * f;
  double logm = two_s + two_s * q;
  double ed = (double)e;
  return ed * CGD_LN2_HI + (ed * CGD_LN2_LO + logm);
}

CGD_HD double cgd_pow(double x, double y)
{
  return cgd_exp(y * cgd_log(x));
}

/* min/max with the IEEE semantics of the reference language (a NaN operand
 * propagates; -0 < +0) - used by the limited upwind reconstruction. */
CGD_HD double cgd_min(double x, double y)
{
  if (x != x) return x;
  if (y != y) return y;
  if (y < x) return y;
  if (y == x && signbit(y) && !signbit(x)) return y;
  return x;
}

CGD_HD double cgd_max(double x, double y)
{
  if (x != x) return x;
  if (y != y) return y;
  if (y > x) return y;
  if (y == x && !signbit(y) && signbit(x)) return y;
  return x;
}

CGD_HD float cgd_minf(float x, float y)
{
  if (x != x) return x;
  if (y != y) return y;
  if (y < x) return y;
  if (y == x && signbit(y) && !signbit(x)) return y;
  return x;
}

CGD_HD float cgd_maxf(float x, float y)
{
  if (x != x) return x;
  if (y != y) return y;
  if (y > x) return y;
  if (y == x && !signbit(y) && signbit(x)) return y;
  return x;
}

#endif /* CGD_MATH_H */
