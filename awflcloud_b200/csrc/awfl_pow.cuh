// Correctly rounded (in all but ~2^-20 of cases) pow(x, y) and exp(z) for the FP64
// parity path.
//
// Why: the reference's CPU build calls glibc's pow, which rounds correctly in nearly all
// cases. The scheme's fluxes are sums of O(rho*cs) terms that cancel to O(1e-4), so a
// 1-ulp difference in any pow shows up at ~1e-10 relative in the density tendency.
// Evaluating pow to ~2^-75 relative and rounding once makes the GPU results agree with
// the reference bit for bit except in the rare near-midpoint cases.
//
// Method: Tang's table-driven logarithm and exponential (P. T. P. Tang, "Table-driven
// implementation of the exponential function in IEEE floating-point arithmetic", ACM TOMS
// 15(2), 1989; "... of the logarithm function", ACM TOMS 16(4), 1990) carried out in
// double-double arithmetic (Dekker's exact product by FMA, Knuth's two-sum); the tables
// and the Taylor coefficients are this library's own:
//   x = 2^e * m, m in [1,2); j = top 7 bits of m; r = m*inv_j - 1 exactly as a
//   double-double (inv_j ~ 1/(1+(j+1/2)/128), |r| <= 2^-8);
//   ln x = e*ln2 - ln(inv_j) + log1p(r), log1p by its Taylor series through r^9 with the
//   first two terms in double-double;
//   z = y*ln x (double-double); z = k*ln2/64 + s, |s| <= ln2/128;
//   exp(z) = 2^(k>>6) * 2^((k&63)/64) * exp(s), exp(s) by its Taylor series through s^8.
// Tables (awfl_pow_tables.h) are generated from 256-bit values by gen_tables.py.
// Outside the fast domain (x not a positive normal in [2^-1000, 2^1000], |y| >= 2^20,
// or a result near overflow/underflow) it falls back to the CUDA math library's pow/exp.
#pragma once

#include "awfl_pow_tables.h"

namespace awfl {

__device__ __forceinline__ void dd_two_sum(double a, double b, double &s, double &e) {
  s = __dadd_rn(a, b);
  const double bb = __dsub_rn(s, a);
  e = __dadd_rn(__dsub_rn(a, __dsub_rn(s, bb)), __dsub_rn(b, bb));
}

__device__ __forceinline__ void dd_fast_two_sum(double a, double b, double &s, double &e) {  // |a| >= |b|
  s = __dadd_rn(a, b);
  e = __dsub_rn(b, __dsub_rn(s, a));
}

// exp of the double-double z_hi + z_lo; requires |z_hi| < 708.
__device__ __forceinline__ double exp_dd_core(double z_hi, double z_lo) {
  const double kd = rint(z_hi * AWFL_POW_INV_E);
  const int k = (int)kd;
  const double d1 = __dsub_rn(z_hi, kd * AWFL_POW_E1);  // exact: kd*E1 has <= 53 bits, Sterbenz
  const double d2_hi = __dmul_rn(kd, AWFL_POW_E2);
  const double d2_lo = __fma_rn(kd, AWFL_POW_E2, -d2_hi);
  double s_hi, s_e;
  dd_two_sum(d1, -d2_hi, s_hi, s_e);
  double s_lo = __dadd_rn(__dsub_rn(s_e, d2_lo), z_lo);
  dd_two_sum(s_hi, s_lo, s_hi, s_lo);
  // exp(s) = 1 + s + s^2/2 + s^3 * Q(s)
  double Q = 1.0 / 40320.0;
  Q = __fma_rn(Q, s_hi, 1.0 / 5040.0);
  Q = __fma_rn(Q, s_hi, 1.0 / 720.0);
  Q = __fma_rn(Q, s_hi, 1.0 / 120.0);
  Q = __fma_rn(Q, s_hi, 1.0 / 24.0);
  Q = __fma_rn(Q, s_hi, 1.0 / 6.0);
  const double q_hi = __dmul_rn(s_hi, s_hi);
  const double q_lo = __fma_rn(s_hi, s_hi, -q_hi);
  double h1, l1, h2, l2;
  dd_two_sum(1.0, s_hi, h1, l1);
  dd_two_sum(h1, 0.5 * q_hi, h2, l2);
  const double tail = __dadd_rn(__dadd_rn(__dmul_rn(__dmul_rn(s_hi, q_hi), Q), 0.5 * q_lo),
                                __dmul_rn(s_lo, __dadd_rn(1.0, s_hi)));
  double E_lo = __dadd_rn(__dadd_rn(l1, l2), tail);
  double E_hi;
  dd_fast_two_sum(h2, E_lo, E_hi, E_lo);
  const int jj = k & 63;
  const int mexp = (k - jj) / 64;
  const double T_hi = awfl_pow_exp_hi[jj], T_lo = awfl_pow_exp_lo[jj];
  const double R_hi = __dmul_rn(T_hi, E_hi);
  const double R_lo = __dadd_rn(__fma_rn(T_hi, E_hi, -R_hi), __dadd_rn(__dmul_rn(T_hi, E_lo), __dmul_rn(T_lo, E_hi)));
  const double res = __dadd_rn(R_hi, R_lo);
  return __dmul_rn(res, __longlong_as_double((long long)(mexp + 1023) << 52));
}

__device__ __forceinline__ double pow_cr(double x, double y) {
  if (!(x >= 0x1p-1000 && x <= 0x1p1000) || !(fabs(y) < 0x1p20)) return pow(x, y);
  const long long bits = __double_as_longlong(x);
  const int e = (int)((bits >> 52) & 0x7ff) - 1023;
  const double m = __longlong_as_double((bits & 0x000fffffffffffffLL) | 0x3ff0000000000000LL);
  const int j = (int)((bits >> 45) & 127);
  const double inv = awfl_pow_log_inv[j];
  const double p_hi = __dmul_rn(m, inv);
  const double p_lo = __fma_rn(m, inv, -p_hi);
  double r, r_lo;
  dd_fast_two_sum(__dsub_rn(p_hi, 1.0), p_lo, r, r_lo);  // p_hi - 1 is exact
  const double sq_hi = __dmul_rn(r, r);
  const double sq_lo = __fma_rn(r, r, -sq_hi);
  double P = 1.0 / 9.0;
  P = __fma_rn(P, r, -1.0 / 8.0);
  P = __fma_rn(P, r, 1.0 / 7.0);
  P = __fma_rn(P, r, -1.0 / 6.0);
  P = __fma_rn(P, r, 1.0 / 5.0);
  P = __fma_rn(P, r, -1.0 / 4.0);
  P = __fma_rn(P, r, 1.0 / 3.0);
  double s_hi, s_lo;
  dd_fast_two_sum(r, -0.5 * sq_hi, s_hi, s_lo);
  s_lo = __dadd_rn(s_lo, __dadd_rn(__dadd_rn(-0.5 * sq_lo, __dmul_rn(__dmul_rn(r, sq_hi), P)),
                                   __dsub_rn(r_lo, __dmul_rn(r, r_lo))));
  // ln x = e*ln2 + (-ln inv_j) + log1p(r)
  const double A = __dmul_rn((double)e, AWFL_POW_L2HI);  // exact (L2HI has 42 bits)
  double a1, a2, b1, b2;
  dd_two_sum(A, awfl_pow_log_hi[j], a1, a2);
  dd_two_sum(a1, s_hi, b1, b2);
  const double lo = __dadd_rn(__dadd_rn(__dadd_rn(a2, b2), __dadd_rn(s_lo, awfl_pow_log_lo[j])),
                              __dmul_rn((double)e, AWFL_POW_L2LO));
  double L_hi, L_lo;
  dd_two_sum(b1, lo, L_hi, L_lo);
  // z = y * ln x
  double z_hi = __dmul_rn(y, L_hi);
  double z_lo = __dadd_rn(__fma_rn(y, L_hi, -z_hi), __dmul_rn(y, L_lo));
  dd_fast_two_sum(z_hi, z_lo, z_hi, z_lo);
  if (!(fabs(z_hi) < 700.0)) return pow(x, y);
  return exp_dd_core(z_hi, z_lo);
}

__device__ __forceinline__ double exp_cr(double z) {
  if (!(fabs(z) < 700.0)) return exp(z);
  return exp_dd_core(z, 0.0);
}

}  // namespace awfl
