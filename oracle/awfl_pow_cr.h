/* Correctly rounded pow/exp for the CPU test oracles (TEST INFRASTRUCTURE ONLY).
 *
 * The same algorithm as the library's device pow (awflcloud_b200/csrc/awfl_pow.cuh):
 * Tang's table-driven logarithm and exponential (ACM TOMS 1989/1990) in double-double
 * arithmetic, written in plain C with fma(): ln x through a
 * 128-entry table and a degree-9 log1p series, exp through 2^(j/64) and a degree-8
 * series, ~2^-75 relative before the single final rounding.
 *
 * Used to build oracle variants whose only difference from the reference's CPU build is
 * the rounding of pow/exp: glibc's pow is not correctly rounded in ~0.08% of calls
 * (measured against 200-bit values), and the scheme amplifies those last-bit
 * differences into ~1e-12 relative differences of the perturbation fields. With a
 * correctly rounded pow on both sides the GPU FP64 path and the CPU arithmetic agree
 * bit for bit.
 */
#ifndef AWFL_POW_CR_H
#define AWFL_POW_CR_H

#include <math.h>
#include <stdint.h>
#include <string.h>

#include "../awflcloud_b200/csrc/awfl_pow_tables.h"

static inline double awfl_t_ll2d(int64_t v) { double d; memcpy(&d, &v, 8); return d; }
static inline int64_t awfl_t_d2ll(double v) { int64_t d; memcpy(&d, &v, 8); return d; }

static inline void awfl_t_two_sum(double a, double b, double *s, double *e) {
  double ss = a + b, bb = ss - a;
  *e = (a - (ss - bb)) + (b - bb);
  *s = ss;
}

static inline void awfl_t_fast_two_sum(double a, double b, double *s, double *e) {
  double ss = a + b;
  *e = b - (ss - a);
  *s = ss;
}

static inline double awfl_t_exp_core(double z_hi, double z_lo) {
  const double kd = nearbyint(z_hi * AWFL_POW_INV_E);
  const int k = (int)kd;
  const double d1 = z_hi - kd * AWFL_POW_E1;
  const double d2_hi = kd * AWFL_POW_E2;
  const double d2_lo = fma(kd, AWFL_POW_E2, -d2_hi);
  double s_hi, s_e, s_lo;
  awfl_t_two_sum(d1, -d2_hi, &s_hi, &s_e);
  s_lo = (s_e - d2_lo) + z_lo;
  awfl_t_two_sum(s_hi, s_lo, &s_hi, &s_lo);
  double Q = 1.0 / 40320.0;
  Q = fma(Q, s_hi, 1.0 / 5040.0);
  Q = fma(Q, s_hi, 1.0 / 720.0);
  Q = fma(Q, s_hi, 1.0 / 120.0);
  Q = fma(Q, s_hi, 1.0 / 24.0);
  Q = fma(Q, s_hi, 1.0 / 6.0);
  const double q_hi = s_hi * s_hi;
  const double q_lo = fma(s_hi, s_hi, -q_hi);
  double h1, l1, h2, l2, E_hi, E_lo;
  awfl_t_two_sum(1.0, s_hi, &h1, &l1);
  awfl_t_two_sum(h1, 0.5 * q_hi, &h2, &l2);
  const double tail = ((s_hi * q_hi) * Q + 0.5 * q_lo) + s_lo * (1.0 + s_hi);
  E_lo = (l1 + l2) + tail;
  awfl_t_fast_two_sum(h2, E_lo, &E_hi, &E_lo);
  const int jj = k & 63;
  const int mexp = (k - jj) / 64;
  const double T_hi = awfl_pow_exp_hi[jj], T_lo = awfl_pow_exp_lo[jj];
  const double R_hi = T_hi * E_hi;
  const double R_lo = fma(T_hi, E_hi, -R_hi) + (T_hi * E_lo + T_lo * E_hi);
  const double res = R_hi + R_lo;
  return res * awfl_t_ll2d((int64_t)(mexp + 1023) << 52);
}

static inline double awfl_test_pow_cr(double x, double y) {
  if (!(x >= 0x1p-1000 && x <= 0x1p1000) || !(fabs(y) < 0x1p20)) return pow(x, y);
  const int64_t bits = awfl_t_d2ll(x);
  const int e = (int)((bits >> 52) & 0x7ff) - 1023;
  const double m = awfl_t_ll2d((bits & 0x000fffffffffffffLL) | 0x3ff0000000000000LL);
  const int j = (int)((bits >> 45) & 127);
  const double inv = awfl_pow_log_inv[j];
  const double p_hi = m * inv;
  const double p_lo = fma(m, inv, -p_hi);
  double r, r_lo;
  awfl_t_fast_two_sum(p_hi - 1.0, p_lo, &r, &r_lo);
  const double sq_hi = r * r;
  const double sq_lo = fma(r, r, -sq_hi);
  double P = 1.0 / 9.0;
  P = fma(P, r, -1.0 / 8.0);
  P = fma(P, r, 1.0 / 7.0);
  P = fma(P, r, -1.0 / 6.0);
  P = fma(P, r, 1.0 / 5.0);
  P = fma(P, r, -1.0 / 4.0);
  P = fma(P, r, 1.0 / 3.0);
  double s_hi, s_lo;
  awfl_t_fast_two_sum(r, -0.5 * sq_hi, &s_hi, &s_lo);
  s_lo = s_lo + ((-0.5 * sq_lo + (r * sq_hi) * P) + (r_lo - r * r_lo));
  const double A = (double)e * AWFL_POW_L2HI;
  double a1, a2, b1, b2, L_hi, L_lo;
  awfl_t_two_sum(A, awfl_pow_log_hi[j], &a1, &a2);
  awfl_t_two_sum(a1, s_hi, &b1, &b2);
  const double lo = ((a2 + b2) + (s_lo + awfl_pow_log_lo[j])) + (double)e * AWFL_POW_L2LO;
  awfl_t_two_sum(b1, lo, &L_hi, &L_lo);
  double z_hi = y * L_hi;
  double z_lo = fma(y, L_hi, -z_hi) + y * L_lo;
  awfl_t_fast_two_sum(z_hi, z_lo, &z_hi, &z_lo);
  if (!(fabs(z_hi) < 700.0)) return pow(x, y);
  return awfl_t_exp_core(z_hi, z_lo);
}

static inline double awfl_test_exp_cr(double z) {
  if (!(fabs(z) < 700.0)) return exp(z);
  return awfl_t_exp_core(z, 0.0);
}

#endif
