// Hand-written discrete adjoint (reverse mode) of one cell's reconstruction and of one
// face's Riemann flux, host + device.
//
// Each *_vjp function re-evaluates its forward part (the linearisation point), keeping
// the intermediates, and then walks them backwards: given the adjoint of the outputs it
// returns the adjoint of the inputs (a vector-Jacobian product). The forward part is the
// same mathematical function as the FP64 path (awfl_device.cuh) but evaluated with
// reciprocals and contracted multiply-adds -- the adjoint is the derivative at the
// trajectory, not a bit-exact replay, and a 1-ulp change of the linearisation point moves
// it by ~1e-16 relative.
//
// Forward arithmetic restated (Spatial = Spatial_euler3d_cons_expl_cart_fv_Agrid.h):
//   weno_vjp      Weno:93-172 compute_weno_coefs (+ map_weights :12-17, convexify :20-25)
//   gll_vjp       Spatial:1800-1833 reconstruct_gll_values
//   cell_vjp      Spatial:665-811 / 1028-1171 / 1385-1552 (recon + hydrostasis + wall),
//                 diffTransformEulerConsX/Y/Z Spatial:1837-2091, compute_timeAvg[_edges]
//                 Spatial:2130-2177, z gravity source quadrature Spatial:1489-1496
//   riemann_vjp   Spatial:842-902 / 1202-1260 / 1583-1644 (y averages not divided by density)
#pragma once

#include <cmath>

#include "awfl_internal.h"
#include "awfl_tv.h"

#if defined(__CUDACC__)
#define AWFL_AHD __host__ __device__ __forceinline__
#define AWFL_UNROLL _Pragma("unroll")
#else
#define AWFL_AHD inline
#define AWFL_UNROLL
#endif

namespace awfl {
namespace adj {

// Reciprocal for the reverse sweeps (a derivative, not a replay of the reference's
// rounding, so about an ulp is enough): on the device the hardware's approximate
// reciprocal (rcp.approx.ftz.f64, ~2^-20 relative) refined by two Newton-Raphson steps
// y <- y + y(1 - x y) (each doubles the correct bits), a few FMAs instead of an IEEE
// division; on the host (the CPU checks of these functions) the plain division.
AWFL_AHD double arcp(double x) {
#if defined(__CUDA_ARCH__)
  double y;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
  y = fma(y, fma(-x, y, 1.0), y);
  return fma(y, fma(-x, y, 1.0), y);
#else
  return 1. / x;
#endif
}

template <int N> AWFL_AHD double tv(const double *a) {
  if constexpr (N == 3) return awfl_tv_n3<double>(a);
  else if constexpr (N == 5) return awfl_tv_n5<double>(a);
  else return awfl_tv_n9<double>(a);
}
template <int N> AWFL_AHD void tv_grad(const double *a, double lam, double *g) {
  if constexpr (N == 3) awfl_tv_grad_n3<double>(a, lam, g);
  else if constexpr (N == 5) awfl_tv_grad_n5<double>(a, lam, g);
  else awfl_tv_grad_n9<double>(a, lam, g);
}

// ---------------------------------------------------------------------------------------
// WENO polynomial coefficients of one stencil, forward only (Weno:93-172).
// ---------------------------------------------------------------------------------------
template <int ORD>
AWFL_AHD void weno_fwd(const Tables<ORD> &T, const double (&u)[ORD], double (&aw)[ORD]) {
  constexpr int HS = (ORD - 1) / 2;
  constexpr double eps = 1.0e-20;
  double a[HS + 2][ORD];
  AWFL_UNROLL for (int i = 0; i < HS + 1; i++) {
    AWFL_UNROLL for (int ii = 0; ii < HS + 1; ii++) {
      double t = 0.;
      AWFL_UNROLL for (int s = 0; s < HS + 1; s++) t += T.recon[(i * ORD + s) * ORD + ii] * u[i + s];
      a[i][ii] = t;
    }
  }
  const double rid = arcp(T.idl[HS + 1]);
  AWFL_UNROLL for (int ii = 0; ii < ORD; ii++) {
    double t = 0.;
    AWFL_UNROLL for (int s = 0; s < ORD; s++) t += T.recon[((HS + 1) * ORD + s) * ORD + ii] * u[s];
    if (ii < HS + 1) {
      AWFL_UNROLL for (int i = 0; i < HS + 1; i++) t -= T.idl[i] * a[i][ii];
    }
    a[HS + 1][ii] = t * rid;
  }
  double tvs[HS + 2];
  double lo = 0.;
  AWFL_UNROLL for (int i = 0; i < HS + 1; i++) {
    tvs[i] = tv<HS + 1>(a[i]);
    lo += tvs[i];
  }
  lo *= 1. / (HS + 1);
  tvs[HS + 1] = lo + (tv<ORD>(a[HS + 1]) - lo) * T.sigma;
  double w[HS + 2], S = 0.;
  AWFL_UNROLL for (int i = 0; i < HS + 2; i++) {
    w[i] = T.idl[i] * arcp(tvs[i] * tvs[i] + eps);
    S += w[i];
  }
  double r = arcp(S + eps);
  S = 0.;
  AWFL_UNROLL for (int i = 0; i < HS + 2; i++) {
    const double x = w[i] * r, d = T.idl[i];
    w[i] = x * (d + d * d - 3. * d * x + x * x) * arcp(d * d + x * (1. - 2. * d));
    S += w[i];
  }
  r = arcp(S + eps);
  AWFL_UNROLL for (int ii = 0; ii < ORD; ii++) {
    double t = 0.;
    AWFL_UNROLL for (int i = 0; i < HS + 2; i++) {
      if (i <= HS && ii > HS) continue;  // lower-order polynomials have degree HS
      t += w[i] * a[i][ii];
    }
    aw[ii] = t * r;
  }
}

// ---------------------------------------------------------------------------------------
// Reverse of weno_fwd: lu += (d aw / d u)^T law.
// ---------------------------------------------------------------------------------------
template <int ORD>
AWFL_AHD void weno_vjp(const Tables<ORD> &T, const double (&u)[ORD], const double (&law)[ORD], double (&lu)[ORD]) {
  constexpr int HS = (ORD - 1) / 2;
  constexpr int NP = HS + 2;
  constexpr double eps = 1.0e-20;
  // ---- forward, keeping intermediates
  double a[NP][ORD];
  AWFL_UNROLL for (int i = 0; i < HS + 1; i++) {
    AWFL_UNROLL for (int ii = 0; ii < HS + 1; ii++) {
      double t = 0.;
      AWFL_UNROLL for (int s = 0; s < HS + 1; s++) t += T.recon[(i * ORD + s) * ORD + ii] * u[i + s];
      a[i][ii] = t;
    }
  }
  const double rid = arcp(T.idl[HS + 1]);
  AWFL_UNROLL for (int ii = 0; ii < ORD; ii++) {
    double t = 0.;
    AWFL_UNROLL for (int s = 0; s < ORD; s++) t += T.recon[((HS + 1) * ORD + s) * ORD + ii] * u[s];
    if (ii < HS + 1) {
      AWFL_UNROLL for (int i = 0; i < HS + 1; i++) t -= T.idl[i] * a[i][ii];
    }
    a[HS + 1][ii] = t * rid;
  }
  double tvs[NP];
  double lo = 0.;
  AWFL_UNROLL for (int i = 0; i < HS + 1; i++) {
    tvs[i] = tv<HS + 1>(a[i]);
    lo += tvs[i];
  }
  lo *= 1. / (HS + 1);
  tvs[HS + 1] = lo + (tv<ORD>(a[HS + 1]) - lo) * T.sigma;
  double w0[NP], dd[NP], S1 = 0.;
  AWFL_UNROLL for (int i = 0; i < NP; i++) {
    dd[i] = arcp(tvs[i] * tvs[i] + eps);
    w0[i] = T.idl[i] * dd[i];
    S1 += w0[i];
  }
  const double r1 = arcp(S1 + eps);
  double w1[NP], w2[NP], S2 = 0.;
  AWFL_UNROLL for (int i = 0; i < NP; i++) {
    const double x = w0[i] * r1, d = T.idl[i];
    w1[i] = x;
    w2[i] = x * (d + d * d - 3. * d * x + x * x) * arcp(d * d + x * (1. - 2. * d));
    S2 += w2[i];
  }
  const double r2 = arcp(S2 + eps);
  // ---- reverse
  double la[NP][ORD];
  double lw[NP];
  AWFL_UNROLL for (int i = 0; i < NP; i++) {
    double t = 0.;
    AWFL_UNROLL for (int ii = 0; ii < ORD; ii++) {
      if (i <= HS && ii > HS) {
        la[i][ii] = 0.;
        continue;
      }
      t += law[ii] * a[i][ii];
      la[i][ii] = w2[i] * r2 * law[ii];
    }
    lw[i] = t;  // adjoint of w3 = w2 * r2
  }
  // w3 = w2 / (S2 + eps)
  {
    double dot = 0.;
    AWFL_UNROLL for (int i = 0; i < NP; i++) dot += lw[i] * w2[i] * r2;
    AWFL_UNROLL for (int i = 0; i < NP; i++) lw[i] = r2 * (lw[i] - dot);
  }
  // mapping w2 = x N(x) / D(x)
  AWFL_UNROLL for (int i = 0; i < NP; i++) {
    const double x = w1[i], d = T.idl[i];
    const double N = d + d * d - 3. * d * x + x * x, D = d * d + x * (1. - 2. * d);
    const double rD = arcp(D);
    const double dm = ((N + x * (2. * x - 3. * d)) - x * N * (1. - 2. * d) * rD) * rD;
    lw[i] *= dm;
  }
  // w1 = w0 / (S1 + eps)
  {
    double dot = 0.;
    AWFL_UNROLL for (int i = 0; i < NP; i++) dot += lw[i] * w1[i];
    AWFL_UNROLL for (int i = 0; i < NP; i++) lw[i] = r1 * (lw[i] - dot);
  }
  // w0 = idl / (tv^2 + eps)
  double ltv[NP];
  AWFL_UNROLL for (int i = 0; i < NP; i++) ltv[i] = -2. * tvs[i] * w0[i] * dd[i] * lw[i];
  // bridge smoothness relaxed toward the low-order mean by sigma
  {
    const double llo = (1. - T.sigma) * ltv[HS + 1];
    ltv[HS + 1] *= T.sigma;
    AWFL_UNROLL for (int i = 0; i < HS + 1; i++) ltv[i] += llo * (1. / (HS + 1));
  }
  AWFL_UNROLL for (int i = 0; i < HS + 1; i++) tv_grad<HS + 1>(a[i], ltv[i], la[i]);
  tv_grad<ORD>(a[HS + 1], ltv[HS + 1], la[HS + 1]);
  // bridge polynomial: a_hi = (raw - sum_i idl_i a_i) / idl_{hs+1}
  double lraw[ORD];
  AWFL_UNROLL for (int ii = 0; ii < ORD; ii++) {
    lraw[ii] = la[HS + 1][ii] * rid;
    if (ii < HS + 1) {
      AWFL_UNROLL for (int i = 0; i < HS + 1; i++) la[i][ii] -= T.idl[i] * lraw[ii];
    }
  }
  AWFL_UNROLL for (int s = 0; s < ORD; s++) {
    double t = 0.;
    AWFL_UNROLL for (int ii = 0; ii < ORD; ii++) t += T.recon[((HS + 1) * ORD + s) * ORD + ii] * lraw[ii];
    lu[s] += t;
  }
  AWFL_UNROLL for (int i = 0; i < HS + 1; i++) {
    AWFL_UNROLL for (int s = 0; s < HS + 1; s++) {
      double t = 0.;
      AWFL_UNROLL for (int ii = 0; ii < HS + 1; ii++) t += T.recon[(i * ORD + s) * ORD + ii] * la[i][ii];
      lu[i + s] += t;
    }
  }
}

// ---------------------------------------------------------------------------------------
// Stencil -> GLL values (Spatial:1800-1833), forward and reverse.
// ---------------------------------------------------------------------------------------
template <int ORD>
AWFL_AHD void gll_fwd(const Tables<ORD> &T, const double (&s)[ORD], bool doweno,
                      double (&out)[OrdTraits<ORD>::NGLL]) {
  constexpr int NG = OrdTraits<ORD>::NGLL;
  double c[ORD];
  if (doweno) weno_fwd<ORD>(T, s, c);
  AWFL_UNROLL for (int ii = 0; ii < NG; ii++) {
    double t = 0.;
    AWFL_UNROLL for (int m = 0; m < ORD; m++) t += (doweno ? T.c2g[m * NG + ii] * c[m] : T.s2g[m * NG + ii] * s[m]);
    out[ii] = t;
  }
}

template <int ORD>
AWFL_AHD void gll_vjp(const Tables<ORD> &T, const double (&s)[ORD], bool doweno,
                      const double (&lout)[OrdTraits<ORD>::NGLL], double (&ls)[ORD]) {
  constexpr int NG = OrdTraits<ORD>::NGLL;
  if (doweno) {
    double lc[ORD];
    AWFL_UNROLL for (int m = 0; m < ORD; m++) {
      double t = 0.;
      AWFL_UNROLL for (int ii = 0; ii < NG; ii++) t += T.c2g[m * NG + ii] * lout[ii];
      lc[m] = t;
    }
    weno_vjp<ORD>(T, s, lc, ls);
  } else {
    AWFL_UNROLL for (int m = 0; m < ORD; m++) {
      double t = 0.;
      AWFL_UNROLL for (int ii = 0; ii < NG; ii++) t += T.s2g[m * NG + ii] * lout[ii];
      ls[m] += t;
    }
  }
}

// Per-cell constants of the reconstruction (a subset of SweepArgs).
struct CellArgs {
  int nz, bc, weno_s, weno_w;
  double dxd, dt;
  const double *dens_c, *denstheta_c, *dens_g, *denstheta_g, *pres_g;
};

// ---------------------------------------------------------------------------------------
// Forward of one cell: GLL values + ADER differential transform + time averages.
// Returns the edges and, for z, the gravity source average (the linearisation point).
// Q/F/G receive the transform levels when non-null (used by cell_vjp).
// ---------------------------------------------------------------------------------------
template <int ORD, int DIR>
struct CellFwd {
  static constexpr int NG = OrdTraits<ORD>::NGLL;
  static constexpr int NA = NG;
  double q[5][NA][NG];
  double f[4][NA][NG];
  double g[NA][NG];
  double sr[NA][NG];
};

// Level 0 of one cell: GLL values of the five variables, hydrostasis added back, the
// wall's zero normal momentum at a z boundary point.
template <int ORD, int DIR>
AWFL_AHD void cell_level0(const Tables<ORD> &T, const double (&sten)[5][ORD], int kb, const CellArgs &A,
                          double (&q0)[5][OrdTraits<ORD>::NGLL]) {
  constexpr int HS = (ORD - 1) / 2;
  constexpr int NG = OrdTraits<ORD>::NGLL;
  AWFL_UNROLL for (int v = 0; v < 5; v++) {
    const bool doweno = (v == idR || v == idT) ? A.weno_s : A.weno_w;
    gll_fwd<ORD>(T, sten[v], doweno, q0[v]);
  }
  AWFL_UNROLL for (int ii = 0; ii < NG; ii++) {
    if (DIR == 2) {
      q0[idR][ii] += A.dens_g[kb * NG + ii];
      q0[idT][ii] += A.denstheta_g[kb * NG + ii];
    } else {
      q0[idR][ii] += A.dens_c[HS + kb];
      q0[idT][ii] += A.denstheta_c[HS + kb];
    }
  }
  if (DIR == 2 && A.bc == BC_WALL && kb == A.nz - 1) q0[idW][NG - 1] = 0.;
  if (DIR == 2 && A.bc == BC_WALL && kb == 0) q0[idW][0] = 0.;
}

// ADER differential transform of one cell from its level 0 (X.q[v][0][ii] set on entry).
template <int ORD, int DIR>
AWFL_AHD void cell_dt(const Tables<ORD> &T, int kb, const CellArgs &A, CellFwd<ORD, DIR> &X) {
  constexpr int NG = OrdTraits<ORD>::NGLL;
  constexpr int NA = NG;
  constexpr int NM = 1 + DIR;
  const bool wtop = DIR == 2 && A.bc == BC_WALL && kb == A.nz - 1;
  const bool wbot = DIR == 2 && A.bc == BC_WALL && kb == 0;
  AWFL_UNROLL for (int ii = 0; ii < NG; ii++) {
    const double rr = arcp(X.q[idR][0][ii]);
    const double mn = X.q[NM][0][ii] * rr;
    AWFL_UNROLL for (int x = 0; x < 4; x++) X.f[x][0][ii] = mn * X.q[x + 1][0][ii];
    X.g[0][ii] = ::pow(X.q[idT][0][ii], GAMMA);
  }
  if (DIR == 2) {
    const double fill = -(X.q[idR][0][NG - 1] - A.dens_g[kb * NG + NG - 1]) * GRAV;
    AWFL_UNROLL for (int ii = 0; ii < NG; ii++) X.sr[0][ii] = fill;
  }
  const double rdx = arcp(A.dxd);
  AWFL_UNROLL for (int kt = 0; kt < NA - 1; kt++) {
    const double rk = 1. / (kt + 1.);
    const double cg = kt == 0 ? C0 : 0.5 * C0;
    AWFL_UNROLL for (int ii = 0; ii < NG; ii++) {
      double dq[5] = {0., 0., 0., 0., 0.};
      AWFL_UNROLL for (int s = 0; s < NG; s++) {
        const double D = T.deriv[s * NG + ii];
        dq[idR] += D * X.q[NM][kt][s];
        AWFL_UNROLL for (int m = 1; m <= 3; m++) {
          double xm = X.f[m - 1][kt][s];
          if (m == NM) {
            xm += cg * X.g[kt][s];
            if (DIR == 2 && kt == 0) xm -= A.pres_g[kb * NG + s];  // a constant: no adjoint term
          }
          dq[m] += D * xm;
        }
        dq[idT] += D * X.f[3][kt][s];
      }
      AWFL_UNROLL for (int m = 0; m < 5; m++) X.q[m][kt + 1][ii] = -dq[m] * rdx * rk;
      if (DIR == 2) {
        X.q[idW][kt + 1][ii] += X.sr[kt][ii] * rk;
        X.sr[kt + 1][ii] = -X.q[idR][kt + 1][ii] * GRAV;
      }
    }
    if (wtop) X.q[idW][kt + 1][NG - 1] = 0.;
    if (wbot) X.q[idW][kt + 1][0] = 0.;
    AWFL_UNROLL for (int ii = 0; ii < NG; ii++) {
      const double rr0 = arcp(X.q[idR][0][ii]);
      AWFL_UNROLL for (int x = 0; x < 4; x++) {
        double tot = 0.;
        AWFL_UNROLL for (int ir = 0; ir <= kt + 1; ir++) tot += X.q[NM][ir][ii] * X.q[x + 1][kt + 1 - ir][ii];
        AWFL_UNROLL for (int ir = 1; ir <= kt + 1; ir++) tot -= X.q[idR][ir][ii] * X.f[x][kt + 1 - ir][ii];
        X.f[x][kt + 1][ii] = tot * rr0;
      }
      double tg = 0.;
      AWFL_UNROLL for (int ir = 0; ir <= kt; ir++) {
        tg += (kt + 1. - ir) * GAMMA * X.g[ir][ii] * X.q[idT][kt + 1 - ir][ii];
        if (ir > 0) tg -= (kt + 1. - ir) * X.q[idT][ir][ii] * X.g[kt + 1 - ir][ii];
      }
      X.g[kt + 1][ii] = (GAMMA * X.g[0][ii] * X.q[idT][kt + 1][ii] + tg * rk) * arcp(X.q[idT][0][ii]);
    }
  }
}

template <int ORD, int DIR>
AWFL_AHD void cell_fwd(const Tables<ORD> &T, const double (&sten)[5][ORD], int kb, const CellArgs &A,
                       CellFwd<ORD, DIR> &X) {
  constexpr int NG = OrdTraits<ORD>::NGLL;
  double q0[5][NG];
  cell_level0<ORD, DIR>(T, sten, kb, A, q0);
  AWFL_UNROLL for (int v = 0; v < 5; v++)
    AWFL_UNROLL for (int ii = 0; ii < NG; ii++) X.q[v][0][ii] = q0[v][ii];
  cell_dt<ORD, DIR>(T, kb, A, X);
}

// Edges (and z source) of a forward cell record.
template <int ORD, int DIR>
AWFL_AHD void cell_edges(const Tables<ORD> &T, const CellFwd<ORD, DIR> &X, double dt, double (&eL)[5],
                         double (&eR)[5], double &src) {
  constexpr int NG = OrdTraits<ORD>::NGLL;
  constexpr int NA = NG;
  AWFL_UNROLL for (int v = 0; v < 5; v++) {
    double l = X.q[v][0][0], r = X.q[v][0][NG - 1], dm = dt;
    AWFL_UNROLL for (int kt = 1; kt < NA; kt++) {
      l += X.q[v][kt][0] * dm * (1. / (kt + 1.));
      r += X.q[v][kt][NG - 1] * dm * (1. / (kt + 1.));
      dm *= dt;
    }
    eL[v] = l;
    eR[v] = r;
  }
  src = 0.;
  if (DIR == 2) {
    AWFL_UNROLL for (int ii = 0; ii < NG; ii++) {
      double t = X.sr[0][ii], dm = dt;
      AWFL_UNROLL for (int kt = 1; kt < NA; kt++) {
        t += X.sr[kt][ii] * dm * (1. / (kt + 1.));
        dm *= dt;
      }
      src += t * T.wts[ii];
    }
  }
}

// ---------------------------------------------------------------------------------------
// Reverse of one cell
// ---------------------------------------------------------------------------------------
// Reverse of the ADER part: (leL, leR, lsrc) -> lq0, the adjoint of the level-0 values
// (after hydrostasis; zero at a wall's zeroed boundary point). X from cell_dt.
template <int ORD, int DIR>
AWFL_AHD void cell_dt_vjp(const Tables<ORD> &T, int kb, const CellArgs &A, const CellFwd<ORD, DIR> &X,
                          const double (&leL)[5], const double (&leR)[5], double lsrc,
                          double (&lq0)[5][OrdTraits<ORD>::NGLL]) {
  constexpr int NG = OrdTraits<ORD>::NGLL;
  constexpr int NA = NG;
  constexpr int NM = 1 + DIR;
  const bool wtop = DIR == 2 && A.bc == BC_WALL && kb == A.nz - 1;
  const bool wbot = DIR == 2 && A.bc == BC_WALL && kb == 0;

  double lq[5][NA][NG], lf[4][NA][NG], lg[NA][NG], lsr[NA][NG];
  AWFL_UNROLL for (int kt = 0; kt < NA; kt++) {
    AWFL_UNROLL for (int ii = 0; ii < NG; ii++) {
      AWFL_UNROLL for (int v = 0; v < 5; v++) lq[v][kt][ii] = 0.;
      AWFL_UNROLL for (int x = 0; x < 4; x++) lf[x][kt][ii] = 0.;
      lg[kt][ii] = 0.;
      lsr[kt][ii] = 0.;
    }
  }
  // time averages of the edges and of the source
  {
    double dm = 1.;
    AWFL_UNROLL for (int kt = 0; kt < NA; kt++) {
      const double c = kt == 0 ? 1. : dm * (1. / (kt + 1.));
      AWFL_UNROLL for (int v = 0; v < 5; v++) {
        lq[v][kt][0] += leL[v] * c;
        lq[v][kt][NG - 1] += leR[v] * c;
      }
      if (DIR == 2) {
        AWFL_UNROLL for (int ii = 0; ii < NG; ii++) lsr[kt][ii] += lsrc * T.wts[ii] * c;
      }
      dm *= A.dt;
    }
  }
  const double rdx = arcp(A.dxd);
  AWFL_UNROLL for (int kt = NA - 2; kt >= 0; kt--) {
    const double rk = 1. / (kt + 1.);
    const double cg = kt == 0 ? C0 : 0.5 * C0;
    // (f, g) at level kt+1
    AWFL_UNROLL for (int ii = 0; ii < NG; ii++) {
      const double rT0 = arcp(X.q[idT][0][ii]);
      const double lG = lg[kt + 1][ii];
      const double lnum = lG * rT0;
      lq[idT][0][ii] -= lG * X.g[kt + 1][ii] * rT0;
      lg[0][ii] += lnum * GAMMA * X.q[idT][kt + 1][ii];
      lq[idT][kt + 1][ii] += lnum * GAMMA * X.g[0][ii];
      const double ltg = lnum * rk;
      AWFL_UNROLL for (int ir = 0; ir <= kt; ir++) {
        const double c = (kt + 1. - ir) * ltg;
        lg[ir][ii] += c * GAMMA * X.q[idT][kt + 1 - ir][ii];
        lq[idT][kt + 1 - ir][ii] += c * GAMMA * X.g[ir][ii];
        if (ir > 0) {
          lq[idT][ir][ii] -= c * X.g[kt + 1 - ir][ii];
          lg[kt + 1 - ir][ii] -= c * X.q[idT][ir][ii];
        }
      }
      const double rR0 = arcp(X.q[idR][0][ii]);
      AWFL_UNROLL for (int x = 0; x < 4; x++) {
        const double lF = lf[x][kt + 1][ii];
        const double lt = lF * rR0;
        lq[idR][0][ii] -= lF * X.f[x][kt + 1][ii] * rR0;
        AWFL_UNROLL for (int ir = 0; ir <= kt + 1; ir++) {
          lq[NM][ir][ii] += lt * X.q[x + 1][kt + 1 - ir][ii];
          lq[x + 1][kt + 1 - ir][ii] += lt * X.q[NM][ir][ii];
        }
        AWFL_UNROLL for (int ir = 1; ir <= kt + 1; ir++) {
          lq[idR][ir][ii] -= lt * X.f[x][kt + 1 - ir][ii];
          lf[x][kt + 1 - ir][ii] -= lt * X.q[idR][ir][ii];
        }
      }
    }
    // q at level kt+1 from the derivative of level kt
    if (wtop) lq[idW][kt + 1][NG - 1] = 0.;
    if (wbot) lq[idW][kt + 1][0] = 0.;
    AWFL_UNROLL for (int ii = 0; ii < NG; ii++) {
      if (DIR == 2) {
        lq[idR][kt + 1][ii] -= GRAV * lsr[kt + 1][ii];
        lsr[kt][ii] += lq[idW][kt + 1][ii] * rk;
      }
      double ldq[5];
      AWFL_UNROLL for (int m = 0; m < 5; m++) ldq[m] = -lq[m][kt + 1][ii] * rdx * rk;
      AWFL_UNROLL for (int s = 0; s < NG; s++) {
        const double D = T.deriv[s * NG + ii];
        lq[NM][kt][s] += D * ldq[idR];
        AWFL_UNROLL for (int m = 1; m <= 3; m++) {
          lf[m - 1][kt][s] += D * ldq[m];
          if (m == NM) lg[kt][s] += cg * D * ldq[m];
        }
        lf[3][kt][s] += D * ldq[idT];
      }
    }
  }
  // level 0: fluxes and pressure of the GLL values
  AWFL_UNROLL for (int ii = 0; ii < NG; ii++) {
    const double rr = arcp(X.q[idR][0][ii]);
    lq[idT][0][ii] += lg[0][ii] * GAMMA * X.g[0][ii] * arcp(X.q[idT][0][ii]);
    AWFL_UNROLL for (int x = 0; x < 4; x++) {
      const double l0 = lf[x][0][ii] * rr;
      lq[NM][0][ii] += l0 * X.q[x + 1][0][ii];
      lq[x + 1][0][ii] += l0 * X.q[NM][0][ii];
      lq[idR][0][ii] -= l0 * X.f[x][0][ii];
    }
  }
  if (DIR == 2) {
    double t = 0.;
    AWFL_UNROLL for (int ii = 0; ii < NG; ii++) t += lsr[0][ii];
    lq[idR][0][NG - 1] -= GRAV * t;
  }
  if (wtop) lq[idW][0][NG - 1] = 0.;
  if (wbot) lq[idW][0][0] = 0.;
  AWFL_UNROLL for (int v = 0; v < 5; v++)
    AWFL_UNROLL for (int ii = 0; ii < NG; ii++) lq0[v][ii] = lq[v][0][ii];
}

// Reverse of one whole cell: (leL, leR, lsrc) -> lsten += d(eL, eR, src)/d(sten)^T (...).
template <int ORD, int DIR>
AWFL_AHD void cell_vjp(const Tables<ORD> &T, const double (&sten)[5][ORD], int kb, const CellArgs &A,
                       const double (&leL)[5], const double (&leR)[5], double lsrc, double (&lsten)[5][ORD]) {
  constexpr int NG = OrdTraits<ORD>::NGLL;
  CellFwd<ORD, DIR> X;
  cell_fwd<ORD, DIR>(T, sten, kb, A, X);
  double lq0[5][NG];
  cell_dt_vjp<ORD, DIR>(T, kb, A, X, leL, leR, lsrc, lq0);
  AWFL_UNROLL for (int v = 0; v < 5; v++) {
    const bool doweno = (v == idR || v == idT) ? A.weno_s : A.weno_w;
    gll_vjp<ORD>(T, sten[v], doweno, lq0[v], lsten[v]);
  }
}

// ---------------------------------------------------------------------------------------
// Upwind characteristic Riemann flux, forward (fast) and reverse.
// ---------------------------------------------------------------------------------------
template <int DIR>
AWFL_AHD void riemann_fwd(const double (&qL)[5], const double (&qR)[5], double (&F)[5]) {
  constexpr int TA = DIR == 0 ? 1 : 0;
  constexpr int TB = DIR == 2 ? 1 : 2;
  constexpr int QN = 1 + DIR, QA = 1 + TA, QB = 1 + TB;
  const double r = 0.5 * (qL[0] + qR[0]);
  double vel[3], t;
  if (DIR == 1) {
    AWFL_UNROLL for (int k = 0; k < 3; k++) vel[k] = 0.5 * (qL[k + 1] + qR[k + 1]);
    t = 0.5 * (qL[4] + qR[4]);
  } else {
    const double rl = arcp(qL[0]), rr = arcp(qR[0]);
    AWFL_UNROLL for (int k = 0; k < 3; k++) vel[k] = 0.5 * (qL[k + 1] * rl + qR[k + 1] * rr);
    t = 0.5 * (qL[4] * rl + qR[4] * rr);
  }
  const double p = C0 * ::pow(r * t, GAMMA);
  const double cs = ::sqrt(GAMMA * p * arcp(r));
  const double vn = vel[DIR], va = vel[TA], vb = vel[TB];
  const double rt = arcp(t), rc = 0.5 * arcp(cs);
  const double *qU = vn > 0 ? qL : qR;
  const double w1 = qU[0] - qU[4] * rt, w2 = qU[QA] - va * qU[4] * rt, w3 = qU[QB] - vb * qU[4] * rt;
  const double w5 = (vn * qR[0] - qR[QN]) * rc + 0.5 * qR[4] * rt;
  const double w6 = (qL[QN] - vn * qL[0]) * rc + 0.5 * qL[4] * rt;
  const double Q0 = w1 + w5 + w6;
  const double QNv = vn * w1 + (vn - cs) * w5 + (vn + cs) * w6;
  const double QAv = w2 + va * (w5 + w6), QBv = w3 + vb * (w5 + w6), Q4 = t * (w5 + w6);
  const double r0 = arcp(Q0);
  F[0] = QNv;
  F[QN] = QNv * QNv * r0 + C0 * ::pow(Q4, GAMMA);
  F[QA] = QNv * QAv * r0;
  F[QB] = QNv * QBv * r0;
  F[4] = QNv * Q4 * r0;
}

template <int DIR>
AWFL_AHD void riemann_vjp(const double (&qL)[5], const double (&qR)[5], const double (&lF)[5], double (&lqL)[5],
                          double (&lqR)[5]) {
  constexpr int TA = DIR == 0 ? 1 : 0;
  constexpr int TB = DIR == 2 ? 1 : 2;
  constexpr int QN = 1 + DIR, QA = 1 + TA, QB = 1 + TB;
  // ---- forward
  const double r = 0.5 * (qL[0] + qR[0]);
  double vel[3], t;
  const double rl = arcp(qL[0]), rrr = arcp(qR[0]);
  if (DIR == 1) {
    AWFL_UNROLL for (int k = 0; k < 3; k++) vel[k] = 0.5 * (qL[k + 1] + qR[k + 1]);
    t = 0.5 * (qL[4] + qR[4]);
  } else {
    AWFL_UNROLL for (int k = 0; k < 3; k++) vel[k] = 0.5 * (qL[k + 1] * rl + qR[k + 1] * rrr);
    t = 0.5 * (qL[4] * rl + qR[4] * rrr);
  }
  const double p = C0 * ::pow(r * t, GAMMA);
  const double cs = ::sqrt(GAMMA * p * arcp(r));
  const double vn = vel[DIR], va = vel[TA], vb = vel[TB];
  const double rt = arcp(t), rc = 0.5 * arcp(cs);
  const bool left = vn > 0;
  const double *qU = left ? qL : qR;
  const double w1 = qU[0] - qU[4] * rt, w2 = qU[QA] - va * qU[4] * rt, w3 = qU[QB] - vb * qU[4] * rt;
  const double w5 = (vn * qR[0] - qR[QN]) * rc + 0.5 * qR[4] * rt;
  const double w6 = (qL[QN] - vn * qL[0]) * rc + 0.5 * qL[4] * rt;
  const double W = w5 + w6;
  const double Q0 = w1 + W;
  const double QNv = vn * w1 + (vn - cs) * w5 + (vn + cs) * w6;
  const double QAv = w2 + va * W, QBv = w3 + vb * W, Q4 = t * W;
  const double r0 = arcp(Q0);
  const double pw = ::pow(Q4, GAMMA);
  // ---- reverse: fluxes -> characteristic state
  const double lQN = lF[0] + lF[QN] * 2. * QNv * r0 + (lF[QA] * QAv + lF[QB] * QBv + lF[4] * Q4) * r0;
  const double lQ0 = -(lF[QN] * QNv * QNv + lF[QA] * QNv * QAv + lF[QB] * QNv * QBv + lF[4] * QNv * Q4) * r0 * r0;
  const double lQA = lF[QA] * QNv * r0, lQB = lF[QB] * QNv * r0;
  const double lQ4 = lF[QN] * C0 * GAMMA * pw * arcp(Q4) + lF[4] * QNv * r0;
  const double lw1 = lQ0 + vn * lQN, lw2 = lQA, lw3 = lQB;
  const double lWc = lQ0 + va * lQA + vb * lQB + t * lQ4;
  const double lw5 = lWc + (vn - cs) * lQN;
  const double lw6 = lWc + (vn + cs) * lQN;
  double lvn = lQN * (w1 + W);
  double lcs = lQN * (w6 - w5);
  double lva = lQA * W, lvb = lQB * W;
  double lt = lQ4 * W;
  double gL[5] = {0., 0., 0., 0., 0.}, gR[5] = {0., 0., 0., 0., 0.};
  // w5 = (vn qR0 - qRN) / (2 cs) + qR4 / (2 t)
  lvn += lw5 * qR[0] * rc;
  gR[0] += lw5 * vn * rc;
  gR[QN] -= lw5 * rc;
  gR[4] += lw5 * 0.5 * rt;
  lcs -= lw5 * (vn * qR[0] - qR[QN]) * rc * arcp(cs);
  lt -= lw5 * 0.5 * qR[4] * rt * rt;
  // w6 = (qLN - vn qL0) / (2 cs) + qL4 / (2 t)
  lvn -= lw6 * qL[0] * rc;
  gL[0] -= lw6 * vn * rc;
  gL[QN] += lw6 * rc;
  gL[4] += lw6 * 0.5 * rt;
  lcs -= lw6 * (qL[QN] - vn * qL[0]) * rc * arcp(cs);
  lt -= lw6 * 0.5 * qL[4] * rt * rt;
  // upwind w1..w3
  {
    double *gU = left ? gL : gR;
    gU[0] += lw1;
    gU[QA] += lw2;
    gU[QB] += lw3;
    gU[4] -= (lw1 + lw2 * va + lw3 * vb) * rt;
    lt += (lw1 + lw2 * va + lw3 * vb) * qU[4] * rt * rt;
    lva -= lw2 * qU[4] * rt;
    lvb -= lw3 * qU[4] * rt;
  }
  // cs = sqrt(gamma p / r), p = C0 (r t)^gamma
  const double lp = lcs * cs * arcp(2. * p);
  double lr = -lcs * cs * arcp(2. * r) + lp * GAMMA * p * arcp(r);
  lt += lp * GAMMA * p * rt;
  gL[0] += 0.5 * lr;
  gR[0] += 0.5 * lr;
  double lvel[3];
  lvel[DIR] = lvn;
  lvel[TA] = lva;
  lvel[TB] = lvb;
  if (DIR == 1) {
    AWFL_UNROLL for (int k = 0; k < 3; k++) {
      gL[k + 1] += 0.5 * lvel[k];
      gR[k + 1] += 0.5 * lvel[k];
    }
    gL[4] += 0.5 * lt;
    gR[4] += 0.5 * lt;
  } else {
    AWFL_UNROLL for (int k = 0; k < 3; k++) {
      gL[k + 1] += 0.5 * lvel[k] * rl;
      gL[0] -= 0.5 * lvel[k] * qL[k + 1] * rl * rl;
      gR[k + 1] += 0.5 * lvel[k] * rrr;
      gR[0] -= 0.5 * lvel[k] * qR[k + 1] * rrr * rrr;
    }
    gL[4] += 0.5 * lt * rl;
    gL[0] -= 0.5 * lt * qL[4] * rl * rl;
    gR[4] += 0.5 * lt * rrr;
    gR[0] -= 0.5 * lt * qR[4] * rrr * rrr;
  }
  AWFL_UNROLL for (int v = 0; v < 5; v++) {
    lqL[v] = gL[v];
    lqR[v] = gR[v];
  }
}

}  // namespace adj
}  // namespace awfl
