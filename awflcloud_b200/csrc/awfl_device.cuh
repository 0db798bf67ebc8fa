// Device building blocks of the AWFL Euler-3D ADER/WENO step (FP64 parity path).
//
// Every function reproduces the arithmetic of the reference (mrnorman/awflCloud) in its
// evaluation order; the file:line cited is the reference code restated:
//   Spatial  = Spatial_euler3d_cons_expl_cart_fv_Agrid.h
//   Weno     = WenoLimiter.h
// The translation unit that includes this header is compiled with --fmad=false so that
// no multiply-add is contracted, like the reference's CPU build, and every pow is the
// correctly rounded pow_cr (awfl_pow.cuh), like glibc's.
#pragma once

#include <cstdint>
#include <type_traits>

#include "awfl_div.cuh"
#include "awfl_internal.h"
#include "awfl_pow.cuh"
#include "awfl_tv.h"

namespace awfl {

// One copy per translation unit that includes this header (awfl_fp64.cu, awfl_adjoint.cu);
// each is uploaded by that unit's upload function.
static __constant__ Tables<5> c_tab5;
static __constant__ Tables<9> c_tab9;

template <int ORD> __device__ __forceinline__ const Tables<ORD> &tab();
template <> __device__ __forceinline__ const Tables<5> &tab<5>() { return c_tab5; }
template <> __device__ __forceinline__ const Tables<9> &tab<9>() { return c_tab9; }

// Out-of-line forms of the two largest pieces of the per-cell FP64 code, the correctly
// rounded pow and the reconstruction of one variable (stencil and GLL values passed by
// value): one copy of their instructions in the kernel instead of one per call site. The
// fully inlined sweep outgrew the instruction cache (ncu: instruction-fetch stalls of 2.5
// cycles per issued instruction, the largest stall); out of line, the FP64 step took
// 7.38 ms instead of 9.73 ms at 256x256x128. The arithmetic is the same either way.
static __device__ __noinline__ double pow_gamma_call(double x) { return pow_cr(x, GAMMA); }
__device__ __forceinline__ double pow_gamma(double x) { return pow_gamma_call(x); }
template <class Sc> __device__ __forceinline__ Sc pow_gamma(const Sc &x) { return pow_cr(x, GAMMA); }

// The scalar type Sc is double for the FP64 path and Dual (awfl_dual.cuh) for the
// tangent-linear sweep; both evaluate the same expressions in the same order.
template <int N, class Sc> __device__ __forceinline__ Sc tv_eval(const Sc *a) {
  if constexpr (N == 3) return awfl_tv_n3<Sc>(a);
  else if constexpr (N == 5) return awfl_tv_n5<Sc>(a);
  else return awfl_tv_n9<Sc>(a);
}

// Weno:93-172 -- WENO polynomial coefficients of one ord-cell stencil.
template <int ORD, class Sc>
__device__ __forceinline__ void weno_coefs(const Sc (&u)[ORD], Sc (&aw)[ORD]) {
  constexpr int HS = (ORD - 1) / 2;
  const Tables<ORD> &T = tab<ORD>();
  const double eps = 1.0e-20;
  Sc a[HS + 2][ORD];
#pragma unroll
  for (int j = 0; j < HS + 2; j++)
#pragma unroll
    for (int i = 0; i < ORD; i++) a[j][i] = 0.;
#pragma unroll
  for (int i = 0; i < HS + 1; i++)
#pragma unroll
    for (int ii = 0; ii < HS + 1; ii++)
#pragma unroll
      for (int s = 0; s < HS + 1; s++) a[i][ii] += T.recon[(i * ORD + s) * ORD + ii] * u[i + s];
#pragma unroll
  for (int ii = 0; ii < ORD; ii++)
#pragma unroll
    for (int s = 0; s < ORD; s++) a[HS + 1][ii] += T.recon[((HS + 1) * ORD + s) * ORD + ii] * u[s];
#pragma unroll
  for (int i = 0; i < HS + 1; i++)
#pragma unroll
    for (int ii = 0; ii < HS + 1; ii++) a[HS + 1][ii] -= T.idl[i] * a[i][ii];
  const Rcp<double> ridl = rcp_known(T.idl[HS + 1], T.ridl);
#pragma unroll
  for (int ii = 0; ii < ORD; ii++) a[HS + 1][ii] = divd(a[HS + 1][ii], ridl);
  Sc tv[HS + 2];
#pragma unroll
  for (int i = 0; i < HS + 1; i++) tv[i] = tv_eval<HS + 1>(a[i]);
  tv[HS + 1] = tv_eval<ORD>(a[HS + 1]);
  Sc lo_avg = 0.;
#pragma unroll
  for (int i = 0; i < HS + 1; i++) lo_avg += tv[i];
  lo_avg = divk(lo_avg, HS + 1);
  tv[HS + 1] = lo_avg + (tv[HS + 1] - lo_avg) * T.sigma;
  Sc wts[HS + 2];
#pragma unroll
  for (int i = 0; i < HS + 2; i++) wts[i] = T.idl[i] / (tv[i] * tv[i] + eps);
  // convexify (Weno:20-25)
  {
    Sc sum = 0.;
#pragma unroll
    for (int i = 0; i < HS + 2; i++) sum += wts[i];
    const Rcp<Sc> rs = make_rcp<Sc>(sum + eps);
#pragma unroll
    for (int i = 0; i < HS + 2; i++) wts[i] = divr(wts[i], rs);
  }
  // map_weights (Weno:12-17)
#pragma unroll
  for (int i = 0; i < HS + 2; i++) {
    const double d = T.idl[i];
    wts[i] = wts[i] * (d + d * d - 3. * d * wts[i] + wts[i] * wts[i]) / (d * d + wts[i] * (1. - 2. * d));
  }
  {
    Sc sum = 0.;
#pragma unroll
    for (int i = 0; i < HS + 2; i++) sum += wts[i];
    const Rcp<Sc> rs = make_rcp<Sc>(sum + eps);
#pragma unroll
    for (int i = 0; i < HS + 2; i++) wts[i] = divr(wts[i], rs);
  }
#pragma unroll
  for (int i = 0; i < ORD; i++) aw[i] = 0.;
#pragma unroll
  for (int i = 0; i < HS + 2; i++)
#pragma unroll
    for (int ii = 0; ii < ORD; ii++) aw[ii] += wts[i] * a[i][ii];
}

// Spatial:1800-1833 -- ord stencil averages -> ngll GLL point values.
template <int ORD, class Sc>
__device__ __forceinline__ void reconstruct_gll(const Sc (&sten)[ORD], Sc (&out)[OrdTraits<ORD>::NGLL],
                                                bool doweno) {
  constexpr int NG = OrdTraits<ORD>::NGLL;
  const Tables<ORD> &T = tab<ORD>();
  if (doweno) {
    Sc wc[ORD];
    weno_coefs<ORD>(sten, wc);
#pragma unroll
    for (int ii = 0; ii < NG; ii++) {
      Sc tmp = 0;
#pragma unroll
      for (int s = 0; s < ORD; s++) tmp += T.c2g[s * NG + ii] * wc[s];
      out[ii] = tmp;
    }
  } else {
#pragma unroll
    for (int ii = 0; ii < NG; ii++) {
      Sc tmp = 0;
#pragma unroll
      for (int s = 0; s < ORD; s++) tmp += T.s2g[s * NG + ii] * sten[s];
      out[ii] = tmp;
    }
  }
}

template <int ORD> struct StenV { double v[ORD]; };
template <int ORD> struct GllV { double v[OrdTraits<ORD>::NGLL]; };
template <int ORD> static __device__ __noinline__ GllV<ORD> reconstruct_gll_call(StenV<ORD> s, bool doweno) {
  GllV<ORD> o;
  reconstruct_gll<ORD>(s.v, o.v, doweno);
  return o;
}
template <int ORD, class Sc>
__device__ __forceinline__ void reconstruct_gll_any(const Sc (&sten)[ORD], Sc (&out)[OrdTraits<ORD>::NGLL],
                                                    bool doweno) {
  if constexpr (std::is_same<Sc, double>::value) {
    StenV<ORD> s;
#pragma unroll
    for (int m = 0; m < ORD; m++) s.v[m] = sten[m];
    const GllV<ORD> o = reconstruct_gll_call<ORD>(s, doweno);
#pragma unroll
    for (int ii = 0; ii < OrdTraits<ORD>::NGLL; ii++) out[ii] = o.v[ii];
  } else {
    reconstruct_gll<ORD>(sten, out, doweno);
  }
}

// Reconstruction + ADER differential transform + edge time average of one cell
// (the K2 kernels: Spatial:665-811 x, 1028-1171 y, 1385-1552 z; diffTransformEulerConsX/Y/Z
// at Spatial:1837-2091; compute_timeAvg[_edges] at Spatial:2130-2177).
// sten(v, s) returns stencil value s of variable v. kb is the k index of the cell (z) or of
// the line (x, y). Outputs: the time-averaged left/right edge states and, for z, the
// time-averaged, GLL-weighted gravity source.
// A recorder that keeps nothing (the default): rec.level0(v, ii, x) sees every level-0
// value (after hydrostasis and the wall), for the adjoint's tape; rec.series(q) sees the
// whole ADER series q[v][kt][ii] before the edge time average, for the tracer transport.
struct NoRecord {
  template <class Sc> __device__ __forceinline__ void level0(int, int, const Sc &) const {}
  template <class Q> __device__ __forceinline__ void series(const Q &) const {}
};

template <int ORD, int DIR, class Sten, class Sc, class Rec = NoRecord>
__device__ __forceinline__ void cell_recon(const Sten &sten, int kb, const SweepArgs &A, Sc (&eL)[5], Sc (&eR)[5],
                                           Sc &src_avg, const Rec &rec = Rec()) {
  constexpr int HS = (ORD - 1) / 2;
  constexpr int NG = OrdTraits<ORD>::NGLL;
  constexpr int NA = NG;  // nAder = ngll (Temporal_ader.h:8)
  constexpr int NM = 1 + DIR;  // normal momentum
  const Tables<ORD> &T = tab<ORD>();

  Sc q[5][NA][NG];
#pragma unroll
  for (int v = 0; v < 5; v++) {
    Sc s[ORD];
#pragma unroll
    for (int m = 0; m < ORD; m++) s[m] = sten(v, m);
    const bool doweno = (v == idR || v == idT) ? A.weno_s : A.weno_w;
    reconstruct_gll_any<ORD>(s, q[v][0], doweno);
  }
  // add hydrostasis back on (x/y: cell averages, Spatial:680,697; z: GLL values, :1400,:1421)
#pragma unroll
  for (int ii = 0; ii < NG; ii++) {
    if (DIR == 2) {
      q[idR][0][ii] += A.dens_g[kb * NG + ii];
      q[idT][0][ii] += A.denstheta_g[kb * NG + ii];
    } else {
      q[idR][0][ii] += A.dens_c[HS + kb];
      q[idT][0][ii] += A.denstheta_c[HS + kb];
    }
  }
  if (DIR == 2 && A.bc == BC_WALL) {  // Spatial:1413-1416
    if (kb == A.nz - 1) q[idW][0][NG - 1] = 0;
    if (kb == 0) q[idW][0][0] = 0;
  }
#pragma unroll
  for (int v = 0; v < 5; v++)
#pragma unroll
    for (int ii = 0; ii < NG; ii++) rec.level0(v, ii, q[v][0][ii]);
  // level-0 flux products (Spatial:704-715 and y/z equivalents)
  Sc f[4][NA][NG];
  Sc g[NA][NG];
  Sc srcfill = 0;
  Rcp<Sc> rr[NG];  // the density of each GLL point: divisor of its velocities and products
  const Rcp<double> rdx = rcp_known(A.dxd, A.rdxd);
#pragma unroll
  for (int ii = 0; ii < NG; ii++) {
    const Sc r = q[idR][0][ii];
    rr[ii] = make_rcp<Sc>(r);
    const Sc u = divr(q[idU][0][ii], rr[ii]);
    const Sc v = divr(q[idV][0][ii], rr[ii]);
    const Sc w = divr(q[idW][0][ii], rr[ii]);
    const Sc t = divr(q[idT][0][ii], rr[ii]);
    const Sc vn = NM == 1 ? u : (NM == 2 ? v : w);
    f[0][0][ii] = r * vn * u;
    f[1][0][ii] = r * vn * v;
    f[2][0][ii] = r * vn * w;
    f[3][0][ii] = r * vn * t;
    g[0][ii] = pow_gamma(r * t);
    if (DIR == 2) srcfill = -(q[idR][0][ii] - A.dens_g[kb * NG + ii]) * GRAV;
  }
  // The z source SArray is filled by a scalar assignment inside the kk loop, so every entry
  // holds the kk = ngll-1 value (Spatial:1439).
  Sc sr[NA][NG];
#pragma unroll
  for (int kt = 0; kt < NA; kt++)
#pragma unroll
    for (int ii = 0; ii < NG; ii++) sr[kt][ii] = srcfill;

  // diffTransformEulerCons{X,Y,Z}
#pragma unroll
  for (int kt = 1; kt < NA; kt++)
#pragma unroll
    for (int ii = 0; ii < NG; ii++) {
      f[0][kt][ii] = 0; f[1][kt][ii] = 0; f[2][kt][ii] = 0; f[3][kt][ii] = 0;
      g[kt][ii] = 0;
    }
#pragma unroll
  for (int kt = 0; kt < NA - 1; kt++) {
#pragma unroll
    for (int ii = 0; ii < NG; ii++) {
      Sc dq[5] = {0., 0., 0., 0., 0.};
#pragma unroll
      for (int s = 0; s < NG; s++) {
        const double D = T.deriv[s * NG + ii];
        dq[idR] += D * (q[NM][kt][s]);
#pragma unroll
        for (int m = 1; m <= 3; m++) {
          if (m == NM) {
            if (DIR == 2 && kt == 0) {
              dq[m] += D * (f[m - 1][kt][s] + C0 * g[kt][s] - A.pres_g[kb * NG + s]);
            } else if (kt == 0) {
              dq[m] += D * (f[m - 1][kt][s] + C0 * g[kt][s]);
            } else {
              dq[m] += D * (f[m - 1][kt][s] + C0 * g[kt][s] / 2);
            }
          } else {
            dq[m] += D * (f[m - 1][kt][s]);
          }
        }
        dq[idT] += D * (f[3][kt][s]);
      }
#pragma unroll
      for (int m = 0; m < 5; m++) q[m][kt + 1][ii] = divk(divd(-dq[m], rdx), kt + 1);
      if (DIR == 2) {
        q[idW][kt + 1][ii] = divk(divd(-dq[idW], rdx), kt + 1) + divk(sr[kt][ii], kt + 1);
        if (A.bc == BC_WALL) {
          if (kb == A.nz - 1) q[idW][kt + 1][NG - 1] = 0;
          if (kb == 0) q[idW][kt + 1][0] = 0;
        }
        sr[kt + 1][ii] = -q[idR][kt + 1][ii] * GRAV;
      }
    }
#pragma unroll
    for (int ii = 0; ii < NG; ii++) {
      Sc tot[4] = {0., 0., 0., 0.};
#pragma unroll
      for (int ir = 0; ir <= kt + 1; ir++) {
#pragma unroll
        for (int x = 0; x < 4; x++)
          tot[x] += q[NM][ir][ii] * q[x + 1][kt + 1 - ir][ii] - q[idR][ir][ii] * f[x][kt + 1 - ir][ii];
      }
#pragma unroll
      for (int x = 0; x < 4; x++) f[x][kt + 1][ii] = divr(tot[x], rr[ii]);
      Sc tg = 0.;
#pragma unroll
      for (int ir = 0; ir <= kt; ir++)
        tg += (kt + 1. - ir) * (GAMMA * g[ir][ii] * q[idT][kt + 1 - ir][ii] - q[idT][ir][ii] * g[kt + 1 - ir][ii]);
      g[kt + 1][ii] = (GAMMA * g[0][ii] * q[idT][kt + 1][ii] + divk(tg, kt + 1)) / q[idT][0][ii];
    }
  }
  rec.series(q);
  // compute_timeAvg_edges (Spatial:2153-2177)
#pragma unroll
  for (int v = 0; v < 5; v++) {
    Sc l = q[v][0][0], r = q[v][0][NG - 1];
    double dtmult = A.dt;
#pragma unroll
    for (int kt = 1; kt < NA; kt++) {
      l += divk(q[v][kt][0] * dtmult, kt + 1);
      r += divk(q[v][kt][NG - 1] * dtmult, kt + 1);
      dtmult *= A.dt;
    }
    eL[v] = l;
    eR[v] = r;
  }
  src_avg = 0.;
  if (DIR == 2) {  // compute_timeAvg (Spatial:2130-2138) + GLL quadrature (Spatial:1489-1496)
    double dtmult = A.dt;
#pragma unroll
    for (int kt = 1; kt < NA; kt++) {
#pragma unroll
      for (int ii = 0; ii < NG; ii++) sr[0][ii] += divk(sr[kt][ii] * dtmult, kt + 1);
      dtmult *= A.dt;
    }
    Sc sa = 0.;
#pragma unroll
    for (int ii = 0; ii < NG; ii++) sa += sr[0][ii] * T.wts[ii];
    src_avg = sa;
  }
}

// Upwind characteristic Riemann flux at one interface (K4: Spatial:842-902 x, 1202-1260 y,
// 1583-1644 z). The y-direction averages are not divided by density (Spatial:1210-1214).
// kf is the interface's k index for the z hydrostatic pressure subtraction (x, y: the
// line's k, unused).
template <int DIR, int NG, class Sc>
__device__ __forceinline__ void riemann(const Sc (&qL)[5], const Sc (&qR)[5], int kf, const SweepArgs &A,
                                        Sc (&F)[5]) {
  constexpr int TA = DIR == 0 ? 1 : 0;  // first tangential velocity slot
  constexpr int TB = DIR == 2 ? 1 : 2;  // second tangential velocity slot
  constexpr int QN = 1 + DIR, QA = 1 + TA, QB = 1 + TB;
  const Sc r = 0.5 * (qL[0] + qR[0]);
  Sc vel[3], t;
  if (DIR == 1) {
    vel[0] = 0.5 * (qL[1] + qR[1]);
    vel[1] = 0.5 * (qL[2] + qR[2]);
    vel[2] = 0.5 * (qL[3] + qR[3]);
    t = 0.5 * (qL[4] + qR[4]);
  } else {
    const Rcp<Sc> rl = make_rcp<Sc>(qL[0]), rg = make_rcp<Sc>(qR[0]);
    vel[0] = 0.5 * (divr(qL[1], rl) + divr(qR[1], rg));
    vel[1] = 0.5 * (divr(qL[2], rl) + divr(qR[2], rg));
    vel[2] = 0.5 * (divr(qL[3], rl) + divr(qR[3], rg));
    t = 0.5 * (divr(qL[4], rl) + divr(qR[4], rg));
  }
  const Sc p = C0 * pow_gamma(r * t);
  const Sc cs2 = GAMMA * p / r;
  const Sc cs = sqrt(cs2);
  const Sc vn = vel[DIR], va = vel[TA], vb = vel[TB];
  const Rcp<Sc> rt = make_rcp<Sc>(t), rt2 = rcp_twice(rt), rc2 = make_rcp<Sc>(2. * cs);
  Sc w1, w2, w3;
  if (vn > 0) {
    w1 = qL[0] - divr(qL[4], rt);
    w2 = qL[QA] - divr(va * qL[4], rt);
    w3 = qL[QB] - divr(vb * qL[4], rt);
  } else {
    w1 = qR[0] - divr(qR[4], rt);
    w2 = qR[QA] - divr(va * qR[4], rt);
    w3 = qR[QB] - divr(vb * qR[4], rt);
  }
  const Sc w5 = divr(vn * qR[0], rc2) - divr(qR[QN], rc2) + divr(qR[4], rt2);
  const Sc w6 = divr(-vn * qL[0], rc2) + divr(qL[QN], rc2) + divr(qL[4], rt2);
  Sc q[5];
  q[0] = w1 + w5 + w6;
  q[QN] = vn * w1 + (vn - cs) * w5 + (vn + cs) * w6;
  q[QA] = w2 + va * w5 + va * w6;
  q[QB] = w3 + vb * w5 + vb * w6;
  q[4] = t * w5 + t * w6;
  const Rcp<Sc> r0 = make_rcp<Sc>(q[0]);
  F[0] = q[QN];
  F[QN] = divr(q[QN] * q[QN], r0) + C0 * pow_gamma(q[4]);
  F[QA] = divr(q[QN] * q[QA], r0);
  F[QB] = divr(q[QN] * q[QB], r0);
  F[4] = divr(q[QN] * q[4], r0);
  if (DIR == 2) {  // Spatial:1628-1629
    if (kf < A.nz) F[idW] -= A.pres_g[kf * NG + 0];
    if (kf == A.nz) F[idW] -= A.pres_g[(A.nz - 1) * NG + NG - 1];
  }
}

}  // namespace awfl
