// FP32 precision form of the AWFL Euler-3D ADER/WENO step: device functions and the
// sweep policy P32, sm_100a.
//
// Same scheme as the reference (Spatial_euler3d_cons_expl_cart_fv_Agrid.h, WenoLimiter.h,
// Temporal_ader.h), same line-sweep kernel skeleton as the FP64 path (awfl_sweep.cuh), but
// FP32 arithmetic (FMA contraction and fast division/sqrt allowed) with the scheme's
// cancellation-prone pieces rewritten in perturbation form, so that single precision
// keeps its ~1e-7 relative accuracy on the perturbation fields:
//
//  * State: FP32 perturbations from the hydrostatic background (rho', rho*u, rho*v, rho*w,
//    (rho*theta)'), like the reference's own state, plus a second FP32 plane holding the
//    Kahan compensation of every stage update (state += dt*tend, Temporal_ader.h:63-65).
//  * Background: computed in FP64 on the host (the reference's profiles) and used as FP32
//    per-row (x/y: cell averages) or per-GLL-point/per-face (z) constants.
//  * Pressure: C0*(rho*theta)^gamma = P_h * (1 + B(x)), x = (rho*theta)'/(rho*theta)_h,
//    B(x) = (1+x)^gamma - 1 by its binomial series (|x| < 0.05; expm1(gamma*log1p(x))
//    otherwise), P_h = C0*(rho*theta)_h^gamma in FP64. Only P_h*B enters derivatives and
//    fluxes: a row-constant P_h cancels exactly in the x/y divergence, and in z it is the
//    reference's own hydrostatic subtraction (Spatial:2042, :1628-1629).
//  * (rho*theta)^gamma time derivatives are carried scaled by (rho*theta)_h^gamma.
//  * Edge states are carried as perturbations; the Riemann mass flux is evaluated as
//    vn*q1 + cs*(w6 - w5) with w6 - w5 expressed through L-R differences of perturbations,
//    instead of vn*w1 + (vn-cs)*w5 + (vn+cs)*w6 whose O(rho*cs) terms cancel.
//  * The CFL time step reads the FP32 state but computes in FP64.
// Every expression equals the reference's in exact arithmetic, including its quirks (y
// averages not divided by density, the filled z gravity source, the z wall).
#pragma once

#include <cuda_runtime.h>

#include <cmath>

#include "awfl_internal.h"
#include "awfl_fp32_args.h"
#include "awfl_pow.cuh"
#include "awfl_sweep.cuh"
#include "awfl_tv.h"

namespace awfl {

// Fast reciprocal (MUFU-based, ~1 ulp): the FP32 form's divisions.
__device__ __forceinline__ float frcp(float x) { return __fdividef(1.f, x); }

constexpr float GAMMAF = (float)GAMMA;
constexpr float GRAVF = (float)GRAV;

// Binomial coefficients C(gamma, n), n = 1..6, of (1+x)^gamma.
constexpr double kB1 = GAMMA;
constexpr double kB2 = kB1 * (GAMMA - 1.0) / 2.0;
constexpr double kB3 = kB2 * (GAMMA - 2.0) / 3.0;
constexpr double kB4 = kB3 * (GAMMA - 3.0) / 4.0;
constexpr double kB5 = kB4 * (GAMMA - 4.0) / 5.0;
constexpr double kB6 = kB5 * (GAMMA - 5.0) / 6.0;

// (1+x)^gamma - 1
__device__ __forceinline__ float binom_gamma_m1(float x) {
  if (fabsf(x) < 0.05f) {
    float p = (float)kB6;
    p = fmaf(p, x, (float)kB5);
    p = fmaf(p, x, (float)kB4);
    p = fmaf(p, x, (float)kB3);
    p = fmaf(p, x, (float)kB2);
    p = fmaf(p, x, (float)kB1);
    return p * x;
  }
  return expm1f(GAMMAF * log1pf(x));
}

template <int ORD> struct Tables32 {
  static constexpr int HS = (ORD - 1) / 2;
  static constexpr int NG = OrdTraits<ORD>::NGLL;
  float recon[ORD * ORD * ORD];
  // the high-order candidate's coefficients straight from the stencil: (its full-stencil
  // map minus the idl-weighted low-order candidates' maps) / idl[hs+1], formed in FP64
  float hi[ORD * ORD];
  float c2g[ORD * NG];
  float s2g[ORD * NG];
  float deriv[NG * NG];
  float idl[HS + 2];
  float sigma;
  float wts[NG];
};
// One copy per translation unit that includes this header (awfl_fp32.cu, awfl_ens32.cu),
// each uploaded by upload_tables32_here.
static __constant__ Tables32<5> c32_tab5;
static __constant__ Tables32<9> c32_tab9;
template <int ORD> __device__ __forceinline__ const Tables32<ORD> &tab32();
template <> __device__ __forceinline__ const Tables32<5> &tab32<5>() { return c32_tab5; }
template <> __device__ __forceinline__ const Tables32<9> &tab32<9>() { return c32_tab9; }

template <int N> __device__ __forceinline__ float tv_evalf(const float *a);
template <> __device__ __forceinline__ float tv_evalf<3>(const float *a) { return awfl_tv_n3<float>(a); }
template <> __device__ __forceinline__ float tv_evalf<5>(const float *a) { return awfl_tv_n5<float>(a); }
template <> __device__ __forceinline__ float tv_evalf<9>(const float *a) { return awfl_tv_n9<float>(a); }

// Two independent FP32 lanes evaluated with the paired sm_100 instructions (FFMA2, FMUL2,
// FADD2: one instruction, two results, each rounded like the scalar operation), so that
// two variables' reconstructions issue half the instructions. Divisions stay per lane.
struct F2 {
  float2 v;
  __device__ __forceinline__ F2() {}
  __device__ __forceinline__ F2(float2 x) : v(x) {}
  __device__ __forceinline__ F2(float a, float b) : v(make_float2(a, b)) {}
  __device__ __forceinline__ explicit F2(double c) : v(make_float2((float)c, (float)c)) {}
  __device__ __forceinline__ explicit F2(float c) : v(make_float2(c, c)) {}
};
__device__ __forceinline__ F2 operator+(F2 a, F2 b) { return F2(__fadd2_rn(a.v, b.v)); }
__device__ __forceinline__ F2 operator-(F2 a, F2 b) { return F2(__fadd2_rn(a.v, make_float2(-b.v.x, -b.v.y))); }
__device__ __forceinline__ F2 operator*(F2 a, F2 b) { return F2(__fmul2_rn(a.v, b.v)); }
__device__ __forceinline__ F2 operator*(float c, F2 b) { return F2(__fmul2_rn(make_float2(c, c), b.v)); }
__device__ __forceinline__ F2 operator*(F2 a, float c) { return F2(__fmul2_rn(a.v, make_float2(c, c))); }
__device__ __forceinline__ F2 operator+(F2 a, float c) { return F2(__fadd2_rn(a.v, make_float2(c, c))); }
__device__ __forceinline__ F2 operator+(float c, F2 a) { return F2(__fadd2_rn(make_float2(c, c), a.v)); }
__device__ __forceinline__ F2 &operator+=(F2 &a, F2 b) { return a = a + b; }

// fma / reciprocal / quotient on either scalar type
__device__ __forceinline__ float fmaT(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ F2 fmaT(float a, F2 b, F2 c) { return F2(__ffma2_rn(make_float2(a, a), b.v, c.v)); }
__device__ __forceinline__ F2 fmaT(F2 a, F2 b, F2 c) { return F2(__ffma2_rn(a.v, b.v, c.v)); }
__device__ __forceinline__ F2 fmaT(F2 a, float b, F2 c) { return F2(__ffma2_rn(a.v, make_float2(b, b), c.v)); }
__device__ __forceinline__ float rcpT(float x) { return frcp(x); }
__device__ __forceinline__ F2 rcpT(F2 x) { return F2(frcp(x.v.x), frcp(x.v.y)); }
__device__ __forceinline__ float divT(float a, float b) { return __fdividef(a, b); }
__device__ __forceinline__ F2 divT(float a, F2 b) { return F2(__fdividef(a, b.v.x), __fdividef(a, b.v.y)); }
__device__ __forceinline__ F2 divT(F2 a, F2 b) { return F2(__fdividef(a.v.x, b.v.x), __fdividef(a.v.y, b.v.y)); }

template <int N> __device__ __forceinline__ F2 tv_evalf2(const F2 *a) {
  if constexpr (N == 3) return awfl_tv_n3<F2>(a);
  else if constexpr (N == 5) return awfl_tv_n5<F2>(a);
  else return awfl_tv_n9<F2>(a);
}
template <int N> __device__ __forceinline__ float tv_evalT(const float *a) { return tv_evalf<N>(a); }
template <int N> __device__ __forceinline__ F2 tv_evalT(const F2 *a) { return tv_evalf2<N>(a); }

// WenoLimiter.h:93-172 in FP32.
template <int ORD, class T>
__device__ __forceinline__ void weno_coefs32(const T (&u)[ORD], T (&aw)[ORD]) {
  constexpr int HS = (ORD - 1) / 2;
  const Tables32<ORD> &Tb = tab32<ORD>();
  const float eps = 1.0e-20f;
  // Structural zeros (symmetric stencils; checked when the tables are uploaded) are left
  // out: the centred low-order candidate's odd coefficients and the high-order map's odd
  // coefficients take nothing from the stencil's centre value.
  T a[HS + 2][ORD];
#pragma unroll
  for (int i = 0; i < HS + 1; i++)
#pragma unroll
    for (int ii = 0; ii < HS + 1; ii++) {
      T acc = T(0.f);
#pragma unroll
      for (int s = 0; s < HS + 1; s++) {
        if (HS % 2 == 0 && i == HS / 2 && s == HS / 2 && ii % 2 == 1) continue;
        acc = fmaT(Tb.recon[(i * ORD + s) * ORD + ii], u[i + s], acc);
      }
      a[i][ii] = acc;
    }
#pragma unroll
  for (int ii = 0; ii < ORD; ii++) {
    T acc = T(0.f);
#pragma unroll
    for (int s = 0; s < ORD; s++) {
      if (s == HS && ii % 2 == 1) continue;
      acc = fmaT(Tb.hi[s * ORD + ii], u[s], acc);
    }
    a[HS + 1][ii] = acc;
  }
  T tv[HS + 2];
#pragma unroll
  for (int i = 0; i < HS + 1; i++) tv[i] = tv_evalT<HS + 1>(a[i]);
  tv[HS + 1] = tv_evalT<ORD>(a[HS + 1]);
  T lo_avg = T(0.f);
#pragma unroll
  for (int i = 0; i < HS + 1; i++) lo_avg += tv[i];
  lo_avg = lo_avg * (1.0f / (HS + 1));
  tv[HS + 1] = fmaT(tv[HS + 1] - lo_avg, Tb.sigma, lo_avg);
  T wts[HS + 2];
  T sum = T(0.f);
#pragma unroll
  for (int i = 0; i < HS + 2; i++) {
    wts[i] = divT(Tb.idl[i], fmaT(tv[i], tv[i], T(eps)));
    sum += wts[i];
  }
  T inv = rcpT(sum + eps);
  sum = T(0.f);
#pragma unroll
  for (int i = 0; i < HS + 2; i++) {
    const T w = wts[i] * inv;
    const float d = Tb.idl[i];
    const T num = w * ((d + d * d) + (w * w - (3.f * d) * w));
    const T den = (d * d) + w * (1.f - 2.f * d);
    wts[i] = divT(num, den);
    sum += wts[i];
  }
  inv = rcpT(sum + eps);
#pragma unroll
  for (int ii = 0; ii < ORD; ii++) aw[ii] = T(0.f);
#pragma unroll
  for (int i = 0; i < HS + 2; i++) {
    const T w = wts[i] * inv;
#pragma unroll
    for (int ii = 0; ii < ORD; ii++) {
      if (i < HS + 1 && ii > HS) continue;  // zero coefficients of the low-order candidates
      aw[ii] = fmaT(w, a[i][ii], aw[ii]);
    }
  }
}
template <int ORD, class T>
__device__ __forceinline__ void reconstruct_gll32(const T (&sten)[ORD], T (&out)[OrdTraits<ORD>::NGLL], bool doweno) {
  constexpr int NG = OrdTraits<ORD>::NGLL;
  const Tables32<ORD> &Tb = tab32<ORD>();
  if (doweno) {
    T wc[ORD];
    weno_coefs32<ORD>(sten, wc);
    // polynomial coefficients -> values at the GLL points, which sit symmetrically about
    // the cell centre (x = 0): the centre takes the constant coefficient alone, the mirror
    // points x and -x the even part plus and minus the odd part
    static_assert(NG % 2 == 1, "an odd number of GLL points, one at the centre");
    out[NG / 2] = wc[0];
#pragma unroll
    for (int ii = 0; ii < NG / 2; ii++) {
      const int jr = NG - 1 - ii;
      T ev = T(0.f), od = T(0.f);
#pragma unroll
      for (int s = 0; s < ORD; s += 2) ev = fmaT(Tb.c2g[s * NG + jr], wc[s], ev);
#pragma unroll
      for (int s = 1; s < ORD; s += 2) od = fmaT(Tb.c2g[s * NG + jr], wc[s], od);
      out[jr] = ev + od;
      out[ii] = ev - od;
    }
  } else {
#pragma unroll
    for (int ii = 0; ii < NG; ii++) {
      T tmp = T(0.f);
#pragma unroll
      for (int s = 0; s < ORD; s++) tmp = fmaT(Tb.s2g[s * NG + ii], sten[s], tmp);
      out[ii] = tmp;
    }
  }
}

// A recorder that keeps nothing (the default of cell_recon32): rec.series32(q, rtot) sees
// the whole ADER series q[v][kt][ii] (level 0 as perturbations) and the total density of
// the GLL points before the edge time average, for the tracer transport.
struct NoRecord32 {
  template <class Q, class Rt> __device__ __forceinline__ void series32(const Q &, const Rt &) const {}
};

template <int ORD, int DIR, class Sten, class Rec = NoRecord32>
__device__ __forceinline__ void cell_recon32(const Sten &sten, int kb, const SweepArgs32 &A, float (&eL)[5],
                                             float (&eR)[5], float &src_avg, const Rec &rec = Rec()) {
  constexpr int HS = (ORD - 1) / 2;
  constexpr int NG = OrdTraits<ORD>::NGLL;
  constexpr int NA = NG;
  constexpr int NM = 1 + DIR;
  const Tables32<ORD> &T = tab32<ORD>();

  float q[5][NA][NG];  // level 0: rho' (perturbation), rho*u/v/w, (rho*theta)' (perturbation)
  // (rho', (rho theta)') and (rho u, rho v) in pairs on the paired FP32 instructions
#pragma unroll
  for (int pr = 0; pr < 2; pr++) {
    const int va = pr == 0 ? idR : idU, vb = pr == 0 ? idT : idV;
    F2 s2[ORD], o2[NG];
#pragma unroll
    for (int m = 0; m < ORD; m++) s2[m] = F2(sten(va, m), sten(vb, m));
    reconstruct_gll32<ORD>(s2, o2, pr == 0 ? A.weno_s : A.weno_w);
#pragma unroll
    for (int ii = 0; ii < NG; ii++) {
      q[va][0][ii] = o2[ii].v.x;
      q[vb][0][ii] = o2[ii].v.y;
    }
  }
  {
    float s[ORD];
#pragma unroll
    for (int m = 0; m < ORD; m++) s[m] = sten(idW, m);
    reconstruct_gll32<ORD>(s, q[idW][0], A.weno_w);
  }
  if (DIR == 2 && A.bc == BC_WALL) {  // Spatial:1413-1416
    if (kb == A.nz - 1) q[idW][0][NG - 1] = 0.f;
    if (kb == 0) q[idW][0][0] = 0.f;
  }
  float rtot[NG], rttot[NG], Pbg[NG];
  float f[4][NA][NG];
  float g[NA][NG];  // (rho theta)^gamma series / (rho theta)_h^gamma
#pragma unroll
  for (int ii = 0; ii < NG; ii++) {
    float rb, rtb, irtb;
    if (DIR == 2) {
      rb = A.bg.rho_g[kb * NG + ii]; rtb = A.bg.rt_g[kb * NG + ii];
      irtb = A.bg.irt_g[kb * NG + ii]; Pbg[ii] = A.bg.p_g[kb * NG + ii];
    } else {
      rb = A.bg.rho_c[HS + kb]; rtb = A.bg.rt_c[HS + kb];
      irtb = A.bg.irt_c[HS + kb]; Pbg[ii] = A.bg.p_c[HS + kb];
    }
    rtot[ii] = rb + q[idR][0][ii];
    rttot[ii] = rtb + q[idT][0][ii];
    const float ir = frcp(rtot[ii]);
    const float vel[3] = {q[idU][0][ii] * ir, q[idV][0][ii] * ir, q[idW][0][ii] * ir};
    const float th = rttot[ii] * ir;
    const float rvn = q[NM][0][ii];  // r * vn
    f[0][0][ii] = rvn * vel[0];
    f[1][0][ii] = rvn * vel[1];
    f[2][0][ii] = rvn * vel[2];
    f[3][0][ii] = rvn * th;
    g[0][ii] = binom_gamma_m1(q[idT][0][ii] * irtb);  // B(x); the scaled series starts at 1 + B
  }
  // z gravity source: every entry holds the kk = ngll-1 value (Spatial:1439), -(rho')*g
  float sr[NA][NG];
  const float srcfill = DIR == 2 ? -q[idR][0][NG - 1] * GRAVF : 0.f;
#pragma unroll
  for (int kt = 0; kt < NA; kt++)
#pragma unroll
    for (int ii = 0; ii < NG; ii++) sr[kt][ii] = srcfill;

  // diffTransformEulerCons{X,Y,Z} (Spatial:1837-2091)
#pragma unroll
  for (int kt = 0; kt < NA - 1; kt++) {
#pragma unroll
    for (int ii = 0; ii < NG; ii++) {
      float dq[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll
      for (int s = 0; s < NG; s++) {
        if (ii == NG / 2 && s == NG / 2) continue;  // d/dx at the centre: no centre weight
        const float D = T.deriv[s * NG + ii];
        dq[idR] = fmaf(D, q[NM][kt][s], dq[idR]);
#pragma unroll
        for (int m = 1; m <= 3; m++) {
          float fm = f[m - 1][kt][s];
          if (m == NM) fm += kt == 0 ? Pbg[s] * g[0][s] : 0.5f * Pbg[s] * g[kt][s];
          dq[m] = fmaf(D, fm, dq[m]);
        }
        dq[idT] = fmaf(D, f[3][kt][s], dq[idT]);
      }
      const float sc = -A.inv_dxd * (1.0f / (kt + 1));
#pragma unroll
      for (int m = 0; m < 5; m++) q[m][kt + 1][ii] = dq[m] * sc;
      if (DIR == 2) {
        q[idW][kt + 1][ii] = fmaf(sr[kt][ii], 1.0f / (kt + 1), q[idW][kt + 1][ii]);
        if (A.bc == BC_WALL) {
          if (kb == A.nz - 1 && ii == NG - 1) q[idW][kt + 1][ii] = 0.f;
          if (kb == 0 && ii == 0) q[idW][kt + 1][ii] = 0.f;
        }
        sr[kt + 1][ii] = -q[idR][kt + 1][ii] * GRAVF;
      }
    }
    if (kt + 1 < NA - 1) {  // products needed by the next level only
#pragma unroll
      for (int ii = 0; ii < NG; ii++) {
        const float ir0 = frcp(rtot[ii]);
        auto Q = [&](int m, int l) -> float {
          if (l == 0) return m == idR ? rtot[ii] : (m == idT ? rttot[ii] : q[m][0][ii]);
          return q[m][l][ii];
        };
        // Cauchy products of the series; the not-yet-known level kt+1 of f and g enters
        // with a zero coefficient and is left out (an IEEE multiply by zero is not
        // removed by the compiler)
#pragma unroll
        for (int x = 0; x < 4; x++) {
          float tot = 0.f;
#pragma unroll
          for (int ir = 0; ir <= kt + 1; ir++) {
            tot = fmaf(Q(NM, ir), Q(x + 1, kt + 1 - ir), tot);
            if (ir != 0) tot = fmaf(-Q(idR, ir), f[x][kt + 1 - ir][ii], tot);
          }
          f[x][kt + 1][ii] = tot * ir0;
        }
        // scaled (rho theta)^gamma: g~(0) = 1 + B
        auto Gs = [&](int l) -> float { return l == 0 ? 1.f + g[0][ii] : g[l][ii]; };
        float tg = 0.f;
#pragma unroll
        for (int ir = 0; ir <= kt; ir++) {
          float term = GAMMAF * Gs(ir) * Q(idT, kt + 1 - ir);
          if (ir != 0) term = fmaf(-Q(idT, ir), Gs(kt + 1 - ir), term);
          tg = fmaf(kt + 1.f - ir, term, tg);
        }
        g[kt + 1][ii] = fmaf(tg, 1.0f / (kt + 1), GAMMAF * Gs(0) * q[idT][kt + 1][ii]) * frcp(rttot[ii]);
      }
    }
  }
  rec.series32(q, rtot);
  // compute_timeAvg_edges on perturbations (Spatial:2153-2177)
#pragma unroll
  for (int v = 0; v < 5; v++) {
    float l = q[v][0][0], r = q[v][0][NG - 1];
    float dtmult = A.dt;
#pragma unroll
    for (int kt = 1; kt < NA; kt++) {
      const float c = dtmult * (1.0f / (kt + 1));
      l = fmaf(q[v][kt][0], c, l);
      r = fmaf(q[v][kt][NG - 1], c, r);
      dtmult *= A.dt;
    }
    eL[v] = l;
    eR[v] = r;
  }
  src_avg = 0.f;
  if (DIR == 2) {
    float dtmult = A.dt;
#pragma unroll
    for (int kt = 1; kt < NA; kt++) {
#pragma unroll
      for (int ii = 0; ii < NG; ii++) sr[0][ii] = fmaf(sr[kt][ii], dtmult * (1.0f / (kt + 1)), sr[0][ii]);
      dtmult *= A.dt;
    }
    float sa = 0.f;
#pragma unroll
    for (int ii = 0; ii < NG; ii++) sa = fmaf(sr[0][ii], T.wts[ii], sa);
    src_avg = sa;
  }
}

// Upwind Riemann flux in FP32 perturbation form (Spatial:842-902, 1202-1260, 1583-1644).
template <int DIR, int NG>
__device__ __forceinline__ void riemann32(const float (&qL)[5], const float (&qR)[5], int kf, const SweepArgs32 &A,
                                          float (&F)[5]) {
  constexpr int TA = DIR == 0 ? 1 : 0;
  constexpr int TB = DIR == 2 ? 1 : 2;
  constexpr int QN = 1 + DIR, QA = 1 + TA, QB = 1 + TB;
  constexpr int HS = NG == 3 ? 2 : 4;
  // side backgrounds (rho, rho*theta) and the face's pressure background
  float bLr, bLt, bRr, bRt, rtf, irtf, pf;
  if (DIR == 2) {
    const int fL = (kf == 0 && A.bc == BC_PERIODIC) ? A.nz : kf;
    const int fR = (kf == A.nz && A.bc == BC_PERIODIC) ? 0 : kf;
    bLr = A.bg.rho_f[fL]; bLt = A.bg.rt_f[fL];
    bRr = A.bg.rho_f[fR]; bRt = A.bg.rt_f[fR];
    rtf = A.bg.rt_f[kf]; irtf = A.bg.irt_f[kf]; pf = A.bg.p_f[kf];
  } else {
    (void)HS;
    const int k = kf;  // x/y sweeps: the line's k
    bLr = bRr = A.bg.rho_c[HS + k];
    bLt = bRt = A.bg.rt_c[HS + k];
    rtf = bLt; irtf = A.bg.irt_c[HS + k]; pf = A.bg.p_c[HS + k];
  }
  const float rL = bLr + qL[0], rR = bRr + qR[0];
  const float tL = bLt + qL[4], tR = bRt + qR[4];  // total rho*theta
  const float irL = frcp(rL), irR = frcp(rR);
  const float r = 0.5f * (rL + rR);
  float vel[3], t, uL = 0.f, uR = 0.f;
  if (DIR == 1) {  // y: averages not divided by density (Spatial:1210-1214)
    vel[0] = 0.5f * (qL[1] + qR[1]);
    vel[1] = 0.5f * (qL[2] + qR[2]);
    vel[2] = 0.5f * (qL[3] + qR[3]);
    t = 0.5f * (tL + tR);
  } else {
    uL = qL[QN] * irL;
    uR = qR[QN] * irR;
#pragma unroll
    for (int m = 0; m < 3; m++) vel[m] = m == DIR ? 0.5f * (uL + uR) : 0.5f * fmaf(qL[1 + m], irL, qR[1 + m] * irR);
    t = 0.5f * fmaf(tL, irL, tR * irR);
  }
  // cs^2 = gamma*C0*(r t)^gamma / r with (r t)^gamma = (rho theta)_f^gamma (1 + B)
  const float rt = r * t;
  const float cs2 = GAMMAF * pf * (1.f + binom_gamma_m1((rt - rtf) * irtf)) * frcp(r);
  const float cs = sqrtf(cs2);
  const float ics2 = 0.5f * frcp(cs), it2 = 0.5f * frcp(t);
  const float vn = vel[DIR], va = vel[TA], vb = vel[TB];
  float w1, w2, w3;
  if (vn > 0) {
    const float a = tL * (2.f * it2);
    w1 = rL - a;
    w2 = qL[QA] - va * a;
    w3 = qL[QB] - vb * a;
  } else {
    const float a = tR * (2.f * it2);
    w1 = rR - a;
    w2 = qR[QA] - va * a;
    w3 = qR[QB] - vb * a;
  }
  const float dq1 = (bRr - bLr) + (qR[0] - qL[0]);  // q1R - q1L
  const float dqn = qR[QN] - qL[QN];
  const float dq5 = (bLt - bRt) + (qL[4] - qR[4]);  // q5L - q5R
  const float S = fmaf(vn, dq1, -dqn) * ics2 + (tL + tR) * it2;  // w5 + w6
  float d65;                                                        // w6 - w5
  if (DIR == 1) d65 = fmaf(-vn, rL + rR, qL[QN] + qR[QN]) * ics2 + dq5 * it2;
  else d65 = (-dq1) * (uL - uR) * 0.5f * ics2 + dq5 * it2;
  const float q1 = w1 + S;
  const float qn = fmaf(vn, q1, cs * d65);
  const float qa = fmaf(va, S, w2);
  const float qb = fmaf(vb, S, w3);
  const float q5 = t * S;
  // (rho theta) perturbation of the upwind state relative to the face background
  const float q5p = t * fmaf(vn, dq1, -dqn) * ics2 + (0.5f * ((bLt + bRt) - 2.f * rtf) + 0.5f * (qL[4] + qR[4]));
  const float iq1 = frcp(q1);
  F[0] = qn;
  F[QN] = fmaf(qn * qn, iq1, pf * binom_gamma_m1(q5p * irtf));
  F[QA] = qn * qa * iq1;
  F[QB] = qn * qb * iq1;
  F[4] = qn * q5 * iq1;
}

struct P32 {
  using Real = float;
  static constexpr int kWdiv = 1;
  static constexpr bool kAsyncRing = true;
  // interior chunks are staged by tiled TMA: the single-grid sweep reads the tensor map
  // from its kernel parameter, the ensemble's persistent sweep from the work list in
  // global memory (its shared-memory copy of the arguments is no place for one)
  static constexpr bool kTmaRing = true;
  static constexpr bool kSlab = true;  // awfl_split_slab
  static bool prepare_tma(SweepArgs32 &A, int ord, int dir, int C, int W) {
    return prepare_sweep_map32(A, ord, dir, C, W);
  }
  static __device__ __forceinline__ const void *tma_map(const SweepArgs32 &A) { return &A.tmap; }
  static __device__ __forceinline__ const void *tma_map_global(const SweepArgs32 &shared_copy,
                                                               const SweepArgs32 *in_global) {
    return shared_copy.tma ? (const void *)&in_global->tmap : nullptr;
  }
  static __device__ __forceinline__ void flag_timeout(const SweepArgs32 &A) {
    if (A.err) atomicOr(A.err, 1u);
  }
  static constexpr int min_blocks(int) { return 1; }  // forcing more CTAs per SM measured slower
  using Args = SweepArgs32;
  // the Kahan compensations of the cell's five variables, loaded before the reconstruction
  struct Aux {
    float c[5];
  };
  static __device__ __forceinline__ void load_aux(const Args &A, long g0, long sv, Aux &aux) {
#pragma unroll
    for (int v = 0; v < 5; v++) aux.c[v] = A.comp[g0 + v * sv];
  }

  template <int ORD, int DIR, class S>
  static __device__ __forceinline__ void recon(const S &sten, int kb, const Args &A, float (&eL)[5], float (&eR)[5],
                                               float &src, long) {
    cell_recon32<ORD, DIR>(sten, kb, A, eL, eR, src);
  }
  template <int DIR, int NG>
  static __device__ __forceinline__ void flux(const float (&qL)[5], const float (&qR)[5], int kf, const Args &A,
                                              float (&F)[5]) {
    riemann32<DIR, NG>(qL, qR, kf, A, F);
  }
  template <int DIR>
  static __device__ __forceinline__ float tendency(int v, float Fl, float Fr, float sa, const Args &A) {
    const float d = (Fl - Fr) * A.inv_dxd;
    if (DIR == 0) return (A.sim2d && v == idV) ? 0.f : d;
    if (DIR == 1) return d;
    return (A.sim2d && v == idV) ? 0.f : (v == idW ? sa + d : d);
  }
  // Kahan-compensated stage update: s += dt*tnd with the running compensation c.
  static __device__ __forceinline__ void apply(const Args &A, long g, float orig, float tnd, const Aux &aux, int v) {
    const float y = A.dt * tnd - aux.c[v];
    const float t = orig + y;
    A.comp[g] = __fsub_rn(__fsub_rn(t, orig), y);
    A.state[g] = t;
  }
  static __device__ __forceinline__ float load(const Args &A, long g) { return A.state[g]; }
  static __device__ __forceinline__ void store(const Args &A, long g, float x) { A.state[g] = x; }
  static __device__ __forceinline__ void store_tend(const Args &A, long g, float x) { A.tend[g] = x; }
};

// Single-grid sweep shapes of the FP32 form, ord 5 (chunk C x lines W; measured at
// 256x256x128 with TMA staging against x {16,8} {32,4} {4,32} {8,32} {16,16}, y {8,16}
// {16,8} {16,16} {8,32} {4,16}, z {8,16} {16,8} {8,32} {4,64} {4,16}): x 8 x 16, y 4 x 32,
// z 4 x 32 (y/z: a warp = 8 lines x 4 positions, 32-byte row segments).
template <> struct PolicyShape<P32, 5, 0> { static constexpr int C = 8, W = 16; };
template <> struct PolicyShape<P32, 5, 1> { static constexpr int C = 4, W = 32; };

// Uploads the FP32 tables into this translation unit's constant memory.
static inline cudaError_t upload_tables32_here(int ord, const double *recon, const double *c2g, const double *s2g,
                                               const double *deriv, const double *idl, double sigma,
                                               const double *wts) {
  auto fill = [&](auto &t, int o, int g) {
    const int hs = (o - 1) / 2;
    for (int i = 0; i < o * o * o; i++) t.recon[i] = (float)recon[i];
    for (int sidx = 0; sidx < o; sidx++)
      for (int ii = 0; ii < o; ii++) {
        double m = recon[((hs + 1) * o + sidx) * o + ii];
        if (ii <= hs)
          for (int i = 0; i <= hs; i++)
            if (sidx - i >= 0 && sidx - i <= hs) m -= idl[i] * recon[(i * o + (sidx - i)) * o + ii];
        t.hi[sidx * o + ii] = (float)(m / idl[hs + 1]);
      }
    for (int i = 0; i < o * g; i++) { t.c2g[i] = (float)c2g[i]; t.s2g[i] = (float)s2g[i]; }
    for (int i = 0; i < g * g; i++) t.deriv[i] = (float)deriv[i];
    for (int i = 0; i < hs + 2; i++) t.idl[i] = (float)idl[i];
    t.sigma = (float)sigma;
    for (int i = 0; i < g; i++) t.wts[i] = (float)wts[i];
  };
  // the structural zeros and symmetries the FP32 reconstruction leaves out of its sums
  auto structure_ok = [&](const auto &t, int o, int g) {
    const int hs = (o - 1) / 2;
    double dmax = 0, rmax = 0;
    for (int x = 0; x < g * g; x++) dmax = fmax(dmax, fabs((double)t.deriv[x]));
    for (int x = 0; x < o * o * o; x++) rmax = fmax(rmax, fabs((double)t.recon[x]));
    bool ok = g % 2 == 1 && hs % 2 == 0 && t.c2g[0 * g + g / 2] == 1.f &&
              fabs((double)t.deriv[(g / 2) * g + g / 2]) <= 1e-6 * dmax;
    for (int sidx = 1; sidx < o; sidx++) ok = ok && t.c2g[sidx * g + g / 2] == 0.f;
    for (int sidx = 0; sidx < o; sidx++)
      for (int ii = 0; ii < g; ii++)
        ok = ok && t.c2g[sidx * g + ii] == ((sidx % 2) ? -1.f : 1.f) * t.c2g[sidx * g + (g - 1 - ii)];
    double hmax = 0;
    for (int x = 0; x < o * o; x++) hmax = fmax(hmax, fabs((double)t.hi[x]));
    for (int ii = 1; ii < o; ii += 2) {
      ok = ok && fabs((double)t.hi[hs * o + ii]) <= 1e-6 * hmax;
      if (ii <= hs) ok = ok && fabs((double)t.recon[((hs / 2) * o + hs / 2) * o + ii]) <= 1e-6 * rmax;
    }
    return ok;
  };
  if (ord == 5) {
    Tables32<5> t;
    fill(t, 5, 3);
    if (!structure_ok(t, 5, 3)) return cudaErrorInvalidValue;
    return cudaMemcpyToSymbol(c32_tab5, &t, sizeof t);
  }
  Tables32<9> t;
  fill(t, 9, 5);
  if (!structure_ok(t, 9, 5)) return cudaErrorInvalidValue;
  return cudaMemcpyToSymbol(c32_tab9, &t, sizeof t);
}

}  // namespace awfl
