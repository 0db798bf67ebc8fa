// Tracer transport of the FP32 precision form: the reference's tracer code (Spatial:624-955
// and the y/z equivalents, compiled out there by NO_TRACERS) in FP32 arithmetic beside the
// FP32 form's state split, as the reference applies tracer tendencies in every precision
// (Temporal_ader.h:67-69). The tracers stay FP64 arrays (rho*tracer, the layout of the FP64
// path's), the way the FP32 state keeps a compensation plane beside its FP32 values: the
// reconstruction, the ADER series, the fluxes and the limiter run in FP32, the division
// by the density and the update in FP64. Per directional split:
//
//   tracer_divide_kernel   tracers /= (rho' + rho_h), in place (awfl_trc.cuh)
//   sweep_kernel<P32Trc>   the FP32 form's fused state split (the P32 arithmetic) that also
//                          records, per cell, the total density and normal-momentum ADER
//                          series, the pre-split rho' and the reciprocal densities of the
//                          GLL points, and per face the FP32 form's Riemann mass flux, the
//                          upwind velocity and density and the limiter's velocity
//   tracer_cell32_kernel   per cell and tracer: reconstruction of tracer/density, the
//                          rho*tracer ADER series (diffTransformTracer, Spatial:2095-2125),
//                          its edge time average (Spatial:760-809, 1123-1170, 1500-1548) and
//                          the upwind tracer fluxes of the faces the cell is upwind of
//                          (Spatial:891-901, 1249-1259, 1633-1643)
//   tracer_limit_*_kernel  the positivity limiter with the serial face order's result
//   tracer_update_kernel   tendency, density multiplied back, apply; halos as the reference
//                          leaves them (awfl_trc.cuh)
// Compiled with the FP32 form's flags (multiply-add contraction, fast division).
#include <cuda_runtime.h>

#include <type_traits>

#include "awfl_fp32.cuh"
#include "awfl_internal.h"

namespace awfl {

// Recording FP32 policy: the P32 arithmetic plus the tracer split's records (floats; the
// layout of trc_cell_planes: R is the total density series, U the normal momentum; the
// reciprocal planes Y and YUP stay unused, recomputed where they are needed), A.tend
// pointing at the record base.
// 4 CTAs per SM at ord 5 (at most 128 registers, no spills): 3% faster per step with
// tracers than the compiler's choice of 133-134 registers for the x and y sweeps, and than 5
#ifndef AWFL_TRC32_SWEEP_MINB
#define AWFL_TRC32_SWEEP_MINB 4
#endif
struct P32Trc : P32 {
  static constexpr bool kSlab = false;
  static constexpr bool kFaceRec = true;
  static constexpr int min_blocks(int ord) { return ord == 5 ? AWFL_TRC32_SWEEP_MINB : 1; }
  template <int ORD> struct Rec {
    float *base;
    long n, cell;
    int nm;
    template <class Q, class Rt> __device__ __forceinline__ void series32(const Q &q, const Rt &rtot) const {
      constexpr int NG = OrdTraits<ORD>::NGLL;
      constexpr long NS = trc_series_planes<NG>();
#pragma unroll
      for (int kt = 0; kt < NG - 1; kt++)
#pragma unroll
        for (int ii = 0; ii < NG; ii++) {
          base[(kt * NG + ii) * n + cell] = kt == 0 ? rtot[ii] : q[idR][kt][ii];
          base[(NS + kt * NG + ii) * n + cell] = q[nm][kt][ii];
        }
    }
  };
  template <int ORD, int DIR, class S>
  static __device__ __forceinline__ void recon(const S &sten, int kb, const Args &A, float (&eL)[5], float (&eR)[5],
                                               float &src, long cell) {
    if (cell < 0) {  // the periodic prologue's repeat of cell L-1: recorded in its chunk
      cell_recon32<ORD, DIR>(sten, kb, A, eL, eR, src);
      return;
    }
    constexpr int NG = OrdTraits<ORD>::NGLL;
    constexpr int HS = (ORD - 1) / 2;
    const long n = (long)A.nx * A.ny * A.nz;
    cell_recon32<ORD, DIR>(sten, kb, A, eL, eR, src, Rec<ORD>{A.tend, n, cell, 1 + DIR});
    A.tend[2 * trc_series_planes<NG>() * n + cell] = sten(idR, HS);
  }
  // the face records, from the perturbation states the sweep's own Riemann flux saw: the
  // sides' total densities with the background riemann32 gives them (z: the face's own
  // rows, a periodic face 0 taking the top face's)
  template <int ORD, int DIR>
  static __device__ __forceinline__ void face_rec(const Args &A, long face, int kf, const float (&qL)[5],
                                                  const float (&qR)[5], const float (&F)[5]) {
    constexpr int NG = OrdTraits<ORD>::NGLL;
    constexpr int HS = (ORD - 1) / 2;
    constexpr int NM = 1 + DIR;
    const long n = (long)A.nx * A.ny * A.nz, nfm = (long)(A.nx + 1) * (A.ny + 1) * (A.nz + 1);
    float bL, bR;
    if (DIR == 2) {
      bL = A.bg.rho_f[(kf == 0 && A.bc == BC_PERIODIC) ? A.nz : kf];
      bR = A.bg.rho_f[(kf == A.nz && A.bc == BC_PERIODIC) ? 0 : kf];
    } else {
      bL = bR = A.bg.rho_c[HS + kf];
    }
    const float rL = bL + qL[0], rR = bR + qR[0];
    const float vn = DIR == 1 ? 0.5f * (qL[NM] + qR[NM]) : 0.5f * (qL[NM] / rL + qR[NM] / rR);
    float *fr = A.tend + trc_cell_planes<NG>() * n + face;
    fr[0] = F[0];
    fr[nfm] = vn;
    fr[2 * nfm] = 0.5f * (qL[NM] + qR[NM]);
    fr[3 * nfm] = vn > 0 ? rL : rR;
  }
};

template <int ORD, int DIR> struct PolicyShape<P32Trc, ORD, DIR> : PolicyShape<P32, ORD, DIR> {};

namespace {

struct TracerArgs32 {
  using Flux = float;
  SweepArgs32 A;             // the FP32 split's arguments (background, grid, bc, dt)
  const double *dens_c;      // (nz+2hs): rho_h of the cell rows, FP64
  double dt, dxd;            // FP64 time step and spacing of the update
  double *tr;                // (ntr, nz+2hs, ny+2hs, nx+2hs), rho*tracer, FP64
  int ntr;
  unsigned long long pos;    // bit l: tracer l is positive definite (limited)
  const float *R, *U;        // (ngll*(ngll-1), ncell): recorded total density / normal-momentum series
  const float *D;            // (ncell): recorded pre-split rho'
  const float *F0, *VN, *UN, *RUP;  // (nface) each: the recorded face values
  float *TF, *TF2;           // (ntr, nface): unscaled / limited tracer fluxes
  int *flag, *list, *count;  // the limiter's lines to redo in serial order: flags, list, length
};

// The FP32 form's arithmetic of the shared kernels (awfl_trc.cuh): the division by the
// density and the update in FP64 on the FP64 tracers, the limiter in FP32.
__device__ __forceinline__ double trc_divisor(const TracerArgs32 &T, int hs, int k, long g) {
  return (double)T.A.state[g] + T.dens_c[hs + k];
}
__device__ __forceinline__ float trc_dens(const TracerArgs32 &T, int hs, int k) { return T.A.bg.rho_c[hs + k]; }
__device__ __forceinline__ float trc_div_up(const TracerArgs32 &T, float a, long fi) { return a * frcp(T.RUP[fi]); }
__device__ __forceinline__ float limit_face(const TracerArgs32 &T, float F, float f1, float f2, double q, float dens) {
  const float eps = 1.e-10f;
  const float fluxOut = T.A.dt * (f2 - f1) * T.A.inv_dxd;
  const float r = (float)q * dens / (fluxOut + eps);
  return F * (1.f < r ? 1.f : r);  // F * min(1, r)
}
__device__ __forceinline__ double trc_update(const TracerArgs32 &T, double q, int hs, int k, long c, float Fl,
                                             float Fr) {
  const double dens = (double)T.D[c] + T.dens_c[hs + k];  // the divisor of tracer_divide_kernel
  const double tend = (double)((Fl - Fr) * T.A.inv_dxd);
  return q * dens + T.dt * tend;
}

}  // namespace
}  // namespace awfl

// The limiter, update and division kernels are bound by memory latency, not bandwidth:
// registers capped for 16 CTAs of 128 threads per SM (32) made the FP32 form's step with
// three tracers 16% faster than the compiler's 36-64 registers (12 CTAs: slower)
#ifndef AWFL_TRC_LIMIT_MINB
#define AWFL_TRC_LIMIT_MINB 16
#endif
#ifndef AWFL_TRC_UPDATE_MINB
#define AWFL_TRC_UPDATE_MINB 16
#endif
#ifndef AWFL_TRC_DIVIDE_MINB
#define AWFL_TRC_DIVIDE_MINB 16
#endif
#include "awfl_trc.cuh"

namespace awfl {
namespace {

// One lane or a pair of lanes (two tracers on the paired FP32 instructions: one
// instruction, two results, each rounded like the scalar operation).
__device__ __forceinline__ float lane_of(float x, int) { return x; }
__device__ __forceinline__ float lane_of(F2 x, int w) { return w ? x.v.y : x.v.x; }
template <class TT> __device__ __forceinline__ TT pair_of(float a, float b);
template <> __device__ __forceinline__ float pair_of<float>(float a, float) { return a; }
template <> __device__ __forceinline__ F2 pair_of<F2>(float a, float b) { return F2(a, b); }
__device__ __forceinline__ bool is_zero(float x) { return x == 0.f; }
__device__ __forceinline__ bool is_zero(F2 x) { return x.v.x == 0.f && x.v.y == 0.f; }
// max(0, x) on the lanes whose tracer is positive definite
__device__ __forceinline__ float clamp_pos(float x, bool p0, bool) { return p0 ? fmaxf(0.f, x) : x; }
__device__ __forceinline__ F2 clamp_pos(F2 x, bool p0, bool p1) {
  return F2(p0 ? fmaxf(0.f, x.v.x) : x.v.x, p1 ? fmaxf(0.f, x.v.y) : x.v.y);
}

// Tracers l0 (TT = float) or l0 and l0+1 (TT = F2) of one cell: reconstruction of
// tracer/density, times the recorded density, the rho*u*tracer series and
// diffTransformTracer (Spatial:2095-2125) along the recorded series, the edge time average
// (Spatial:2153-2177) and the fluxes of the faces the cell is upwind of. t0, t1: the
// tracers at this cell; off: the stencil's offsets from it; rser, ruser, ry: the cell's
// recorded density and normal-momentum series and reciprocal densities.
template <int ORD, class TT>
__device__ __forceinline__ void tracer_cell32_body(const TracerArgs32 &T, const double *t0, const double *t1,
                                                   const long (&off)[ORD],
                                                   const float (&rser)[OrdTraits<ORD>::NGLL - 1][OrdTraits<ORD>::NGLL],
                                                   const float (&ruser)[OrdTraits<ORD>::NGLL - 1][OrdTraits<ORD>::NGLL],
                                                   const float (&ry)[OrdTraits<ORD>::NGLL], int l0,
                                                   const UpwindFaces &U, float *TF, long nface) {
  constexpr int NG = OrdTraits<ORD>::NGLL;
  constexpr int NL = std::is_same<TT, F2>::value ? 2 : 1;
  const SweepArgs32 &A = T.A;
  const bool pos0 = (T.pos >> l0) & 1ull, pos1 = NL == 2 && ((T.pos >> (l0 + 1)) & 1ull);
  TT s[ORD];
#pragma unroll
  for (int m = 0; m < ORD; m++) s[m] = pair_of<TT>((float)t0[off[m]], (float)t1[off[m]]);
  TT rt[NG][NG], rut[NG][NG];
  // stencils of zeros (tracers absent from this part of the domain) reconstruct to +0 at
  // every GLL point, WENO or not: every sum starts at +0 and adds products with a zero
  // factor, and the weights stay finite (eps keeps them off 1/0)
  bool zero = true;
#pragma unroll
  for (int m = 0; m < ORD; m++) zero = zero && is_zero(s[m]);
  if (zero) {
#pragma unroll
    for (int ii = 0; ii < NG; ii++) rt[0][ii] = TT(0.f);
  } else {
    reconstruct_gll32<ORD>(s, rt[0], A.weno_s != 0);
  }
  const Tables32<ORD> &TB = tab32<ORD>();
#pragma unroll
  for (int ii = 0; ii < NG; ii++) rt[0][ii] = clamp_pos(rt[0][ii] * rser[0][ii], pos0, pos1);
#pragma unroll
  for (int ii = 0; ii < NG; ii++) rut[0][ii] = (rt[0][ii] * ruser[0][ii]) * ry[ii];
#pragma unroll
  for (int kt = 0; kt < NG - 1; kt++) {
    const float sc = -A.inv_dxd * (1.0f / (kt + 1));
#pragma unroll
    for (int ii = 0; ii < NG; ii++) {
      TT df = TT(0.f);
#pragma unroll
      for (int q = 0; q < NG; q++) df = fmaT(TB.deriv[q * NG + ii], rut[kt][q], df);
      rt[kt + 1][ii] = df * sc;
    }
    if (kt + 1 < NG - 1) {  // the last level of rho*u*tracer reaches no edge
#pragma unroll
      for (int ii = 0; ii < NG; ii++) {
        TT tot = TT(0.f);
#pragma unroll
        for (int ir = 0; ir <= kt + 1; ir++) {
          tot = fmaT(ruser[ir][ii], rt[kt + 1 - ir][ii], tot);
          if (ir != 0) tot = fmaT(-rser[ir][ii], rut[kt + 1 - ir][ii], tot);  // rut[kt+1] is not known yet
        }
        rut[kt + 1][ii] = tot * ry[ii];
      }
    }
  }
  TT tl = rt[0][0], trr = rt[0][NG - 1];
  float dtmult = A.dt;
#pragma unroll
  for (int kt = 1; kt < NG; kt++) {
    const float cf = dtmult * (1.0f / (kt + 1));
    tl = fmaT(rt[kt][0], cf, tl);
    trr = fmaT(rt[kt][NG - 1], cf, trr);
    dtmult *= A.dt;
  }
  tl = clamp_pos(tl, pos0, pos1);
  trr = clamp_pos(trr, pos0, pos1);
#pragma unroll
  for (int w = 0; w < NL; w++) put_upwind_fluxes<float>(T, TF + w * nface, U, lane_of(tl, w), lane_of(trr, w));
}

// One thread per cell for all its tracers, two at a time on the paired FP32 instructions
// (a last single tracer on one lane): the cell's records, stencil offsets and upwind faces
// are read and worked out once.
#ifndef AWFL_TRC32_CELL_MINB
#define AWFL_TRC32_CELL_MINB 8
#endif
template <int ORD, int DIR>
__global__ void __launch_bounds__(128, ORD == 5 ? AWFL_TRC32_CELL_MINB : 1) tracer_cell32_kernel(TracerArgs32 T) {
  constexpr int HS = (ORD - 1) / 2;
  constexpr int NG = OrdTraits<ORD>::NGLL;
  const SweepArgs32 &A = T.A;
  const Geo<DIR> G(A, HS);
  const unsigned ncell = (unsigned)G.nz * G.ny * G.nx;
  const unsigned c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncell) return;
  if (c < G.nlines()) T.flag[c] = 0;  // the limiter's per-line flags (ncell >= nlines)
  if (c == 0) *T.count = 0;
  int i, j, k;
  unflat(c, G.nx, G.ny, k, j, i);
  const int p0 = DIR == 0 ? i : (DIR == 1 ? j : k);
  const int n = G.n();
  // the stencil's state offsets along the line; halo positions read the interior cell
  // whose value the boundary condition copies there
  const long gsd = DIR == 0 ? 1 : (DIR == 1 ? G.sy : G.sz);
  long off[ORD];
  if (p0 >= HS && p0 < n - HS) {
#pragma unroll
    for (int m = 0; m < ORD; m++) off[m] = (m - HS) * gsd;
  } else {
#pragma unroll
    for (int m = 0; m < ORD; m++) {
      bool wall;
      off[m] = (halo_src(p0 - HS + m, n, A.bc, wall) - p0) * gsd;
    }
  }
  float rser[NG - 1][NG], ruser[NG - 1][NG], ry[NG];
  {
    const float *r = T.R + c, *u = T.U + c;  // plane by plane, ncell apart
#pragma unroll
    for (int kt = 0; kt < NG - 1; kt++)
#pragma unroll
      for (int ii = 0; ii < NG; ii++) {
        rser[kt][ii] = *r;
        ruser[kt][ii] = *u;
        r += ncell;
        u += ncell;
      }
  }
  // 1/rho of the GLL points: the recording sweep's own reciprocal of the same value
#pragma unroll
  for (int ii = 0; ii < NG; ii++) ry[ii] = frcp(rser[0][ii]);
  const long fs = DIR == 0 ? 1 : (DIR == 1 ? G.nx : (long)G.nx * G.ny), fl = G.face(k, j, i);
  const UpwindFaces U = upwind_faces(T, p0, n, A.bc == BC_PERIODIC, fl, fs, fl - p0 * fs);
  const long nface = G.nface();
  const double *t = T.tr + G.g(k, j, i);
  for (int l = 0; l < T.ntr; l += 2) {
    if (l + 1 < T.ntr)
      tracer_cell32_body<ORD, F2>(T, t + l * G.sv, t + (l + 1) * G.sv, off, rser, ruser, ry, l, U, T.TF + l * nface,
                                  nface);
    else
      tracer_cell32_body<ORD, float>(T, t + l * G.sv, t + l * G.sv, off, rser, ruser, ry, l, U, T.TF + l * nface,
                                     nface);
  }
}

template <int ORD, int DIR>
cudaError_t run32(const TracerArgs32 &T, int io, cudaStream_t st) {
  constexpr int HS = (ORD - 1) / 2;
  constexpr int NG = OrdTraits<ORD>::NGLL;
  const SweepArgs32 &A = T.A;
  const long ncell = (long)A.nz * A.ny * A.nx;
  const long nf = (long)(A.nz + (DIR == 2)) * (A.ny + (DIR == 1)) * (A.nx + (DIR == 0));
  const unsigned gc = (unsigned)((ncell + 127) / 128), gf = (unsigned)((nf + 127) / 128);
  if (!(io & TRC_IN_DIVIDED)) tracer_divide_kernel<TracerArgs32><<<gc, 128, 0, st>>>(T, HS);
  cudaError_t e = launch_sweep_t<P32Trc, ORD, DIR>(A, st);  // state split + records
  if (e != cudaSuccess) return e;
  tracer_cell32_kernel<ORD, DIR><<<gc, 128, 0, st>>>(T);
  const long nlines = DIR == 0 ? (long)A.nz * A.ny : (DIR == 1 ? (long)A.nz * A.nx : (long)A.ny * A.nx);
  tracer_limit_faces_kernel<TracerArgs32, DIR><<<gf, 128, 0, st>>>(T, HS);
  const long lw = (nlines * T.ntr + 3) / 4;  // one warp per flagged line and tracer, grid-strided
  tracer_limit_lines_kernel<TracerArgs32, DIR><<<(unsigned)(lw < 148 * 8 ? lw : 148 * 8), 128, 0, st>>>(T, HS);
  tracer_update_kernel<TracerArgs32, DIR><<<gc, 128, 0, st>>>(T, HS, (io & TRC_OUT_DIVIDED) != 0);
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_split_tracers32(int ord, int dir, const SweepArgs32 &Ain, const double *dens_c, double dt,
                                   double dxd, double *tracers, int ntr, unsigned long long pos, float *scratch,
                                   int io, cudaStream_t st) {
  const int ng = ord == 5 ? 3 : 5;
  const long ncell = (long)Ain.nz * Ain.ny * Ain.nx;
  const long nfmax = (long)(Ain.nz + 1) * (Ain.ny + 1) * (Ain.nx + 1);
  if (nfmax >= (1L << 31)) return cudaErrorInvalidValue;  // 32-bit cell and face indices
  TracerArgs32 T;
  T.A = Ain;
  T.A.tend = scratch;  // the recording sweep's record base
  T.A.mode = MODE_APPLY;
  T.dens_c = dens_c;
  T.dt = dt;
  T.dxd = dxd;
  T.tr = tracers;
  T.ntr = ntr;
  T.pos = pos;
  const long ns = (long)ng * (ng - 1), ncp = 2 * ns + 1 + ng;  // trc_series_planes, trc_cell_planes
  T.R = scratch;
  T.U = scratch + ns * ncell;
  T.D = scratch + 2 * ns * ncell;
  T.F0 = scratch + ncp * ncell;
  T.VN = T.F0 + nfmax;
  T.UN = T.VN + nfmax;
  T.RUP = T.UN + nfmax;
  T.TF = scratch + ncp * ncell + 5 * nfmax;
  T.TF2 = T.TF + (long)ntr * nfmax;
  T.flag = reinterpret_cast<int *>(T.TF2 + (long)ntr * nfmax);
  long lines = (long)Ain.nz * Ain.ny;  // as tracer_scratch_bytes
  if ((long)Ain.nz * Ain.nx > lines) lines = (long)Ain.nz * Ain.nx;
  if ((long)Ain.ny * Ain.nx > lines) lines = (long)Ain.ny * Ain.nx;
  T.list = T.flag + lines;
  T.count = T.list + lines;
  if (ord == 5) {
    if (dir == 0) return run32<5, 0>(T, io, st);
    if (dir == 1) return run32<5, 1>(T, io, st);
    return run32<5, 2>(T, io, st);
  }
  if (dir == 0) return run32<9, 0>(T, io, st);
  if (dir == 1) return run32<9, 1>(T, io, st);
  return run32<9, 2>(T, io, st);
}

cudaError_t upload_tables_tracers32(int ord, const double *recon, const double *c2g, const double *s2g,
                                    const double *deriv, const double *idl, double sigma, const double *wts) {
  return upload_tables32_here(ord, recon, c2g, s2g, deriv, idl, sigma, wts);
}

}  // namespace awfl
