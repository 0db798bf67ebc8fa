// Tracer transport of the FP64 path: the reference's tracer code, which it compiles out
// with NO_TRACERS (Spatial:10), built in. Per directional split:
//
//   tracer_divide_kernel  tracers /= density, in place (Spatial:624-627)
//   sweep_kernel<P64Trc>  the state's fused split (the P64 arithmetic, so the state is
//                         bit-identical to awfl_split's) that also records, per cell, the
//                         density and normal-momentum ADER series, the pre-split density
//                         perturbation and, per face, the Riemann mass flux, the upwind
//                         velocity and density and the limiter's velocity
//   tracer_cell_kernel    per cell and tracer: the reconstruction of tracer/density, the
//                         rho*tracer ADER series (diffTransformTracer, Spatial:2095-2125)
//                         along the recorded series, its edge time average
//                         (Spatial:760-809, 1123-1170, 1500-1548) and the upwind tracer
//                         fluxes of the faces the cell is upwind of (Spatial:891-901, with
//                         the edge BCs of Spatial:816-837) from the recorded face values
//   tracer_limit_faces_kernel / tracer_limit_lines_kernel
//                         the positivity limiter (Spatial:904-935, 1262-1293, 1646-1677)
//                         with the result of the reference's serial face order: per face,
//                         then the few lines where that order matters again in series
//   tracer_update_kernel  per cell: tendency, density multiplied back, apply
//                         (Spatial:948-955; Temporal_ader.h:67-69), and the halo cells of
//                         this direction left holding tracer/density, as the reference's
//                         in-place halo fill leaves them
//
// Decisions where the reference's code is not well defined: the limiter follows the
// reference's serial loop order (it scales tracerFlux in place while other iterations of
// its parallel_for read it, so only the serial order gives one result); the y branch for v < 0 reads the faces along y (the reference indexes tracerFlux(tr,k,j,ind_j),
// Spatial:1285-1286); a periodic z wraps like x and y (the reference reads outside the
// array there). Stencil halos are computed from the boundary conditions (periodic wrap;
// wall: the edge cell, the state's normal momentum zero), as the reference's halo fill
// writes them. Compiled with --fmad=false like the FP64 path.
#include <cuda_runtime.h>

#include "awfl_internal.h"
#include "awfl_p64.cuh"

namespace awfl {

// Recording FP64 policy: the P64 arithmetic plus the records above, written by the sweep
// itself (A.tend points at the record base): the cell records from cell_recon's series,
// the face records from every face flux it computes.
// 4 CTAs per SM at ord 5, as the plain sweep: 40-72 bytes of spills, 4% faster per step
// with tracers than 3 CTAs without spills (256x256x128, three tracers)
#ifndef AWFL_TRC_SWEEP_MINB
#define AWFL_TRC_SWEEP_MINB 4
#endif
struct P64Trc : P64 {
  static constexpr bool kSlab = false;
  static constexpr bool kFaceRec = true;
  // CTAs per SM (AWFL_TRC_SWEEP_MINB above)
  static constexpr int min_blocks(int ord) { return ord == 5 ? AWFL_TRC_SWEEP_MINB : 1; }
  template <int ORD> struct Rec {
    double *base;
    long n, cell;
    int nm;
    __device__ __forceinline__ void level0(int, int, const double &) const {}
    template <class Q> __device__ __forceinline__ void series(const Q &q) const {
      constexpr int NG = OrdTraits<ORD>::NGLL;
      constexpr long NS = trc_series_planes<NG>();
#pragma unroll
      for (int kt = 0; kt < NG - 1; kt++)
#pragma unroll
        for (int ii = 0; ii < NG; ii++) {
          base[(kt * NG + ii) * n + cell] = q[idR][kt][ii];
          base[(NS + kt * NG + ii) * n + cell] = q[nm][kt][ii];
        }
      // RN(1 / density) of the GLL points (the sweep's own reciprocals, rr in cell_recon)
#pragma unroll
      for (int ii = 0; ii < NG; ii++) base[(2 * NS + 1 + ii) * n + cell] = 1.0 / q[idR][0][ii];
    }
  };
  template <int ORD, int DIR, class S>
  static __device__ __forceinline__ void recon(const S &sten, int kb, const Args &A, double (&eL)[5],
                                               double (&eR)[5], double &src, long cell) {
    if (cell < 0) {  // the periodic prologue's repeat of cell L-1: recorded in its chunk
      cell_recon<ORD, DIR>(sten, kb, A, eL, eR, src);
      return;
    }
    constexpr int NG = OrdTraits<ORD>::NGLL;
    constexpr int HS = (ORD - 1) / 2;
    const long n = (long)A.nx * A.ny * A.nz;
    cell_recon<ORD, DIR>(sten, kb, A, eL, eR, src, Rec<ORD>{A.tend, n, cell, 1 + DIR});
    A.tend[2 * trc_series_planes<NG>() * n + cell] = sten(idR, HS);
  }
  // the face records: the tracer face flux's inputs (Spatial:891-901), from the states the
  // sweep's own Riemann flux saw
  template <int ORD, int DIR>
  static __device__ __forceinline__ void face_rec(const Args &A, long face, int, const double (&qL)[5],
                                                  const double (&qR)[5], const double (&F)[5]) {
    constexpr int NG = OrdTraits<ORD>::NGLL;
    constexpr int NM = 1 + DIR;
    const long n = (long)A.nx * A.ny * A.nz, nfm = (long)(A.nx + 1) * (A.ny + 1) * (A.nz + 1);
    double *fr = A.tend + trc_cell_planes<NG>() * n + face;
    const double vn = DIR == 1 ? 0.5 * (qL[NM] + qR[NM]) : 0.5 * (qL[NM] / qL[0] + qR[NM] / qR[0]);
    fr[0] = F[0];
    fr[nfm] = vn;
    fr[2 * nfm] = 0.5 * (qL[NM] + qR[NM]);
    const double rup = vn > 0 ? qL[0] : qR[0];
    fr[3 * nfm] = rup;
    fr[4 * nfm] = 1.0 / rup;  // RN(1/rup): the tracer fluxes' shared divisor
  }
};

template <int ORD, int DIR> struct PolicyShape<P64Trc, ORD, DIR> : PolicyShape<P64, ORD, DIR> {};

namespace {

struct TracerArgs {
  using Flux = double;
  SweepArgs A;               // background, grid, bc, dt of this split
  double *tr;                // (ntr, nz+2hs, ny+2hs, nx+2hs), rho*tracer
  int ntr;
  unsigned long long pos;    // bit l: tracer l is positive definite (limited)
  const double *R, *U;       // (ngll*(ngll-1), ncell): recorded density / normal-momentum series
  const double *D;           // (ncell): recorded pre-split rho'
  const double *Y;           // (ngll, ncell): recorded RN(1 / rho) of the GLL points
  const double *F0, *VN, *UN, *RUP, *YUP;  // (nface) each: the recorded face values
  double *TF, *TF2;          // (ntr, nface): unscaled / limited tracer fluxes
  int *flag, *list, *count;  // the limiter's lines to redo in serial order: flags, list, length
};

// The FP64 path's arithmetic of the shared kernels (awfl_trc.cuh): the reference's
// expressions in its order, IEEE division.
__device__ __forceinline__ double trc_divisor(const TracerArgs &T, int hs, int k, long g) {
  return T.A.state[g] + T.A.dens_c[hs + k];
}
__device__ __forceinline__ double trc_dens(const TracerArgs &T, int hs, int k) { return T.A.dens_c[hs + k]; }
// a / (the upwind density of face fi), correctly rounded through its recorded reciprocal
__device__ __forceinline__ double trc_div_up(const TracerArgs &T, double a, long fi) {
  return divr_any(a, rcp_known(T.RUP[fi], T.YUP[fi]));
}
// factor and scaled flux of one face from its upwind cell's two faces (f1 = min(., 0) of
// the left one, f2 = max(., 0) of the right one; q: the cell's tracer / density)
__device__ __forceinline__ double limit_face(const TracerArgs &T, double F, double f1, double f2, double q,
                                             double dens) {
  const double eps = 1.e-10;
  const double fluxOut = divr_any(T.A.dt * (f2 - f1), rcp_known(T.A.dxd, T.A.rdxd));
  const double r = q * dens / (fluxOut + eps);
  return F * (1. < r ? 1. : r);  // F * min(1, r)
}
__device__ __forceinline__ double trc_update(const TracerArgs &T, double q, int hs, int k, long c, double Fl,
                                             double Fr) {
  const double dens = T.D[c] + T.A.dens_c[hs + k];
  const double tend = -(Fr - Fl) / T.A.dxd;
  return q * dens + T.A.dt * tend;  // Spatial:952-953, then Temporal_ader.h:67-69
}

}  // namespace
}  // namespace awfl

// The limiter, update and division kernels are bound by memory latency, not bandwidth:
// registers capped for 16 (limiter, division: 32 registers) and 12 (update: 40) CTAs of 128
// threads per SM, a few bytes of spills, made the FP64 step with three tracers 10% faster
// than the compiler's 36-72 registers (12 for the limiter, or 16 for the update: slower)
#ifndef AWFL_TRC_LIMIT_MINB
#define AWFL_TRC_LIMIT_MINB 16
#endif
#ifndef AWFL_TRC_UPDATE_MINB
#define AWFL_TRC_UPDATE_MINB 12
#endif
#ifndef AWFL_TRC_DIVIDE_MINB
#define AWFL_TRC_DIVIDE_MINB 16
#endif
#include "awfl_trc.cuh"

namespace awfl {
namespace {

// ord 5: 8 CTAs per SM (64 registers; measured 5% faster than 6 CTAs at 78 registers,
// the compiler's choice, despite a 16-byte spill)
#ifndef AWFL_TRC_CELL_MINB
#define AWFL_TRC_CELL_MINB 8
#endif
// One thread per cell and tracer; the blocks of one run of 128 cells are consecutive for
// the tracers (block b: cells (b / ntr) * 128 .., tracer b % ntr), so the recorded series
// that they share is read from DRAM once.
template <int ORD, int DIR>
__global__ void __launch_bounds__(128, ORD == 5 ? AWFL_TRC_CELL_MINB : 1) tracer_cell_kernel(TracerArgs T) {
  constexpr int HS = (ORD - 1) / 2;
  constexpr int NG = OrdTraits<ORD>::NGLL;
  const SweepArgs &A = T.A;
  const Geo<DIR> G(A, HS);
  const unsigned ncell = (unsigned)G.nz * G.ny * G.nx;
  const unsigned cb = blockIdx.x / (unsigned)T.ntr;
  const int l = (int)(blockIdx.x - cb * (unsigned)T.ntr);
  const unsigned c = cb * blockDim.x + threadIdx.x;
  if (c >= ncell) return;
  if (l == 0 && c < G.nlines()) T.flag[c] = 0;  // the limiter's per-line flags (ncell >= nlines)
  if (l == 0 && c == 0) *T.count = 0;
  int i, j, k;
  unflat(c, G.nx, G.ny, k, j, i);
  const int p0 = DIR == 0 ? i : (DIR == 1 ? j : k);
  const int n = G.n();
  const bool posdef = (T.pos >> l) & 1ull;
  // the stencil of tracer / density (divided by tracer_divide_kernel); halo positions
  // read the interior cell whose value the boundary condition copies there
  const double *tr = T.tr + l * G.sv + G.g(k, j, i);  // this cell's tracer
  const long gsd = DIR == 0 ? 1 : (DIR == 1 ? G.sy : G.sz);  // state stride along the line
  double s[ORD];
  if (p0 >= HS && p0 < n - HS) {  // the whole stencil inside the line
#pragma unroll
    for (int m = 0; m < ORD; m++) s[m] = tr[(m - HS) * gsd];
  } else {
#pragma unroll
    for (int m = 0; m < ORD; m++) {
      bool wall;
      const int p = halo_src(p0 - HS + m, n, A.bc, wall);
      s[m] = tr[(p - p0) * gsd];
    }
  }
  double rt[NG][NG], rut[NG][NG];
  // a stencil of zeros (a tracer absent from this part of the domain) reconstructs to +0
  // at every GLL point, WENO or not: every sum of the reconstruction starts at +0 and adds
  // products with a zero factor, and its weights stay finite (eps keeps them off 1/0)
  bool zero = true;
#pragma unroll
  for (int m = 0; m < ORD; m++) zero = zero && s[m] == 0.;
  if (zero) {
#pragma unroll
    for (int ii = 0; ii < NG; ii++) rt[0][ii] = 0.;
  } else {
    reconstruct_gll_any<ORD>(s, rt[0], A.weno_s != 0);
  }
  double rser[NG - 1][NG], ruser[NG - 1][NG];
  {
    const double *r = T.R + c, *u = T.U + c;  // plane by plane, ncell apart
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
  // the divisors through their correctly rounded reciprocals (IEEE quotients bit for bit):
  // the GLL points' densities (reciprocals recorded by the sweep) and dx
  Rcp<double> rr[NG];
  {
    const double *y = T.Y + c;
#pragma unroll
    for (int ii = 0; ii < NG; ii++) rr[ii] = rcp_known(rser[0][ii], y[ii * (long)ncell]);
  }
  const Rcp<double> rdx = rcp_known(A.dxd, A.rdxd);
  const Tables<ORD> &TB = tab<ORD>();
#pragma unroll
  for (int ii = 0; ii < NG; ii++) {
    rt[0][ii] *= rser[0][ii];
    if (posdef) rt[0][ii] = dmax(0., rt[0][ii]);
  }
#pragma unroll
  for (int ii = 0; ii < NG; ii++) rut[0][ii] = divr_any(rt[0][ii] * ruser[0][ii], rr[ii]);
  // diffTransformTracer (Spatial:2095-2125)
#pragma unroll
  for (int kt = 1; kt < NG; kt++)
#pragma unroll
    for (int ii = 0; ii < NG; ii++) rut[kt][ii] = 0;
#pragma unroll
  for (int kt = 0; kt < NG - 1; kt++) {
#pragma unroll
    for (int ii = 0; ii < NG; ii++) {
      double df = 0;
#pragma unroll
      for (int q = 0; q < NG; q++) df += TB.deriv[q * NG + ii] * rut[kt][q];
      rt[kt + 1][ii] = divk_any(divr_any(-df, rdx), kt + 1);
    }
    if (kt + 1 < NG - 1) {  // the last level of rho*u*tracer reaches no edge
#pragma unroll
      for (int ii = 0; ii < NG; ii++) {
        double tot = 0;
#pragma unroll
        for (int ir = 0; ir <= kt + 1; ir++)
          tot += ruser[ir][ii] * rt[kt + 1 - ir][ii] - rser[ir][ii] * rut[kt + 1 - ir][ii];
        rut[kt + 1][ii] = divr_any(tot, rr[ii]);
      }
    }
  }
  // compute_timeAvg_edges (Spatial:2153-2177), then the positivity clamp of the edges
  double tl = rt[0][0], trr = rt[0][NG - 1];
  double dtmult = A.dt;
#pragma unroll
  for (int kt = 1; kt < NG; kt++) {
    tl += divk_any(rt[kt][0] * dtmult, kt + 1);
    trr += divk_any(rt[kt][NG - 1] * dtmult, kt + 1);
    dtmult *= A.dt;
  }
  if (posdef) {
    tl = dmax(0., tl);
    trr = dmax(0., trr);
  }
  // the fluxes of the faces this cell is upwind of
  const long fs = DIR == 0 ? 1 : (DIR == 1 ? G.nx : (long)G.nx * G.ny), fl = G.face(k, j, i);
  write_upwind_fluxes<double>(T, T.TF + (long)l * G.nface(), p0, n, A.bc == BC_PERIODIC, fl, fs, fl - p0 * fs, tl, trr);
}

template <int ORD, int DIR>
cudaError_t run(const TracerArgs &T, int io, cudaStream_t st) {
  constexpr int HS = (ORD - 1) / 2;
  constexpr int NG = OrdTraits<ORD>::NGLL;
  const SweepArgs &A = T.A;
  const long ncell = (long)A.nz * A.ny * A.nx;
  const long nf = (long)(A.nz + (DIR == 2)) * (A.ny + (DIR == 1)) * (A.nx + (DIR == 0));
  const unsigned gc = (unsigned)((ncell + 127) / 128), gf = (unsigned)((nf + 127) / 128);
  if (!(io & TRC_IN_DIVIDED)) tracer_divide_kernel<TracerArgs><<<gc, 128, 0, st>>>(T, HS);
  cudaError_t e = launch_sweep_t<P64Trc, ORD, DIR>(A, st);  // state split + records
  if (e != cudaSuccess) return e;
  tracer_cell_kernel<ORD, DIR><<<gc * (unsigned)T.ntr, 128, 0, st>>>(T);
  const long nlines = DIR == 0 ? (long)A.nz * A.ny : (DIR == 1 ? (long)A.nz * A.nx : (long)A.ny * A.nx);
  tracer_limit_faces_kernel<TracerArgs, DIR><<<gf, 128, 0, st>>>(T, HS);
  const long lw = (nlines * T.ntr + 3) / 4;  // one warp per flagged line and tracer, grid-strided
  tracer_limit_lines_kernel<TracerArgs, DIR><<<(unsigned)(lw < 148 * 8 ? lw : 148 * 8), 128, 0, st>>>(T, HS);
  tracer_update_kernel<TracerArgs, DIR><<<gc, 128, 0, st>>>(T, HS, (io & TRC_OUT_DIVIDED) != 0);
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_split_tracers(int ord, int dir, const SweepArgs &Ain, double *tracers, int ntr,
                                 unsigned long long pos, double *scratch, int io, cudaStream_t st) {
  const int ng = ord == 5 ? 3 : 5;
  const long ncell = (long)Ain.nz * Ain.ny * Ain.nx;
  const long nfmax = (long)(Ain.nz + 1) * (Ain.ny + 1) * (Ain.nx + 1);
  if (nfmax >= (1L << 31)) return cudaErrorInvalidValue;  // 32-bit cell and face indices
  TracerArgs T;
  T.A = Ain;
  T.A.tend = scratch;  // the recording sweep's record base
  T.A.mode = MODE_APPLY;
  T.tr = tracers;
  T.ntr = ntr;
  T.pos = pos;
  const long ns = (long)ng * (ng - 1), ncp = 2 * ns + 1 + ng;  // trc_series_planes, trc_cell_planes
  T.R = scratch;
  T.U = scratch + ns * ncell;
  T.D = scratch + 2 * ns * ncell;
  T.Y = T.D + ncell;
  T.F0 = scratch + ncp * ncell;
  T.VN = T.F0 + nfmax;
  T.UN = T.VN + nfmax;
  T.RUP = T.UN + nfmax;
  T.YUP = T.RUP + nfmax;
  T.TF = scratch + ncp * ncell + 5 * nfmax;
  T.TF2 = T.TF + (long)ntr * nfmax;
  T.flag = reinterpret_cast<int *>(T.TF2 + (long)ntr * nfmax);
  long lines = (long)Ain.nz * Ain.ny;  // as tracer_scratch_bytes
  if ((long)Ain.nz * Ain.nx > lines) lines = (long)Ain.nz * Ain.nx;
  if ((long)Ain.ny * Ain.nx > lines) lines = (long)Ain.ny * Ain.nx;
  T.list = T.flag + lines;
  T.count = T.list + lines;
  if (ord == 5) {
    if (dir == 0) return run<5, 0>(T, io, st);
    if (dir == 1) return run<5, 1>(T, io, st);
    return run<5, 2>(T, io, st);
  }
  if (dir == 0) return run<9, 0>(T, io, st);
  if (dir == 1) return run<9, 1>(T, io, st);
  return run<9, 2>(T, io, st);
}

size_t tracer_scratch_bytes(int ord, int nx, int ny, int nz, int ntr, int elem) {
  const int ng = ord == 5 ? 3 : 5;
  const long ncell = (long)nz * ny * nx;
  const long nfmax = (long)(nz + 1) * (ny + 1) * (nx + 1);
  long lines = (long)nz * ny;  // the most lines of one direction: the limiter's flags and list
  if ((long)nz * nx > lines) lines = (long)nz * nx;
  if ((long)ny * nx > lines) lines = (long)ny * nx;
  const long elems = (2L * ng * (ng - 1) + 1 + ng) * ncell + 5 * nfmax + 2L * ntr * nfmax;
  return (size_t)elem * (size_t)elems + sizeof(int) * (2 * (size_t)lines + 1);
}

cudaError_t upload_tables_tracers(int ord, const void *tab, size_t bytes) {
  if (ord == 5) return cudaMemcpyToSymbol(c_tab5, tab, bytes);
  return cudaMemcpyToSymbol(c_tab9, tab, bytes);
}

}  // namespace awfl
