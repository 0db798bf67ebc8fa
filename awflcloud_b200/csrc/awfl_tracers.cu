// Tracer transport of the FP64 path: the reference's tracer code, which it compiles out
// with NO_TRACERS (Spatial:10), built in. Per directional split:
//
//   tracer_divide_kernel  tracers /= density, in place (Spatial:624-627)
//   sweep_kernel<P64Trc>  the state's fused split (the P64 arithmetic, so the state is
//                         bit-identical to awfl_split's) that also records, per cell, the
//                         density and normal-momentum ADER series, the time-averaged edge
//                         states and the pre-split density perturbation
//   tracer_cell_kernel    per cell and tracer: the reconstruction of tracer/density, the
//                         rho*tracer ADER series (diffTransformTracer, Spatial:2095-2125)
//                         along the recorded series and its edge time average
//                         (Spatial:760-809, 1123-1170, 1500-1548)
//   tracer_face_kernel    per face: edge BCs (Spatial:826-835), the state's Riemann flux
//                         (riemann) and the upwind tracer fluxes (Spatial:891-901,
//                         1249-1259, 1633-1643)
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

// Recording FP64 policy: the P64 arithmetic plus, per interior cell, the records the
// tracer kernels read. A.tend points at the record base: R (NG*NG planes of ncell), U
// (NG*NG), E (10: eL, eR), D (1: the pre-split rho', the stencil centre), Y (NG: RN(1/rho)
// of the GLL points).
struct P64Trc : P64 {
  static constexpr bool kSlab = false;
  // the record stores need registers: 3 CTAs per SM at ord 5 instead of the plain sweep's 4
  static constexpr int min_blocks(int ord) { return ord == 5 ? 3 : 1; }
  template <int ORD> struct Rec {
    double *base;
    long n, cell;
    int nm;
    __device__ __forceinline__ void level0(int, int, const double &) const {}
    template <class Q> __device__ __forceinline__ void series(const Q &q) const {
      constexpr int NG = OrdTraits<ORD>::NGLL;
#pragma unroll
      for (int kt = 0; kt < NG; kt++)
#pragma unroll
        for (int ii = 0; ii < NG; ii++) {
          base[(kt * NG + ii) * n + cell] = q[idR][kt][ii];
          base[(NG * NG + kt * NG + ii) * n + cell] = q[nm][kt][ii];
        }
      // RN(1 / density) of the GLL points (the sweep's own reciprocals, rr in cell_recon)
#pragma unroll
      for (int ii = 0; ii < NG; ii++) base[(2 * NG * NG + 11 + ii) * n + cell] = 1.0 / q[idR][0][ii];
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
    double *e = A.tend + 2L * NG * NG * n;
#pragma unroll
    for (int v = 0; v < 5; v++) {
      e[v * n + cell] = eL[v];
      e[(5 + v) * n + cell] = eR[v];
    }
    e[10 * n + cell] = sten(idR, HS);
  }
};

template <int ORD, int DIR> struct PolicyShape<P64Trc, ORD, DIR> : PolicyShape<P64, ORD, DIR> {};

namespace {

struct TracerArgs {
  SweepArgs A;               // background, grid, bc, dt of this split (A.state unused)
  double *tr;                // (ntr, nz+2hs, ny+2hs, nx+2hs), rho*tracer
  int ntr;
  unsigned long long pos;    // bit l: tracer l is positive definite (limited)
  const double *R, *U;       // (ngll*ngll, ncell): recorded density / normal-momentum series
  const double *D;           // (ncell): recorded pre-split rho'
  const double *Y;           // (ngll, ncell): recorded RN(1 / rho) of the GLL points
  double *E;                 // (10, ncell): the state's time-averaged edges eL[5], eR[5]
  double *TE;                // (ntr, 2, ncell): the tracers' edges (left, right)
  double *TF, *TF2, *UN;     // (ntr, nface) unscaled / limited fluxes, (nface) limiter velocity
  int *flag;                 // (nlines): the limiter's lines to redo in serial order
};

__device__ __forceinline__ double dmax(double a, double b) { return a > b ? a : b; }
__device__ __forceinline__ double dmin(double a, double b) { return a < b ? a : b; }

// Along-direction geometry of one split: cells (k, j, i); p = the index along DIR.
template <int DIR> struct Geo {
  int nx, ny, nz, hs;
  long sy, sz, sv;  // state strides (halo-inclusive)
  __device__ Geo(const SweepArgs &A, int hs_) : nx(A.nx), ny(A.ny), nz(A.nz), hs(hs_) {
    sy = nx + 2 * hs;
    sz = (long)(ny + 2 * hs) * sy;
    sv = (long)(nz + 2 * hs) * sz;
  }
  __device__ int n() const { return DIR == 0 ? nx : (DIR == 1 ? ny : nz); }
  __device__ long cell(int k, int j, int i) const { return ((long)k * ny + j) * nx + i; }
  // state offset of interior cell (k, j, i)
  __device__ long g(int k, int j, int i) const { return (long)(hs + k) * sz + (long)(hs + j) * sy + hs + i; }
  // face index (faces along DIR: n+1 per line)
  __device__ long face(int k, int j, int i) const {
    if (DIR == 0) return ((long)k * ny + j) * (nx + 1) + i;
    if (DIR == 1) return ((long)k * (ny + 1) + j) * nx + i;
    return ((long)k * ny + j) * nx + i;
  }
  __device__ long nface() const {
    return (long)(nz + (DIR == 2)) * (ny + (DIR == 1)) * (nx + (DIR == 0));
  }
  // cell (k, j, i) moved to index p along DIR
  __device__ void at(int k, int j, int i, int p, int &kk, int &jj, int &ii) const {
    kk = DIR == 2 ? p : k;
    jj = DIR == 1 ? p : j;
    ii = DIR == 0 ? p : i;
  }
};

// Index p (possibly in the halo) -> the interior index whose value the halo holds, and
// whether it is a wall halo (normal momentum zero).
__device__ __forceinline__ int halo_src(int p, int n, int bc, bool &wall) {
  wall = false;
  if (p >= 0 && p < n) return p;
  if (bc == BC_PERIODIC) return p < 0 ? p + n : p - n;
  wall = true;
  return p < 0 ? 0 : n - 1;
}

// (k, j, i) of a flat index over extents ex (fastest) and ey, in 32-bit arithmetic: the
// tracer path's grids hold fewer than 2^31 cells and faces (launch_split_tracers checks)
__device__ __forceinline__ void unflat(unsigned x, unsigned ex, unsigned ey, int &k, int &j, int &i) {
  const unsigned r = x / ex;
  const unsigned kk = r / ey;
  i = (int)(x - r * ex);
  j = (int)(r - kk * ey);
  k = (int)kk;
}

// tracers /= (rho' + rho_h) on the interior cells, with the state before the split
// (Spatial:624-627). The halos are not touched: every kernel of the split maps a halo
// position to the interior cell whose value it holds.
__global__ void __launch_bounds__(128) tracer_divide_kernel(TracerArgs T, int hs) {
  const SweepArgs &A = T.A;
  const Geo<0> G(A, hs);
  const long ncell = (long)G.nz * G.ny * G.nx;
  const long c = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (c >= ncell) return;
  int i, j, k;
  unflat((unsigned)c, G.nx, G.ny, k, j, i);
  const long g = G.g(k, j, i);
  const double dens = A.state[idR * G.sv + g] + A.dens_c[hs + k];
  for (int l = 0; l < T.ntr; l++) T.tr[l * G.sv + g] /= dens;
}

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
  int i, j, k;
  unflat(c, G.nx, G.ny, k, j, i);
  const int p0 = DIR == 0 ? i : (DIR == 1 ? j : k);
  const int n = G.n();
  const bool posdef = (T.pos >> l) & 1ull;
  // the stencil of tracer / density (divided by tracer_divide_kernel); halo positions
  // read the interior cell whose value the boundary condition copies there
  const double *tr = T.tr + l * G.sv;
  double s[ORD];
#pragma unroll
  for (int m = 0; m < ORD; m++) {
    bool wall;
    const int p = halo_src(p0 - HS + m, n, A.bc, wall);
    int kk, jj, ii;
    G.at(k, j, i, p, kk, jj, ii);
    s[m] = tr[G.g(kk, jj, ii)];
  }
  double rt[NG][NG], rut[NG][NG];
  reconstruct_gll_any<ORD>(s, rt[0], A.weno_s != 0);
  double rser[NG][NG], ruser[NG][NG];
#pragma unroll
  for (int kt = 0; kt < NG; kt++)
#pragma unroll
    for (int ii = 0; ii < NG; ii++) {
      rser[kt][ii] = T.R[(kt * NG + ii) * (long)ncell + c];
      ruser[kt][ii] = T.U[(kt * NG + ii) * (long)ncell + c];
    }
  // the divisors through their correctly rounded reciprocals (IEEE quotients bit for bit):
  // the GLL points' densities (reciprocals recorded by the sweep) and dx
  Rcp<double> rr[NG];
#pragma unroll
  for (int ii = 0; ii < NG; ii++) rr[ii] = rcp_known(rser[0][ii], T.Y[ii * (long)ncell + c]);
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
#pragma unroll
    for (int ii = 0; ii < NG; ii++) {
      double tot = 0;
#pragma unroll
      for (int ir = 0; ir <= kt + 1; ir++) tot += ruser[ir][ii] * rt[kt + 1 - ir][ii] - rser[ir][ii] * rut[kt + 1 - ir][ii];
      rut[kt + 1][ii] = divr_any(tot, rr[ii]);
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
  T.TE[(2L * l) * ncell + c] = tl;
  T.TE[(2L * l + 1) * ncell + c] = trr;
}

// The left (side 0) and right (side 1) values at face f along a line, with the edge BCs:
// periodic faces 0 and n both see (right edge of cell n-1, left edge of cell 0); at a wall
// the outside value copies the inside one (Spatial:816-837).
template <int DIR, int NG>
__global__ void __launch_bounds__(128) tracer_face_kernel(TracerArgs T, int hs) {
  const SweepArgs &A = T.A;
  const Geo<DIR> G(A, hs);
  const long nf = G.nface();
  const long f = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (f >= nf) return;
  const long nlines = DIR == 0 ? (long)G.nz * G.ny : (DIR == 1 ? (long)G.nz * G.nx : (long)G.ny * G.nx);
  if (f < nlines) T.flag[f] = 0;  // the limiter's per-line flags (nf > nlines)
  const int fx = G.nx + (DIR == 0), fy = G.ny + (DIR == 1);
  int i, j, k;
  unflat((unsigned)f, fx, fy, k, j, i);
  const int pf = DIR == 0 ? i : (DIR == 1 ? j : k);
  const int n = G.n();
  const long ncell = (long)G.nz * G.ny * G.nx;
  int pl = pf - 1, pr = pf;  // cells whose right / left edges meet at the face
  bool lside_from_right = false, rside_from_left = false;  // wall copies
  if (pf == 0) {
    if (A.bc == BC_PERIODIC) pl = n - 1;
    else { pl = 0; lside_from_right = true; }
  }
  if (pf == n) {
    if (A.bc == BC_PERIODIC) pr = 0;
    else { pr = n - 1; rside_from_left = true; }
  }
  int kl, jl, il, kr, jr, ir;
  G.at(k, j, i, pl, kl, jl, il);
  G.at(k, j, i, pr, kr, jr, ir);
  const long cl = G.cell(kl, jl, il), cr = G.cell(kr, jr, ir);
  double qL[5], qR[5];
#pragma unroll
  for (int v = 0; v < 5; v++) {
    qL[v] = lside_from_right ? T.E[v * ncell + cl] : T.E[(5 + v) * ncell + cl];
    qR[v] = rside_from_left ? T.E[(5 + v) * ncell + cr] : T.E[v * ncell + cr];
  }
  double F[5];
  riemann<DIR, NG>(qL, qR, k, A, F);  // k: the face's k (z) or the line's k
  constexpr int NM = 1 + DIR;
  const double vn = DIR == 1 ? 0.5 * (qL[NM] + qR[NM]) : 0.5 * (qL[NM] / qL[0] + qR[NM] / qR[0]);
  T.UN[f] = 0.5 * (qL[NM] + qR[NM]);
  for (int l = 0; l < T.ntr; l++) {
    const double tL = lside_from_right ? T.TE[(2L * l) * ncell + cl] : T.TE[(2L * l + 1) * ncell + cl];
    const double tR = rside_from_left ? T.TE[(2L * l + 1) * ncell + cr] : T.TE[(2L * l) * ncell + cr];
    T.TF[l * nf + f] = vn > 0 ? F[0] * tL / qL[0] : F[0] * tR / qR[0];
  }
}

// Positivity limiter (Spatial:904-935, 1262-1293, 1646-1677) in the reference's serial
// loop order: along each line the faces are visited in increasing order and each is scaled
// in place by its upwind cell's factor, computed from that cell's two faces as they stand
// at that moment (the face behind already scaled, the face itself and the ones ahead not
// yet) -- the one defined result of the reference's in-place parallel_for, the one its CPU
// build gives when the loop runs in order. Faces of other lines are never read.
//
// The serial order matters only where a face reads a face that has been scaled: face f > 0
// with un > 0 reads face f-1 (as min(., 0)), and face n with un < 0 reads faces 0 (min) and
// 1 (max). So tracer_limit_faces_kernel limits every face at once with all reads unscaled,
// and flags the lines where some scaled face changed a value another face reads; on the
// other lines that result is the serial one, face by face (by induction along the line:
// every read sees the value the serial loop would). tracer_limit_lines_kernel redoes the
// flagged lines serially. Equal reads are compared as values: a read that differs only in
// the sign of a zero leaves the factor unchanged (it enters as f2 - f1 + eps).

// factor and scaled flux of one face from its upwind cell's two faces (f1 = min(., 0) of
// the left one, f2 = max(., 0) of the right one), the reference's arithmetic order
// (q: the cell's tracer / density)
__device__ __forceinline__ double limit_face(double F, double f1, double f2, double q, double dens,
                                             const SweepArgs &A) {
  const double eps = 1.e-10;
  const double fluxOut = divr_any(A.dt * (f2 - f1), rcp_known(A.dxd, A.rdxd));
  return F * dmin(1., q * dens / (fluxOut + eps));
}

template <int DIR> __device__ __forceinline__ long line_of(int k, int j, int i, int ny, int nx) {
  return DIR == 0 ? (long)k * ny + j : (DIR == 1 ? (long)k * nx + i : (long)j * nx + i);
}

template <int DIR>
__global__ void __launch_bounds__(128) tracer_limit_faces_kernel(TracerArgs T, int hs) {
  const SweepArgs &A = T.A;
  const Geo<DIR> G(A, hs);
  const int nf = (int)G.nface();  // < 2^31 (launch_split_tracers)
  const int fi = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (fi >= nf) return;
  const int fx = G.nx + (DIR == 0), fy = G.ny + (DIR == 1);
  int i, j, k;
  unflat((unsigned)fi, fx, fy, k, j, i);
  const int f = DIR == 0 ? i : (DIR == 1 ? j : k);
  const int n = G.n();
  // strides along the line: faces and cells (flat), state (halo-inclusive)
  const int fs = DIR == 0 ? 1 : (DIR == 1 ? G.nx : G.nx * G.ny);
  const long gsd = DIR == 0 ? 1 : (DIR == 1 ? G.sy : G.sz);
  const int f0 = fi - f * fs;  // the line's face 0
  int k0, j0, i0;
  G.at(k, j, i, 0, k0, j0, i0);
  const int c0 = (int)G.cell(k0, j0, i0);  // the line's cell 0
  const long g0 = G.g(k0, j0, i0);
  const double un = T.UN[fi];
  // the upwind cell and the two faces that bound it
  int c = -1;
  if (un > 0) c = f == 0 ? n - 1 : f - 1;
  else if (un < 0) c = f == n ? 0 : f;
  double dens = 0.;
  if (c >= 0) dens = T.D[c0 + c * fs] + A.dens_c[hs + (DIR == 2 ? c : k)];
  // the faces that read this one: f+1 when it is upwinded from cell f; face n reads
  // faces 0 (min) and 1 (max) when it is upwinded from cell 0 -- through the factor of
  // the reader's upwind cell (f, resp. 0), which is zero whatever it reads when the cell
  // holds no tracer
  const bool read_next = f < n && T.UN[fi + fs] > 0;
  const bool read_by_n = (f == 0 || (f == 1 && n >= 2)) && T.UN[f0 + n * fs] < 0;
  bool chained = false;
  for (int l = 0; l < T.ntr; l++) {
    const double *TF = T.TF + (long)l * nf;
    const double *tr = T.tr + l * G.sv + g0;
    const double F = TF[fi];
    double out = F;
    if (((T.pos >> l) & 1ull) && c >= 0) {
      const double Fa = c == f ? F : TF[f0 + c * fs], Fb = c + 1 == f ? F : TF[f0 + (c + 1) * fs];
      out = limit_face(F, dmin(Fa, 0.), dmax(Fb, 0.), tr[c * gsd], dens, A);
      if (read_next || read_by_n) {
        const bool neg = !(dmin(out, 0.) == dmin(F, 0.)), posv = !(dmax(out, 0.) == dmax(F, 0.));
        if ((read_next && neg && tr[f * gsd] != 0.) || (read_by_n && (f == 0 ? neg : posv) && tr[0] != 0.))
          chained = true;
      }
    }
    T.TF2[(long)l * nf + fi] = out;
  }
  if (chained) T.flag[line_of<DIR>(k, j, i, G.ny, G.nx)] = 1;
}

// The flagged lines in the serial order, one thread per line and tracer: walking the faces
// in order, a face keeps the first pass's value unless a face it reads (min of face f-1 for
// un > 0; min of face 0 and max of face 1 for face n with un < 0) now holds a value other
// than the unscaled one the first pass read; only those faces are limited again. The walk
// reads three words per face and recomputes only along the chains.
template <int DIR>
__global__ void __launch_bounds__(128) tracer_limit_lines_kernel(TracerArgs T, int hs) {
  const SweepArgs &A = T.A;
  const Geo<DIR> G(A, hs);
  const int n = G.n();
  const long nlines = DIR == 0 ? (long)G.nz * G.ny : (DIR == 1 ? (long)G.nz * G.nx : (long)G.ny * G.nx);
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  const long line = t / T.ntr;
  const int l = (int)(t - line * T.ntr);
  if (line >= nlines || !T.flag[line] || !((T.pos >> l) & 1ull)) return;
  int k0, j0, i0;  // the line's cell 0
  const unsigned ln = (unsigned)line;
  if (DIR == 0) { i0 = 0; j0 = (int)(ln % (unsigned)G.ny); k0 = (int)(ln / (unsigned)G.ny); }
  else if (DIR == 1) { j0 = 0; i0 = (int)(ln % (unsigned)G.nx); k0 = (int)(ln / (unsigned)G.nx); }
  else { k0 = 0; i0 = (int)(ln % (unsigned)G.nx); j0 = (int)(ln / (unsigned)G.nx); }
  const long nf = G.nface();
  auto face = [&](int p) {
    int kk, jj, ii;
    G.at(k0, j0, i0, p, kk, jj, ii);
    return G.face(kk, jj, ii);
  };
  const double *TF = T.TF + l * nf;
  double *TF2 = T.TF2 + l * nf;
  double sprev = 0., uprev = 0.;      // the face behind: serial (scaled) and unscaled values
  double s0 = 0., u0 = 0., s1 = 0., u1 = 0.;  // faces 0 and 1, likewise
#pragma unroll 4
  for (int f = 0; f <= n; f++) {
    const long fi = face(f);
    const double F = TF[fi];
    double out = TF2[fi];
    const double un = T.UN[fi];
    int c = -1;
    double f1 = 0., f2 = 0.;
    if (un > 0 && f > 0) {
      if (!(dmin(sprev, 0.) == dmin(uprev, 0.))) {  // upwind cell f-1 reads face f-1
        c = f - 1;
        f1 = dmin(sprev, 0.);
        f2 = dmax(F, 0.);
      }
    } else if (un < 0 && f == n) {
      if (!(dmin(s0, 0.) == dmin(u0, 0.)) || (n >= 2 && !(dmax(s1, 0.) == dmax(u1, 0.)))) {  // upwind cell 0
        c = 0;
        f1 = dmin(s0, 0.);
        f2 = dmax(n == 1 ? F : s1, 0.);
      }
    }
    if (c >= 0) {
      int ck, cj, ci;
      G.at(k0, j0, i0, c, ck, cj, ci);
      out = limit_face(F, f1, f2, T.tr[l * G.sv + G.g(ck, cj, ci)], T.D[G.cell(ck, cj, ci)] + A.dens_c[hs + ck], A);
      TF2[fi] = out;
    }
    sprev = out;
    uprev = F;
    if (f == 0) { s0 = out; u0 = F; }
    if (f == 1) { s1 = out; u1 = F; }
  }
}

template <int DIR>
__global__ void __launch_bounds__(128) tracer_update_kernel(TracerArgs T, int hs) {
  const SweepArgs &A = T.A;
  const Geo<DIR> G(A, hs);
  const long ncell = (long)G.nz * G.ny * G.nx;
  const long c = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (c >= ncell) return;
  int i, j, k;
  unflat((unsigned)c, G.nx, G.ny, k, j, i);
  const int p = DIR == 0 ? i : (DIR == 1 ? j : k);
  const int n = G.n();
  const long nf = G.nface();
  int rk, rj, ri;
  G.at(k, j, i, p + 1, rk, rj, ri);
  const long fl = G.face(k, j, i), fr = G.face(rk, rj, ri);
  const long gg = G.g(k, j, i);
  const double dens = T.D[c] + A.dens_c[hs + k];
  // halo cell of index h along DIR (state offset)
  auto halo = [&](int h) -> long {
    int kk, jj, ii;
    G.at(k, j, i, h, kk, jj, ii);
    return G.g(kk, jj, ii);
  };
  for (int l = 0; l < T.ntr; l++) {
    double *t = T.tr + l * G.sv;
    const double q = t[gg];  // tracer / density (tracer_divide_kernel)
    const double tend = -(T.TF2[l * nf + fr] - T.TF2[l * nf + fl]) / A.dxd;
    t[gg] = q * dens + A.dt * tend;  // Spatial:952-953, then Temporal_ader.h:67-69
    if (A.bc == BC_PERIODIC) {
      if (p >= n - hs) t[halo(p - n)] = q;   // low halo (index p - n in [-hs, 0))
      if (p < hs) t[halo(n + p)] = q;        // high halo
    } else {
      if (p == 0)
        for (int h = 1; h <= hs; h++) t[halo(-h)] = q;
      if (p == n - 1)
        for (int h = 0; h < hs; h++) t[halo(n + h)] = q;
    }
  }
}

template <int ORD, int DIR>
cudaError_t run(const TracerArgs &T, cudaStream_t st) {
  constexpr int HS = (ORD - 1) / 2;
  constexpr int NG = OrdTraits<ORD>::NGLL;
  const SweepArgs &A = T.A;
  const long ncell = (long)A.nz * A.ny * A.nx;
  const long nf = (long)(A.nz + (DIR == 2)) * (A.ny + (DIR == 1)) * (A.nx + (DIR == 0));
  const unsigned gc = (unsigned)((ncell + 127) / 128), gf = (unsigned)((nf + 127) / 128);
  tracer_divide_kernel<<<gc, 128, 0, st>>>(T, HS);
  cudaError_t e = launch_sweep_t<P64Trc, ORD, DIR>(A, st);  // state split + records
  if (e != cudaSuccess) return e;
  tracer_cell_kernel<ORD, DIR><<<gc * (unsigned)T.ntr, 128, 0, st>>>(T);
  tracer_face_kernel<DIR, NG><<<gf, 128, 0, st>>>(T, HS);
  const long nlines = DIR == 0 ? (long)A.nz * A.ny : (DIR == 1 ? (long)A.nz * A.nx : (long)A.ny * A.nx);
  tracer_limit_faces_kernel<DIR><<<gf, 128, 0, st>>>(T, HS);
  tracer_limit_lines_kernel<DIR><<<(unsigned)((nlines * T.ntr + 127) / 128), 128, 0, st>>>(T, HS);
  tracer_update_kernel<DIR><<<gc, 128, 0, st>>>(T, HS);
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_split_tracers(int ord, int dir, const SweepArgs &Ain, double *tracers, int ntr,
                                 unsigned long long pos, double *scratch, cudaStream_t st) {
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
  T.R = scratch;
  T.U = scratch + (long)ng * ng * ncell;
  T.E = scratch + 2L * ng * ng * ncell;
  T.D = T.E + 10 * ncell;
  T.Y = T.E + 11 * ncell;
  T.TE = T.E + (11L + ng) * ncell;
  T.TF = T.TE + 2L * ntr * ncell;
  T.TF2 = T.TF + (long)ntr * nfmax;
  T.UN = T.TF2 + (long)ntr * nfmax;
  T.flag = reinterpret_cast<int *>(T.UN + nfmax);
  if (ord == 5) {
    if (dir == 0) return run<5, 0>(T, st);
    if (dir == 1) return run<5, 1>(T, st);
    return run<5, 2>(T, st);
  }
  if (dir == 0) return run<9, 0>(T, st);
  if (dir == 1) return run<9, 1>(T, st);
  return run<9, 2>(T, st);
}

long tracer_scratch_doubles(int ord, int nx, int ny, int nz, int ntr) {
  const int ng = ord == 5 ? 3 : 5;
  const long ncell = (long)nz * ny * nx;
  const long nfmax = (long)(nz + 1) * (ny + 1) * (nx + 1);
  long lines = (long)nz * ny;  // the most lines of one direction: the limiter's int flags
  if ((long)nz * nx > lines) lines = (long)nz * nx;
  if ((long)ny * nx > lines) lines = (long)ny * nx;
  return (2L * ng * ng + 11 + ng) * ncell + 2L * ntr * ncell + 2L * ntr * nfmax + nfmax + lines / 2 + 1;
}

cudaError_t upload_tables_tracers(int ord, const void *tab, size_t bytes) {
  if (ord == 5) return cudaMemcpyToSymbol(c_tab5, tab, bytes);
  return cudaMemcpyToSymbol(c_tab9, tab, bytes);
}

}  // namespace awfl
