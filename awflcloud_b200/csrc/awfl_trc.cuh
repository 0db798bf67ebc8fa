// Tracer transport kernels shared by the FP64 path (awfl_tracers.cu) and the FP32 form
// (awfl_tracers32.cu): the along-line geometry of a split, the in-place division of the
// tracers by the pre-split density (Spatial:624-627), the positivity limiter with the
// result of the reference's serial face order (Spatial:904-935, 1262-1293, 1646-1677) and
// the tendency and update (Spatial:948-955; Temporal_ader.h:67-69).
//
// The including translation unit defines, before including this header, its tracer
// argument struct TA with
//   A                the split's sweep arguments (nx, ny, nz, bc),
//   using Flux       the flux type (double: FP64 path; float: FP32 form),
//   tr               double*, (ntr, nz+2hs, ny+2hs, nx+2hs): the tracers,
//   ntr, pos         the tracer count and the positive-definite bits,
//   D                const Flux*, (ncell): the recorded pre-split rho',
//   F0, VN, UN       const Flux*, (nface) each: per face, recorded by the state's sweep, the
//                    Riemann mass flux, the velocity that picks the upwind side and the
//                    limiter's velocity,
//   TF, TF2          Flux*, (ntr, nface): the unscaled and the limited tracer fluxes,
//   flag, list, count  int*: per line, whether the limiter redoes it in serial order; the
//                    list of those lines and its length (zeroed with the flags before
//                    the limiter runs),
// and these overloads for it:
//   trc_divisor(T, hs, k, g)        the divisor of the division: rho' + rho_h (double)
//   trc_dens(T, hs, k)              rho_h of row k as the limiter adds it to a recorded rho'
//   limit_face(T, F, f1, f2, q, d)  a face's scaled flux from its upwind cell's two faces
//   trc_div_up(T, a, fi)            a divided by the upwind density of face fi (recorded)
//   trc_update(T, q, hs, k, c, Fl, Fr)
//                                   the updated tracer of cell c (row k) from its divided
//                                   value q and its limited face fluxes: q*rho + dt*tend
// Everything here sits in an anonymous namespace: each translation unit compiles its own
// copy with its own floating-point flags.
#pragma once

#include <cuda_runtime.h>

#include "awfl_internal.h"

namespace awfl {
namespace {

template <class R> __device__ __forceinline__ R dmax(R a, R b) { return a > b ? a : b; }
template <class R> __device__ __forceinline__ R dmin(R a, R b) { return a < b ? a : b; }

// Along-direction geometry of one split: cells (k, j, i); p = the index along DIR.
template <int DIR> struct Geo {
  int nx, ny, nz, hs;
  long sy, sz, sv;  // state strides (halo-inclusive)
  template <class SA> __device__ Geo(const SA &A, int hs_) : nx(A.nx), ny(A.ny), nz(A.nz), hs(hs_) {
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
  __device__ long nlines() const {
    return DIR == 0 ? (long)nz * ny : (DIR == 1 ? (long)nz * nx : (long)ny * nx);
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
// tracer path's grids hold fewer than 2^31 cells and faces (the launchers check)
__device__ __forceinline__ void unflat(unsigned x, unsigned ex, unsigned ey, int &k, int &j, int &i) {
  const unsigned r = x / ex;
  const unsigned kk = r / ey;
  i = (int)(x - r * ex);
  j = (int)(r - kk * ey);
  k = (int)kk;
}

template <int DIR> __device__ __forceinline__ long line_of(int k, int j, int i, int ny, int nx) {
  return DIR == 0 ? (long)k * ny + j : (DIR == 1 ? (long)k * nx + i : (long)j * nx + i);
}

// The tracer fluxes (Spatial:891-901, 1249-1259, 1633-1643) of the faces cell p of a line
// is upwind of, from its time-averaged tracer edges tl (left) and tr (right): face flux =
// the state's mass flux F0 times the upwind edge over the upwind density RUP, both recorded
// by the sweep at the face; VN > 0 makes the left cell upwind. Edge BCs (Spatial:816-837):
// periodic faces 0 and n both see (right edge of cell n-1, left edge of cell 0); at a wall
// both sides of face 0 see cell 0's left edge, of face n cell n-1's right edge. Every face
// of the line is written by exactly one cell (face 0 and face n of a periodic line by one
// cell each). fl: this cell's left face, fs: the face stride along the line, f0: face 0.
// Which faces those are, decided once per cell for all its tracers: the left face (fed by
// tl), the right face (tr), and on a periodic line face 0 (tr of cell n-1) and face n
// (tl of cell 0).
struct UpwindFaces {
  long fl, fr, f0, fn;
  bool pl, pr, p0, pn;
};
template <class TA>
__device__ __forceinline__ UpwindFaces upwind_faces(const TA &T, int p, int n, bool periodic, long fl, long fs,
                                                    long f0) {
  UpwindFaces U;
  U.fl = fl;
  U.fr = fl + fs;
  U.f0 = f0;
  U.fn = f0 + (long)n * fs;
  U.pl = (p == 0 && !periodic) || !(T.VN[fl] > 0);
  U.pr = (p == n - 1 && !periodic) || T.VN[U.fr] > 0;
  U.p0 = periodic && p == n - 1 && T.VN[f0] > 0;      // face 0, across the wrap
  U.pn = periodic && p == 0 && !(T.VN[U.fn] > 0);     // face n, likewise
  return U;
}
template <class Fx, class TA>
__device__ __forceinline__ void put_upwind_fluxes(const TA &T, Fx *TF, const UpwindFaces &U, Fx tl, Fx tr) {
  auto put = [&](long fi, Fx t) { TF[fi] = trc_div_up(T, T.F0[fi] * t, fi); };
  if (U.pl) put(U.fl, tl);
  if (U.pr) put(U.fr, tr);
  if (U.p0) put(U.f0, tr);
  if (U.pn) put(U.fn, tl);
}
template <class Fx, class TA>
__device__ __forceinline__ void write_upwind_fluxes(const TA &T, Fx *TF, int p, int n, bool periodic, long fl,
                                                    long fs, long f0, Fx tl, Fx tr) {
  put_upwind_fluxes<Fx>(T, TF, upwind_faces(T, p, n, periodic, fl, fs, f0), tl, tr);
}

// tracers /= (rho' + rho_h) on the interior cells, with the state before the split
// (Spatial:624-627). The halos are not touched: every kernel of the split maps a halo
// position to the interior cell whose value it holds.
#ifndef AWFL_TRC_DIVIDE_MINB
#define AWFL_TRC_DIVIDE_MINB 1
#endif
template <class TA>
__global__ void __launch_bounds__(128, AWFL_TRC_DIVIDE_MINB) tracer_divide_kernel(TA T, int hs) {
  const Geo<0> G(T.A, hs);
  const long ncell = (long)G.nz * G.ny * G.nx;
  const long c = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (c >= ncell) return;
  int i, j, k;
  unflat((unsigned)c, G.nx, G.ny, k, j, i);
  const long g = G.g(k, j, i);
  const double dens = trc_divisor(T, hs, k, idR * G.sv + g);
  for (int l = 0; l < T.ntr; l++) T.tr[l * G.sv + g] /= dens;
}

// Positivity limiter in the reference's serial loop order: along each line the faces are
// visited in increasing order and each is scaled in place by its upwind cell's factor,
// computed from that cell's two faces as they stand at that moment (the face behind
// already scaled, the face itself and the ones ahead not yet) -- the one defined result of
// the reference's in-place parallel_for, the one its CPU build gives when the loop runs in
// order. Faces of other lines are never read.
//
// The serial order matters only where a face reads a face that has been scaled: face f > 0
// with un > 0 reads face f-1 (as min(., 0)), and face n with un < 0 reads faces 0 (min) and
// 1 (max). So tracer_limit_faces_kernel limits every face at once with all reads unscaled,
// and flags the lines where some scaled face changed a value another face reads; on the
// other lines that result is the serial one, face by face (by induction along the line:
// every read sees the value the serial loop would). tracer_limit_lines_kernel redoes the
// flagged lines serially. Equal reads are compared as values: a read that differs only in
// the sign of a zero leaves the factor unchanged (it enters as f2 - f1 + eps).
#ifndef AWFL_TRC_LIMIT_MINB
#define AWFL_TRC_LIMIT_MINB 1
#endif
template <class TA, int DIR>
__global__ void __launch_bounds__(128, AWFL_TRC_LIMIT_MINB) tracer_limit_faces_kernel(TA T, int hs) {
  using Fx = typename TA::Flux;
  const Geo<DIR> G(T.A, hs);
  const int nf = (int)G.nface();  // < 2^31 (the launchers check)
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
  const Fx un = T.UN[fi];
  // the upwind cell and the two faces that bound it
  int c = -1;
  if (un > 0) c = f == 0 ? n - 1 : f - 1;
  else if (un < 0) c = f == n ? 0 : f;
  Fx dens = 0;
  if (c >= 0) dens = T.D[c0 + c * fs] + trc_dens(T, hs, DIR == 2 ? c : k);
  // the faces that read this one: f+1 when it is upwinded from cell f; face n reads
  // faces 0 (min) and 1 (max) when it is upwinded from cell 0 -- through the factor of
  // the reader's upwind cell (f, resp. 0), which is zero whatever it reads when the cell
  // holds no tracer
  const bool read_next = f < n && T.UN[fi + fs] > 0;
  const bool read_by_n = (f == 0 || (f == 1 && n >= 2)) && T.UN[f0 + n * fs] < 0;
  bool chained = false;
  for (int l = 0; l < T.ntr; l++) {
    const Fx *TF = T.TF + (long)l * nf;
    const double *tr = T.tr + l * G.sv + g0;
    const Fx F = TF[fi];
    Fx out = F;
    if (((T.pos >> l) & 1ull) && c >= 0) {
      const Fx Fa = c == f ? F : TF[f0 + c * fs], Fb = c + 1 == f ? F : TF[f0 + (c + 1) * fs];
      out = limit_face(T, F, dmin(Fa, Fx(0)), dmax(Fb, Fx(0)), tr[c * gsd], dens);
      if (read_next || read_by_n) {
        const bool neg = !(dmin(out, Fx(0)) == dmin(F, Fx(0))), posv = !(dmax(out, Fx(0)) == dmax(F, Fx(0)));
        if ((read_next && neg && tr[f * gsd] != 0.) || (read_by_n && (f == 0 ? neg : posv) && tr[0] != 0.))
          chained = true;
      }
    }
    T.TF2[(long)l * nf + fi] = out;
  }
  if (chained) {
    const long line = line_of<DIR>(k, j, i, G.ny, G.nx);
    if (atomicExch(&T.flag[line], 1) == 0) T.list[atomicAdd(T.count, 1)] = (int)line;
  }
}

// The flagged lines in the serial order, one warp per line and tracer: walking the faces
// in order, a face keeps the first pass's value unless a face it reads (min of face f-1 for
// un > 0; min of face 0 and max of face 1 for face n with un < 0) now holds a value other
// than the unscaled one the first pass read; only those faces are limited again. The warp
// loads 32 faces at a time (one per lane) and runs the walk over them uniformly, the
// values coming by shuffle: the loads of a chunk overlap instead of one chain of
// dependent loads per face.
template <class TA, int DIR>
__global__ void __launch_bounds__(128) tracer_limit_lines_kernel(TA T, int hs) {
  using Fx = typename TA::Flux;
  const Geo<DIR> G(T.A, hs);
  const int n = G.n();
  const int lane = threadIdx.x & 31;
  const long nwarps = (long)gridDim.x * (blockDim.x / 32);
  const long items = (long)(*T.count) * T.ntr;
  const long nf = G.nface();
  for (long item = (blockIdx.x * (long)blockDim.x + threadIdx.x) / 32; item < items; item += nwarps) {
    const int l = (int)(item % T.ntr);
    if (!((T.pos >> l) & 1ull)) continue;  // unlimited: the first pass copied the fluxes
    const unsigned ln = (unsigned)T.list[item / T.ntr];
    int k0, j0, i0;  // the line's cell 0
    if (DIR == 0) { i0 = 0; j0 = (int)(ln % (unsigned)G.ny); k0 = (int)(ln / (unsigned)G.ny); }
    else if (DIR == 1) { j0 = 0; i0 = (int)(ln % (unsigned)G.nx); k0 = (int)(ln / (unsigned)G.nx); }
    else { k0 = 0; i0 = (int)(ln % (unsigned)G.nx); j0 = (int)(ln / (unsigned)G.nx); }
    auto face = [&](int p) {
      int kk, jj, ii;
      G.at(k0, j0, i0, p, kk, jj, ii);
      return G.face(kk, jj, ii);
    };
    const Fx *TF = T.TF + l * nf;
    Fx *TF2 = T.TF2 + l * nf;
    Fx sprev = 0, uprev = 0;              // the face behind: serial (scaled) and unscaled values
    Fx s0 = 0, u0 = 0, s1 = 0, u1 = 0;   // faces 0 and 1, likewise
    for (int base = 0; base <= n; base += 32) {
      const int fme = base + lane;
      long fim = 0;
      Fx Fm = 0, Tm = 0, Um = 0;
      if (fme <= n) {
        fim = face(fme);
        Fm = TF[fim];
        Tm = TF2[fim];
        Um = T.UN[fim];
      }
      const int cnt = n + 1 - base < 32 ? n + 1 - base : 32;
      for (int i = 0; i < cnt; i++) {
        const int f = base + i;
        const Fx F = __shfl_sync(0xffffffffu, Fm, i);
        Fx out = __shfl_sync(0xffffffffu, Tm, i);
        const Fx un = __shfl_sync(0xffffffffu, Um, i);
        int c = -1;
        Fx f1 = 0, f2 = 0;
        if (un > 0 && f > 0) {
          if (!(dmin(sprev, Fx(0)) == dmin(uprev, Fx(0)))) {  // upwind cell f-1 reads face f-1
            c = f - 1;
            f1 = dmin(sprev, Fx(0));
            f2 = dmax(F, Fx(0));
          }
        } else if (un < 0 && f == n) {
          if (!(dmin(s0, Fx(0)) == dmin(u0, Fx(0))) || (n >= 2 && !(dmax(s1, Fx(0)) == dmax(u1, Fx(0))))) {
            c = 0;  // upwind cell 0
            f1 = dmin(s0, Fx(0));
            f2 = dmax(n == 1 ? F : s1, Fx(0));
          }
        }
        if (c >= 0) {
          int ck, cj, ci;
          G.at(k0, j0, i0, c, ck, cj, ci);
          out = limit_face(T, F, f1, f2, T.tr[l * G.sv + G.g(ck, cj, ci)], T.D[G.cell(ck, cj, ci)] + trc_dens(T, hs, ck));
          if (lane == i) TF2[fim] = out;
        }
        sprev = out;
        uprev = F;
        if (f == 0) { s0 = out; u0 = F; }
        if (f == 1) { s1 = out; u1 = F; }
      }
    }
  }
}

// Per cell: the tendency of the limited fluxes, density multiplied back and the update
// (Spatial:948-955; Temporal_ader.h:67-69), and the halo cells of this direction left
// holding tracer/density, as the reference's in-place halo fill leaves them. out_divided:
// the interior is left divided by the post-split density (the state's split is done), as
// the next split's tracer_divide_kernel would divide it.
#ifndef AWFL_TRC_UPDATE_MINB
#define AWFL_TRC_UPDATE_MINB 1
#endif
template <class TA, int DIR>
__global__ void __launch_bounds__(128, AWFL_TRC_UPDATE_MINB) tracer_update_kernel(TA T, int hs, bool out_divided) {
  const Geo<DIR> G(T.A, hs);
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
  // halo cell of index h along DIR (state offset)
  auto halo = [&](int h) -> long {
    int kk, jj, ii;
    G.at(k, j, i, h, kk, jj, ii);
    return G.g(kk, jj, ii);
  };
  for (int l = 0; l < T.ntr; l++) {
    double *t = T.tr + l * G.sv;
    const double q = t[gg];  // tracer / density (tracer_divide_kernel)
    const double tn = trc_update(T, q, hs, k, c, T.TF2[l * nf + fl], T.TF2[l * nf + fr]);
    t[gg] = out_divided ? tn / trc_divisor(T, hs, k, idR * G.sv + gg) : tn;
    if (T.A.bc == BC_PERIODIC) {
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

}  // namespace
}  // namespace awfl
