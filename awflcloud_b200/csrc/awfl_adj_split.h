// Reverse (adjoint) of one directional split, as per-thread functions (host + device).
//
// Forward split in direction DIR, on every line of length L along DIR (Temporal_ader.h:
// 63-65 with the tendencies of Spatial_euler3d_cons_expl_cart_fv_Agrid.h:598-957,
// 961-1311, 1315-1697):
//   stencils from the line with its halo (periodic wrap, or a wall copy of the edge cell
//   with zero normal momentum) -> per cell edge states eL, eR (+ z source)
//   -> per face the upwind flux F(qL, qR), where qL/qR are the neighbouring edges; at a
//   periodic end the far edge, at a wall the near edge on both sides
//   -> state += dt * (-(F_right - F_left) / dx (+ source on rho*w for z)).
// Its adjoint maps lam (adjoint of the state after the split) to the adjoint before it:
//   edges    recompute the level-0 GLL values q0 and the edges eL, eR of every cell
//            (the linearisation point)
//   face     lF = dt/dx (lam_right_cell - lam_left_cell) -> (lqL, lqR) per face
//   cell_dt  (lqR of the left face, lqL of the right face, dt*lam_w) -> ADER reverse from
//            q0 -> lq0, the adjoint of the level-0 values
//   weno     per (cell, variable): lq0 -> reconstruction reverse -> adjoint of the ORD
//            stencil values
//   gather   lam += sum of the stencil adjoints that read this cell (through the halo
//            mapping), so no two threads write the same word and the result is
//            independent of the launch order
// Each function handles one index of its own grid: cells (nz*ny*nx), faces along DIR, or
// (variable, cell) pairs. Splitting the cell reverse in two keeps the register footprint
// of each kernel small.
#pragma once

#include "awfl_adj.h"

namespace awfl {
namespace adj {

struct SplitArgs {
  const double *state;  // split-start state, (5, nz+2hs, ny+2hs, nx+2hs); halos not read
  double *edges;        // 10 planes of ncell: eL[v], eR[v]
  double *lam;          // adjoint, state layout: in = after the split, out = before it
  double *lq;           // 10 planes of nface: lqL[v], lqR[v]
  double *ls;           // 5*ORD planes of ncell: adjoint of stencil slot m of variable v
  double *q0;           // 5*NGLL planes of ncell: level-0 values (after hydrostasis)
  double *lq0;          // 5*NGLL planes of ncell: their adjoint
  int nx, ny, nz, hs;
  int sim2d;
  CellArgs ca;          // bc (along DIR), weno switches, dxd, dt, background
};

AWFL_AHD long ncell_of(const SplitArgs &A) { return (long)A.nz * A.ny * A.nx; }

template <int DIR> AWFL_AHD long nface_of(const SplitArgs &A) {
  return DIR == 0 ? (long)A.nz * A.ny * (A.nx + 1)
                  : (DIR == 1 ? (long)A.nz * (A.ny + 1) * A.nx : (long)(A.nz + 1) * A.ny * A.nx);
}
template <int DIR> AWFL_AHD int line_len(const SplitArgs &A) { return DIR == 0 ? A.nx : (DIR == 1 ? A.ny : A.nz); }

AWFL_AHD long sidx(const SplitArgs &A, int v, int i, int j, int k) {
  const int h = A.hs;
  return (((long)v * (A.nz + 2 * h) + k + h) * (A.ny + 2 * h) + j + h) * (A.nx + 2 * h) + i + h;
}
AWFL_AHD long cidx(const SplitArgs &A, int i, int j, int k) { return ((long)k * A.ny + j) * A.nx + i; }

// interior coordinates with the DIR coordinate replaced by p
template <int DIR> AWFL_AHD void at(int i, int j, int k, int p, int &ii, int &jj, int &kk) {
  ii = DIR == 0 ? p : i;
  jj = DIR == 1 ? p : j;
  kk = DIR == 2 ? p : k;
}
template <int DIR> AWFL_AHD long fidx(const SplitArgs &A, int i, int j, int k, int f) {
  if (DIR == 0) return ((long)k * A.ny + j) * (A.nx + 1) + f;
  if (DIR == 1) return ((long)k * (A.ny + 1) + f) * A.nx + i;
  return ((long)f * A.ny + j) * A.nx + i;
}
AWFL_AHD void decode_cell(const SplitArgs &A, long c, int &i, int &j, int &k) {
  i = (int)(c % A.nx);
  const long r = c / A.nx;
  j = (int)(r % A.ny);
  k = (int)(r / A.ny);
}

// ---- edges of one cell (forward recomputation of the linearisation point)
template <int ORD, int DIR> AWFL_AHD void split_edges(const Tables<ORD> &T, const SplitArgs &A, long c) {
  constexpr int HS = (ORD - 1) / 2;
  constexpr int NM = 1 + DIR;
  int i, j, k;
  decode_cell(A, c, i, j, k);
  const int L = line_len<DIR>(A);
  const int p = DIR == 0 ? i : (DIR == 1 ? j : k);
  double sten[5][ORD];
  AWFL_UNROLL for (int m = 0; m < ORD; m++) {
    int q = p - HS + m;
    bool zero_n = false;
    if (q < 0 || q >= L) {
      if (A.ca.bc == BC_PERIODIC) {
        q %= L;
        if (q < 0) q += L;
      } else {
        q = q < 0 ? 0 : L - 1;
        zero_n = true;
      }
    }
    int ii, jj, kk;
    at<DIR>(i, j, k, q, ii, jj, kk);
    AWFL_UNROLL for (int v = 0; v < 5; v++) sten[v][m] = (zero_n && v == NM) ? 0. : A.state[sidx(A, v, ii, jj, kk)];
  }
  CellFwd<ORD, DIR> X;
  cell_fwd<ORD, DIR>(T, sten, k, A.ca, X);
  double eL[5], eR[5], src;
  cell_edges<ORD, DIR>(T, X, A.ca.dt, eL, eR, src);
  const long n = ncell_of(A);
  AWFL_UNROLL for (int v = 0; v < 5; v++) {
    A.edges[v * n + c] = eL[v];
    A.edges[(5 + v) * n + c] = eR[v];
  }
  constexpr int NG = OrdTraits<ORD>::NGLL;
  AWFL_UNROLL for (int v = 0; v < 5; v++)
    AWFL_UNROLL for (int ii = 0; ii < NG; ii++) A.q0[(v * NG + ii) * n + c] = X.q[v][0][ii];
}

// ---- one face: flux adjoint from the two neighbouring cells' lam, then Riemann reverse
template <int DIR> AWFL_AHD void split_face(const SplitArgs &A, long idx) {
  const int L = line_len<DIR>(A);
  int i = 0, j = 0, k = 0, f;
  if (DIR == 0) {
    f = (int)(idx % (A.nx + 1));
    const long r = idx / (A.nx + 1);
    j = (int)(r % A.ny);
    k = (int)(r / A.ny);
  } else if (DIR == 1) {
    i = (int)(idx % A.nx);
    const long r = idx / A.nx;
    f = (int)(r % (A.ny + 1));
    k = (int)(r / (A.ny + 1));
  } else {
    i = (int)(idx % A.nx);
    const long r = idx / A.nx;
    j = (int)(r % A.ny);
    f = (int)(r / A.ny);
  }
  const bool periodic = A.ca.bc == BC_PERIODIC;
  const long n = ncell_of(A);
  int ii, jj, kk;
  // left state: right edge of cell f-1
  at<DIR>(i, j, k, f > 0 ? f - 1 : (periodic ? L - 1 : 0), ii, jj, kk);
  const long cl = cidx(A, ii, jj, kk);
  const int plane_l = (f > 0 || periodic) ? 5 : 0;
  // right state: left edge of cell f
  at<DIR>(i, j, k, f < L ? f : (periodic ? 0 : L - 1), ii, jj, kk);
  const long cr = cidx(A, ii, jj, kk);
  const int plane_r = (f < L || periodic) ? 0 : 5;
  double qL[5], qR[5], lF[5];
  AWFL_UNROLL for (int v = 0; v < 5; v++) {
    qL[v] = A.edges[(plane_l + v) * n + cl];
    qR[v] = A.edges[(plane_r + v) * n + cr];
  }
  const double s = A.ca.dt / A.ca.dxd;
  int ai, aj, ak, bi, bj, bk;
  at<DIR>(i, j, k, f, ai, aj, ak);
  at<DIR>(i, j, k, f - 1, bi, bj, bk);
  AWFL_UNROLL for (int v = 0; v < 5; v++) {
    double l = 0.;
    if (!(A.sim2d && v == idV && DIR != 1)) {
      if (f < L) l += A.lam[sidx(A, v, ai, aj, ak)];
      if (f > 0) l -= A.lam[sidx(A, v, bi, bj, bk)];
    }
    lF[v] = s * l;
  }
  double lqL[5], lqR[5];
  riemann_vjp<DIR>(qL, qR, lF, lqL, lqR);
  const long nf = nface_of<DIR>(A);
  AWFL_UNROLL for (int v = 0; v < 5; v++) {
    A.lq[v * nf + idx] = lqL[v];
    A.lq[(5 + v) * nf + idx] = lqR[v];
  }
}

// ---- one cell: edge adjoints from its faces, then the ADER reverse from q0
template <int ORD, int DIR> AWFL_AHD void split_cell_dt(const Tables<ORD> &T, const SplitArgs &A, long c) {
  constexpr int NG = OrdTraits<ORD>::NGLL;
  int i, j, k;
  decode_cell(A, c, i, j, k);
  const int L = line_len<DIR>(A);
  const int p = DIR == 0 ? i : (DIR == 1 ? j : k);
  const bool periodic = A.ca.bc == BC_PERIODIC;
  const long nf = nface_of<DIR>(A);
  const long fl = fidx<DIR>(A, i, j, k, p), fr = fidx<DIR>(A, i, j, k, p + 1);
  double leL[5], leR[5];
  AWFL_UNROLL for (int v = 0; v < 5; v++) {
    leL[v] = A.lq[(5 + v) * nf + fl];  // right state of the left face
    leR[v] = A.lq[v * nf + fr];        // left state of the right face
  }
  if (p == 0) {  // face 0: periodic -> its twin face L reads eL_0 as its right state
    const long f0 = fidx<DIR>(A, i, j, k, 0), fL = fidx<DIR>(A, i, j, k, L);
    AWFL_UNROLL for (int v = 0; v < 5; v++) leL[v] += periodic ? A.lq[(5 + v) * nf + fL] : A.lq[v * nf + f0];
  }
  if (p == L - 1) {  // face L: periodic -> face 0 reads eR_{L-1} as its left state
    const long f0 = fidx<DIR>(A, i, j, k, 0), fL = fidx<DIR>(A, i, j, k, L);
    AWFL_UNROLL for (int v = 0; v < 5; v++) leR[v] += periodic ? A.lq[v * nf + f0] : A.lq[(5 + v) * nf + fL];
  }
  const double lsrc = DIR == 2 ? A.ca.dt * A.lam[sidx(A, idW, i, j, k)] : 0.;
  const long n = ncell_of(A);
  CellFwd<ORD, DIR> X;
  AWFL_UNROLL for (int v = 0; v < 5; v++)
    AWFL_UNROLL for (int ii = 0; ii < NG; ii++) X.q[v][0][ii] = A.q0[(v * NG + ii) * n + c];
  cell_dt<ORD, DIR>(T, k, A.ca, X);
  double lq0[5][NG];
  cell_dt_vjp<ORD, DIR>(T, k, A.ca, X, leL, leR, lsrc, lq0);
  AWFL_UNROLL for (int v = 0; v < 5; v++)
    AWFL_UNROLL for (int ii = 0; ii < NG; ii++) A.lq0[(v * NG + ii) * n + c] = lq0[v][ii];
}

// ---- one (variable, cell): the reconstruction reverse of that variable's stencil
template <int ORD, int DIR> AWFL_AHD void split_weno(const Tables<ORD> &T, const SplitArgs &A, long idx) {
  constexpr int HS = (ORD - 1) / 2;
  constexpr int NG = OrdTraits<ORD>::NGLL;
  constexpr int NM = 1 + DIR;
  const long n = ncell_of(A);
  const int v = (int)(idx / n);
  const long c = idx - v * n;
  int i, j, k;
  decode_cell(A, c, i, j, k);
  const int L = line_len<DIR>(A);
  const int p = DIR == 0 ? i : (DIR == 1 ? j : k);
  double sten[ORD];
  AWFL_UNROLL for (int m = 0; m < ORD; m++) {
    int q = p - HS + m;
    bool zero_n = false;
    if (q < 0 || q >= L) {
      if (A.ca.bc == BC_PERIODIC) {
        q %= L;
        if (q < 0) q += L;
      } else {
        q = q < 0 ? 0 : L - 1;
        zero_n = true;
      }
    }
    int ii, jj, kk;
    at<DIR>(i, j, k, q, ii, jj, kk);
    sten[m] = (zero_n && v == NM) ? 0. : A.state[sidx(A, v, ii, jj, kk)];
  }
  double lq0[NG], ls[ORD];
  AWFL_UNROLL for (int ii = 0; ii < NG; ii++) lq0[ii] = A.lq0[(v * NG + ii) * n + c];
  AWFL_UNROLL for (int m = 0; m < ORD; m++) ls[m] = 0.;
  const bool doweno = (v == idR || v == idT) ? A.ca.weno_s : A.ca.weno_w;
  gll_vjp<ORD>(T, sten, doweno, lq0, ls);
  AWFL_UNROLL for (int m = 0; m < ORD; m++) A.ls[(v * ORD + m) * n + c] = ls[m];
}

// ---- one cell: lam += every stencil adjoint that read this cell
template <int ORD, int DIR> AWFL_AHD void split_gather(const SplitArgs &A, long c) {
  constexpr int HS = (ORD - 1) / 2;
  constexpr int NM = 1 + DIR;
  int i, j, k;
  decode_cell(A, c, i, j, k);
  const int L = line_len<DIR>(A);
  const int p = DIR == 0 ? i : (DIR == 1 ? j : k);
  const bool periodic = A.ca.bc == BC_PERIODIC;
  const long n = ncell_of(A);
  AWFL_UNROLL for (int v = 0; v < 5; v++) {
    const long g = sidx(A, v, i, j, k);
    double acc = A.lam[g];
    AWFL_UNROLL for (int m = 0; m < ORD; m++) {
      int src = p + HS - m;  // the cell whose slot m is this position
      if (src < 0 || src >= L) {
        if (!periodic) continue;
        src %= L;
        if (src < 0) src += L;
      }
      int ii, jj, kk;
      at<DIR>(i, j, k, src, ii, jj, kk);
      acc += A.ls[(v * ORD + m) * n + cidx(A, ii, jj, kk)];
    }
    if (!periodic && v != NM) {
      if (p == 0) {  // halo slots below the line copy cell 0
        for (int s = 0; s < HS && s < L; s++)
          for (int m = 0; m < HS - s; m++) {
            int ii, jj, kk;
            at<DIR>(i, j, k, s, ii, jj, kk);
            acc += A.ls[(v * ORD + m) * n + cidx(A, ii, jj, kk)];
          }
      }
      if (p == L - 1) {  // halo slots above the line copy cell L-1
        for (int s = (L - HS > 0 ? L - HS : 0); s < L; s++)
          for (int m = L + HS - s; m < ORD; m++) {
            int ii, jj, kk;
            at<DIR>(i, j, k, s, ii, jj, kk);
            acc += A.ls[(v * ORD + m) * n + cidx(A, ii, jj, kk)];
          }
      }
    }
    A.lam[g] = acc;
  }
}

}  // namespace adj
}  // namespace awfl
