// Host driver of the per-thread adjoint functions (awfl_adj_split.h): runs the edges,
// face, cell_dt, weno and gather passes of one split as plain loops, so that tests can check the
// split adjoint, halo mapping included, against finite differences of the oracle's split
// without a GPU, and its forward recomputation against the oracle's tendencies. Built as a
// shared library by tests/test_adjoint_host.py.
#include <vector>

#include "awfl_adj_split.h"

using namespace awfl;

template <int ORD> static void unpack(const double *t, Tables<ORD> &T) {
  constexpr int NG = OrdTraits<ORD>::NGLL, HS = (ORD - 1) / 2;
  for (int x = 0; x < ORD * ORD * ORD; x++) T.recon[x] = *t++;
  for (int x = 0; x < ORD * NG; x++) T.c2g[x] = *t++;
  for (int x = 0; x < ORD * NG; x++) T.s2g[x] = *t++;
  for (int x = 0; x < NG * NG; x++) T.deriv[x] = *t++;
  for (int x = 0; x < HS + 2; x++) T.idl[x] = *t++;
  T.sigma = *t++;
  for (int x = 0; x < NG; x++) T.wts[x] = *t++;
}

template <int ORD, int DIR> static void run(const Tables<ORD> &T, adj::SplitArgs &A) {
  const long n = adj::ncell_of(A), nf = adj::nface_of<DIR>(A);
  constexpr int NG = OrdTraits<ORD>::NGLL;
  std::vector<double> edges(10 * n), lq(10 * nf), ls(5L * ORD * n), q0(5L * NG * n), lq0(5L * NG * n);
  A.edges = edges.data();
  A.lq = lq.data();
  A.ls = ls.data();
  A.q0 = q0.data();
  A.lq0 = lq0.data();
  for (long c = 0; c < n; c++) adj::split_edges<ORD, DIR>(T, A, c);
  for (long f = 0; f < nf; f++) adj::split_face<DIR>(A, f);
  for (long c = 0; c < n; c++) adj::split_cell_dt<ORD, DIR>(T, A, c);
  for (long x = 0; x < 5 * n; x++) adj::split_weno<ORD, DIR>(T, A, x);
  for (long c = 0; c < n; c++) adj::split_gather<ORD, DIR>(A, c);
}

// Tendencies of one split from the adjoint's forward functions (edges, Riemann flux,
// divergence, z source and hydrostatic pressure), for comparison with the oracle's.
template <int ORD, int DIR> static void forward(const Tables<ORD> &T, adj::SplitArgs &A, double *tend) {
  constexpr int NG = OrdTraits<ORD>::NGLL;
  const long n = adj::ncell_of(A);
  const int L = adj::line_len<DIR>(A);
  const bool periodic = A.ca.bc == BC_PERIODIC;
  constexpr int NG_ = OrdTraits<ORD>::NGLL;
  std::vector<double> edges(10 * n), src(n, 0.), q0(5L * NG_ * n);
  A.edges = edges.data();
  A.q0 = q0.data();
  for (long c = 0; c < n; c++) adj::split_edges<ORD, DIR>(T, A, c);
  if (DIR == 2) {  // source: recompute per cell
    for (long c = 0; c < n; c++) {
      int i, j, k;
      adj::decode_cell(A, c, i, j, k);
      double sten[5][ORD];
      for (int m = 0; m < ORD; m++) {
        int q = k - (ORD - 1) / 2 + m;
        bool zero_n = false;
        if (q < 0 || q >= L) {
          if (periodic) { q %= L; if (q < 0) q += L; }
          else { q = q < 0 ? 0 : L - 1; zero_n = true; }
        }
        for (int v = 0; v < 5; v++) sten[v][m] = (zero_n && v == idW) ? 0. : A.state[adj::sidx(A, v, i, j, q)];
      }
      adj::CellFwd<ORD, DIR> X;
      adj::cell_fwd<ORD, DIR>(T, sten, k, A.ca, X);
      double eL[5], eR[5];
      adj::cell_edges<ORD, DIR>(T, X, A.ca.dt, eL, eR, src[c]);
    }
  }
  for (long c = 0; c < n; c++) {
    int i, j, k;
    adj::decode_cell(A, c, i, j, k);
    const int p = DIR == 0 ? i : (DIR == 1 ? j : k);
    double F[2][5];
    for (int s = 0; s < 2; s++) {
      const int f = p + s;
      int ii, jj, kk;
      adj::at<DIR>(i, j, k, f > 0 ? f - 1 : (periodic ? L - 1 : 0), ii, jj, kk);
      const long cl = adj::cidx(A, ii, jj, kk);
      const int pl = (f > 0 || periodic) ? 5 : 0;
      adj::at<DIR>(i, j, k, f < L ? f : (periodic ? 0 : L - 1), ii, jj, kk);
      const long cr = adj::cidx(A, ii, jj, kk);
      const int pr = (f < L || periodic) ? 0 : 5;
      double qL[5], qR[5];
      for (int v = 0; v < 5; v++) {
        qL[v] = edges[(pl + v) * n + cl];
        qR[v] = edges[(pr + v) * n + cr];
      }
      adj::riemann_fwd<DIR>(qL, qR, F[s]);
      if (DIR == 2) F[s][idW] -= f < L ? A.ca.pres_g[f * NG] : A.ca.pres_g[(L - 1) * NG + NG - 1];
    }
    for (int v = 0; v < 5; v++) {
      double t = -(F[1][v] - F[0][v]) / A.ca.dxd + (DIR == 2 && v == idW ? src[c] : 0.);
      if (A.sim2d && v == idV && DIR != 1) t = 0.;
      tend[v * n + c] = t;
    }
  }
}

static void fill_args(adj::SplitArgs &A, int ord, int nx, int ny, int nz, int bc, int weno_s, int weno_w, int sim2d,
                      double dxd, double dt, const double *dens_c, const double *denstheta_c, const double *dens_g,
                      const double *denstheta_g, const double *pres_g, const double *state) {
  A.state = state;
  A.nx = nx; A.ny = ny; A.nz = nz; A.hs = (ord - 1) / 2;
  A.sim2d = sim2d;
  A.ca.nz = nz; A.ca.bc = bc; A.ca.weno_s = weno_s; A.ca.weno_w = weno_w;
  A.ca.dxd = dxd; A.ca.dt = dt;
  A.ca.dens_c = dens_c; A.ca.denstheta_c = denstheta_c; A.ca.dens_g = dens_g; A.ca.denstheta_g = denstheta_g;
  A.ca.pres_g = pres_g;
}

extern "C" int fwd_split_host(int ord, int dir, const double *tables, int nx, int ny, int nz, int bc, int weno_s,
                              int weno_w, int sim2d, double dxd, double dt, const double *dens_c,
                              const double *denstheta_c, const double *dens_g, const double *denstheta_g,
                              const double *pres_g, const double *state, double *tend) {
  adj::SplitArgs A{};
  fill_args(A, ord, nx, ny, nz, bc, weno_s, weno_w, sim2d, dxd, dt, dens_c, denstheta_c, dens_g, denstheta_g, pres_g,
            state);
  if (ord == 5) {
    static Tables<5> T;
    unpack<5>(tables, T);
    if (dir == 0) forward<5, 0>(T, A, tend); else if (dir == 1) forward<5, 1>(T, A, tend); else forward<5, 2>(T, A, tend);
  } else if (ord == 9) {
    static Tables<9> T;
    unpack<9>(tables, T);
    if (dir == 0) forward<9, 0>(T, A, tend); else if (dir == 1) forward<9, 1>(T, A, tend); else forward<9, 2>(T, A, tend);
  } else {
    return -1;
  }
  return 0;
}

extern "C" int adj_split_host(int ord, int dir, const double *tables, int nx, int ny, int nz, int bc, int weno_s,
                              int weno_w, int sim2d, double dxd, double dt, const double *dens_c,
                              const double *denstheta_c, const double *dens_g, const double *denstheta_g,
                              const double *pres_g, const double *state, double *lam) {
  adj::SplitArgs A{};
  fill_args(A, ord, nx, ny, nz, bc, weno_s, weno_w, sim2d, dxd, dt, dens_c, denstheta_c, dens_g, denstheta_g, pres_g,
            state);
  A.lam = lam;
  if (ord == 5) {
    static Tables<5> T;
    unpack<5>(tables, T);
    if (dir == 0) run<5, 0>(T, A); else if (dir == 1) run<5, 1>(T, A); else run<5, 2>(T, A);
  } else if (ord == 9) {
    static Tables<9> T;
    unpack<9>(tables, T);
    if (dir == 0) run<9, 0>(T, A); else if (dir == 1) run<9, 1>(T, A); else run<9, 2>(T, A);
  } else {
    return -1;
  }
  return 0;
}
