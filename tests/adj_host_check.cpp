// Host check of the hand-written reverse-mode functions (awfl_adj.h) against fourth-order
// central finite differences of their own forward functions, on random states near a resting
// hydrostatic atmosphere with winds. Compiled and run by tests/test_adjoint_host.py.
//
// usage: adj_host_check <tables5.bin> <tables9.bin>
//   tablesN.bin: recon, coefs_to_gll, sten_to_gll, deriv, idl, sigma, gll weights (ngll),
//   as little-endian doubles in that order.
// Prints one line per check: "<name> <max relative error>"; exit status 1 if any check
// exceeds its bound.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "awfl_adj.h"

using namespace awfl;

static unsigned long long g_rng = 0x9e3779b97f4a7c15ULL;
static double urand() {  // splitmix64 -> [0,1)
  unsigned long long z = (g_rng += 0x9e3779b97f4a7c15ULL);
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  z ^= z >> 31;
  return (z >> 11) * 0x1.0p-53;
}
static double srand1() { return 2. * urand() - 1.; }

template <int ORD> static bool load_tables(const char *path, Tables<ORD> &T) {
  FILE *f = std::fopen(path, "rb");
  if (!f) return false;
  constexpr int NG = OrdTraits<ORD>::NGLL, HS = (ORD - 1) / 2;
  bool ok = std::fread(T.recon, sizeof(double), ORD * ORD * ORD, f) == (size_t)ORD * ORD * ORD;
  ok = ok && std::fread(T.c2g, sizeof(double), ORD * NG, f) == (size_t)ORD * NG;
  ok = ok && std::fread(T.s2g, sizeof(double), ORD * NG, f) == (size_t)ORD * NG;
  ok = ok && std::fread(T.deriv, sizeof(double), NG * NG, f) == (size_t)NG * NG;
  ok = ok && std::fread(T.idl, sizeof(double), HS + 2, f) == (size_t)HS + 2;
  ok = ok && std::fread(&T.sigma, sizeof(double), 1, f) == 1;
  ok = ok && std::fread(T.wts, sizeof(double), NG, f) == (size_t)NG;
  std::fclose(f);
  return ok;
}

static int g_fail = 0;
static void report(const char *name, double err, double bound) {
  std::printf("%s %.3e\n", name, err);
  if (!(err <= bound)) {
    std::printf("FAIL %s: %.3e > %.1e\n", name, err, bound);
    g_fail = 1;
  }
}

// ---- WENO: <law, J d> (fourth-order central differences) vs <J^T law, d>
template <int ORD> static double check_weno(const Tables<ORD> &T, bool rough) {
  double worst = 0.;
  for (int trial = 0; trial < 200; trial++) {
    double u[ORD], d[ORD], law[ORD], lu[ORD] = {};
    for (int m = 0; m < ORD; m++) {
      const double smooth = 1e-3 * std::sin(0.3 * m + trial);
      u[m] = smooth + (rough ? 1e-3 * srand1() : 1e-6 * srand1());
      d[m] = srand1();
      law[m] = srand1();
    }
    adj::weno_vjp<ORD>(T, u, law, lu);
    auto probe = [&](double h) {
      double up[ORD], a[ORD];
      for (int m = 0; m < ORD; m++) up[m] = u[m] + h * d[m];
      adj::weno_fwd<ORD>(T, up, a);
      double r = 0.;
      for (int m = 0; m < ORD; m++) r += law[m] * a[m];
      return r;
    };
    const double h = rough ? 1e-7 : 1e-9;
    const double fd = (8. * (probe(h) - probe(-h)) - (probe(2 * h) - probe(-2 * h))) / (12. * h);
    double ad = 0., sc = 0.;
    for (int m = 0; m < ORD; m++) {
      ad += lu[m] * d[m];
      sc += std::fabs(lu[m] * d[m]);
    }
    const double e = std::fabs(fd - ad) / (sc > 0 ? sc : 1.);
    if (e > worst) worst = e;
  }
  return worst;
}

// ---- Riemann flux
template <int DIR> static double check_riemann() {
  double worst = 0.;
  for (int trial = 0; trial < 400; trial++) {
    double qL[5], qR[5];
    const double rho = 1.1 + 0.05 * srand1();
    const double th = 300. + 2. * srand1();
    double vel[3] = {8. * srand1(), 8. * srand1(), 8. * srand1()};
    if (std::fabs(vel[DIR]) < 0.5) vel[DIR] = 0.5 + std::fabs(vel[DIR]);  // keep off the upwind switch
    for (int s = 0; s < 2; s++) {
      double *q = s == 0 ? qL : qR;
      const double r = rho * (1. + 1e-3 * srand1());
      q[0] = r;
      for (int k = 0; k < 3; k++) q[k + 1] = r * (vel[k] + 0.05 * srand1());
      q[4] = r * (th + 0.1 * srand1());
    }
    double lF[5], lqL[5], lqR[5], dL[5], dR[5];
    const double scale[5] = {1., 10., 10., 10., 300.};
    for (int v = 0; v < 5; v++) {
      lF[v] = srand1();
      dL[v] = srand1() * scale[v];
      dR[v] = srand1() * scale[v];
    }
    adj::riemann_vjp<DIR>(qL, qR, lF, lqL, lqR);
    auto probe = [&](double h) {
      double pL[5], pR[5], F[5];
      for (int v = 0; v < 5; v++) {
        pL[v] = qL[v] + h * dL[v];
        pR[v] = qR[v] + h * dR[v];
      }
      adj::riemann_fwd<DIR>(pL, pR, F);
      double r = 0.;
      for (int v = 0; v < 5; v++) r += lF[v] * F[v];
      return r;
    };
    const double h = 1e-5;
    const double fd = (8. * (probe(h) - probe(-h)) - (probe(2 * h) - probe(-2 * h))) / (12. * h);
    double ad = 0., sc = 0.;
    for (int v = 0; v < 5; v++) {
      ad += lqL[v] * dL[v] + lqR[v] * dR[v];
      sc += std::fabs(lqL[v] * dL[v]) + std::fabs(lqR[v] * dR[v]);
    }
    const double e = std::fabs(fd - ad) / sc;
    if (e > worst) worst = e;
  }
  return worst;
}

// ---- whole cell (reconstruction + ADER + time averages)
template <int ORD, int DIR> static double check_cell(const Tables<ORD> &T, int bc, int kb, bool weno) {
  constexpr int NG = OrdTraits<ORD>::NGLL, HS = (ORD - 1) / 2;
  const int nz = 6;
  std::vector<double> dens_c(nz + 2 * HS), dth_c(nz + 2 * HS), dens_g(nz * NG), dth_g(nz * NG), pres_g(nz * NG);
  for (int k = 0; k < nz + 2 * HS; k++) {
    dens_c[k] = 1.15 - 0.01 * k;
    dth_c[k] = 345. - 1.0 * k;
  }
  for (int k = 0; k < nz * NG; k++) {
    dens_g[k] = 1.15 - 0.01 * k / NG;
    dth_g[k] = 345. - 1.0 * k / NG;
    pres_g[k] = 1.0e5 - 100. * k / NG;
  }
  adj::CellArgs A;
  A.nz = nz; A.bc = bc; A.weno_s = weno; A.weno_w = weno;
  A.dxd = 312.5; A.dt = 0.7;
  A.dens_c = dens_c.data(); A.denstheta_c = dth_c.data(); A.dens_g = dens_g.data(); A.denstheta_g = dth_g.data();
  A.pres_g = pres_g.data();
  double worst = 0.;
  for (int trial = 0; trial < 60; trial++) {
    double sten[5][ORD], d[5][ORD], ls[5][ORD] = {};
    const double U[3] = {6. + srand1(), -4. + srand1(), 3. + srand1()};
    for (int m = 0; m < ORD; m++) {
      const double ph = 0.4 * m + trial;
      const double rp = 2e-3 * std::sin(ph) + 2e-4 * srand1();  // density perturbation
      const double r = 1.1 + rp;
      sten[0][m] = rp;
      for (int k = 0; k < 3; k++) sten[1 + k][m] = r * (U[k] + 0.3 * std::cos(ph + k) + 0.02 * srand1());
      sten[4][m] = 0.5 * std::sin(ph) + 0.05 * srand1();  // (rho theta) perturbation
    }
    const double scale[5] = {1e-3, 1., 1., 1., 0.3};
    for (int v = 0; v < 5; v++)
      for (int m = 0; m < ORD; m++) d[v][m] = srand1() * scale[v];
    double leL[5], leR[5], lsrc = srand1();
    for (int v = 0; v < 5; v++) {
      leL[v] = srand1();
      leR[v] = srand1();
    }
    adj::cell_vjp<ORD, DIR>(T, sten, kb, A, leL, leR, lsrc, ls);
    // <(leL, leR, lsrc), d(outputs)> by fourth-order central differences
    auto probe = [&](double h) {
      double sp[5][ORD];
      for (int v = 0; v < 5; v++)
        for (int m = 0; m < ORD; m++) sp[v][m] = sten[v][m] + h * d[v][m];
      adj::CellFwd<ORD, DIR> X;
      adj::cell_fwd<ORD, DIR>(T, sp, kb, A, X);
      double eL[5], eR[5], sr;
      adj::cell_edges<ORD, DIR>(T, X, A.dt, eL, eR, sr);
      double r = lsrc * sr;
      for (int v = 0; v < 5; v++) r += leL[v] * eL[v] + leR[v] * eR[v];
      return r;
    };
    const double h = 2e-5;
    const double fd = (8. * (probe(h) - probe(-h)) - (probe(2 * h) - probe(-2 * h))) / (12. * h);
    double ad = 0., sc = 0.;
    for (int v = 0; v < 5; v++)
      for (int m = 0; m < ORD; m++) {
        ad += ls[v][m] * d[v][m];
        sc += std::fabs(ls[v][m] * d[v][m]);
      }
    const double e = std::fabs(fd - ad) / sc;
    if (e > worst) worst = e;
  }
  return worst;
}

template <int ORD> static void run_order(const Tables<ORD> &T) {
  char name[96];
  std::snprintf(name, sizeof name, "weno_smooth_o%d", ORD);
  report(name, check_weno<ORD>(T, false), 1e-6);
  std::snprintf(name, sizeof name, "weno_rough_o%d", ORD);
  report(name, check_weno<ORD>(T, true), 1e-6);
  for (int weno = 0; weno < 2; weno++) {
    std::snprintf(name, sizeof name, "cell_o%d_x_weno%d", ORD, weno);
    report(name, check_cell<ORD, 0>(T, BC_PERIODIC, 2, weno), 1e-6);
    std::snprintf(name, sizeof name, "cell_o%d_y_weno%d", ORD, weno);
    report(name, check_cell<ORD, 1>(T, BC_PERIODIC, 2, weno), 1e-6);
    std::snprintf(name, sizeof name, "cell_o%d_z_weno%d", ORD, weno);
    report(name, check_cell<ORD, 2>(T, BC_PERIODIC, 2, weno), 1e-6);
    std::snprintf(name, sizeof name, "cell_o%d_zwall_bot_weno%d", ORD, weno);
    report(name, check_cell<ORD, 2>(T, BC_WALL, 0, weno), 1e-6);
    std::snprintf(name, sizeof name, "cell_o%d_zwall_top_weno%d", ORD, weno);
    report(name, check_cell<ORD, 2>(T, BC_WALL, 5, weno), 1e-6);
  }
}

int main(int argc, char **argv) {
  if (argc < 3) {
    std::fprintf(stderr, "usage: %s tables5.bin tables9.bin\n", argv[0]);
    return 2;
  }
  static Tables<5> T5;
  static Tables<9> T9;
  if (!load_tables<5>(argv[1], T5) || !load_tables<9>(argv[2], T9)) {
    std::fprintf(stderr, "cannot read tables\n");
    return 2;
  }
  report("riemann_x", check_riemann<0>(), 1e-6);
  report("riemann_y", check_riemann<1>(), 1e-6);
  report("riemann_z", check_riemann<2>(), 1e-6);
  run_order<5>(T5);
  run_order<9>(T9);
  return g_fail;
}
