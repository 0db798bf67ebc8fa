// Test-infrastructure harness around the REFERENCE's own code: it includes the
// unmodified reference headers (Spatial_euler3d_cons_expl_cart_fv_Agrid.h,
// Temporal_ader.h, WenoLimiter.h, TransformMatrices.h) built against the project-written
// stand-ins under oracle/shim/, and exposes a small C ABI so Python can
// (a) generate golden fixtures, (b) time the reference's CPU step as a baseline.
//
// Compiled by oracle/Makefile into oracle/_ref/libawflref_o{ORD}.so. Nothing in the
// shipped library links it.
//
// The only arithmetic written here (not in the reference) is the benchmark initial-data
// extension: a cosine-squared bubble and seeded white theta noise, both integrated with
// the same ord^3 GLL quadrature as Spatial...h:428-485.
#ifdef AWFL_REF_CR_POW
// Variant: the reference's own headers with the pow calls of the spatial operator (time
// step and CFL) bound to a correctly rounded implementation (oracle/awfl_pow_cr.h) instead
// of glibc's. const.h (hence <cmath>) and Profiles.h are included first, so the
// hydrostatic profiles keep glibc's pow/exp and only the operator's call sites see the
// macro.
#include "const.h"
#include "Profiles.h"
#include "awfl_pow_cr.h"
#define pow(a, b) awfl_test_pow_cr((a), (b))
#endif
#include "const.h"
#include "Spatial_euler3d_cons_expl_cart_fv_Agrid.h"
#include "Temporal_ader.h"
#ifdef AWFL_REF_CR_POW
#undef pow
#endif

#include <cstdint>
#include <cstdio>
#include <fstream>
#include <string>
#include <unistd.h>

typedef Spatial_euler3d_cons_expl_cart_fv_Agrid<nTimeDerivs, timeAvg, nAder> Spatial;
typedef Temporal_ader<Spatial> Temporal;

namespace {

struct RefHandle {
  Temporal model;
  Spatial::StateArr state;
  Spatial::TracerArr tracers;
};

// splitmix64 (Steele, Lea & Flood 2014): counter-based, so value i depends only on (seed, i).
inline uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ULL;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
  return x ^ (x >> 31);
}
inline double unit_uniform(uint64_t seed, uint64_t i) {
  // 53 random bits -> [0,1)
  return (double)(splitmix64(seed * 0x100000001B3ULL + i) >> 11) * (1.0 / 9007199254740992.0);
}

}  // namespace

// Number of tracers the next awflref_create registers with addTracer before init, named
// like the reference driver's three (driver.cpp:27-29); 0 by default. Their posDef flags
// (addTracer's second argument, Spatial...h:119-125): true unless set otherwise.
int g_pending_tracers = 0;
int g_pending_pos[64];
bool g_pending_pos_set = false;

extern "C" {

void awflref_set_num_tracers(int n) {
  g_pending_tracers = n < 0 ? 0 : (n > 64 ? 64 : n);
  g_pending_pos_set = false;
}
// posDef flags of the tracers the next awflref_create registers (after set_num_tracers)
void awflref_set_tracer_pos(int n, const int *pos) {
  for (int i = 0; i < 64; i++) g_pending_pos[i] = i < n ? pos[i] : 1;
  g_pending_pos_set = true;
}
// 1 when this build has the reference's tracer transport compiled in (NO_TRACERS not
// defined in its Spatial header)
int awflref_has_tracer_transport() {
#ifdef NO_TRACERS
  return 0;
#else
  return 1;
#endif
}

int awflref_ord() { return ord; }
int awflref_ngll() { return ngll; }
int awflref_hs() { return Spatial::hs; }

void *awflref_create(int nx, int ny, int nz, double xlen, double ylen, double zlen,
                     int bc_x, int bc_y, int bc_z, int weno_scalars, int weno_winds,
                     const char *initData) {
  char path[] = "/tmp/awflref_XXXXXX";
  int fd = mkstemp(path);
  if (fd < 0) return nullptr;
  close(fd);
  {
    std::ofstream f(path);
    auto bc = [](int b) { return b == 0 ? "periodic" : "wall"; };
    char buf[64];
    f << "nx : " << nx << "\nny : " << ny << "\nnz : " << nz << "\n";
    snprintf(buf, sizeof buf, "%.17g", xlen); f << "xlen : " << buf << "\n";
    snprintf(buf, sizeof buf, "%.17g", ylen); f << "ylen : " << buf << "\n";
    snprintf(buf, sizeof buf, "%.17g", zlen); f << "zlen : " << buf << "\n";
    f << "bc_x : " << bc(bc_x) << "\nbc_y : " << bc(bc_y) << "\nbc_z : " << bc(bc_z) << "\n";
    f << "weno_scalars : " << (weno_scalars ? "true" : "false") << "\n";
    f << "weno_winds : " << (weno_winds ? "true" : "false") << "\n";
    f << "initData : " << initData << "\noutFile : none.nc\nperturb : false\n";
  }
  RefHandle *h = new RefHandle();
  static const char *const names[3] = {"uniform", "theta", "block"};
  for (int t = 0; t < g_pending_tracers; t++)
    h->model.spaceOp.addTracer(t < 3 ? names[t] : "tracer" + std::to_string(t),
                               g_pending_pos_set ? g_pending_pos[t] != 0 : true, "");
  try {
    h->model.init(path);
  } catch (...) {
    unlink(path);
    delete h;
    return nullptr;
  }
  unlink(path);
  h->state = h->model.spaceOp.createStateArr();
  h->tracers = h->model.spaceOp.createTracerArr();
  return h;
}

void awflref_destroy(void *p) { delete static_cast<RefHandle *>(p); }

// Reference initState (Spatial...h:345-500), including the hydrostatic background.
void awflref_init_state(void *p) {
  RefHandle *h = static_cast<RefHandle *>(p);
  h->model.spaceOp.initState(h->state);
}

// Reference initTracers (Spatial...h:505-560), run on the tracers awflref_create registered.
void awflref_init_tracers(void *p) {
  RefHandle *h = static_cast<RefHandle *>(p);
  h->model.spaceOp.initTracers(h->tracers);
}

long awflref_tracer_size(void *p) { return (long)static_cast<RefHandle *>(p)->tracers.totElems(); }

void awflref_get_tracers(void *p, double *out) {
  RefHandle *h = static_cast<RefHandle *>(p);
  size_t n = h->tracers.totElems();
  for (size_t i = 0; i < n; i++) out[i] = h->tracers.data()[i];
}

void awflref_set_tracers(void *p, const double *in) {
  RefHandle *h = static_cast<RefHandle *>(p);
  size_t n = h->tracers.totElems();
  for (size_t i = 0; i < n; i++) h->tracers.data()[i] = in[i];
}

// One split of Temporal_ader::timeStep (Temporal_ader.h:50-70): computeTendencies on state
// and tracers for split index spl, then state += dt*stateTend and tracers +=
// dt*tracerTend over the interior (the reference's two apply loops).
void awflref_split(void *p, double dt, int spl) {
  RefHandle *h = static_cast<RefHandle *>(p);
  Spatial &s = h->model.spaceOp;
  int constexpr hs = Spatial::hs;
  real dtloc = dt;
  s.computeTendencies(h->state, h->model.stateTendArr, h->tracers, h->model.tracerTendArr, dtloc, spl);
  auto &st = h->state;
  auto &tr = h->tracers;
  auto &tend = h->model.stateTendArr;
  auto &ttend = h->model.tracerTendArr;
  for (int l = 0; l < Spatial::numState; l++)
    for (int k = 0; k < s.nz; k++)
      for (int j = 0; j < s.ny; j++)
        for (int i = 0; i < s.nx; i++) st(l, hs + k, hs + j, hs + i) += dtloc * tend(l, k, j, i);
  for (int l = 0; l < s.numTracers; l++)
    for (int k = 0; k < s.nz; k++)
      for (int j = 0; j < s.ny; j++)
        for (int i = 0; i < s.nx; i++) tr(l, hs + k, hs + j, hs + i) += dtloc * ttend(l, k, j, i);
}

// Spatial::output (Spatial...h:1705-1791) on the current state and tracers; the netCDF
// stand-in keeps every variable it wrote (awflref_output_size / awflref_output_get).
void awflref_output(void *p, double etime) {
  RefHandle *h = static_cast<RefHandle *>(p);
  yakl::netcdf_record().clear();
  h->model.spaceOp.output(h->state, h->tracers, etime);
}
long awflref_output_size(const char *name) {
  auto &m = yakl::netcdf_record();
  auto it = m.find(name);
  return it == m.end() ? -1 : (long)it->second.size();
}
void awflref_output_get(const char *name, double *out) {
  auto &m = yakl::netcdf_record();
  auto it = m.find(name);
  if (it == m.end()) return;
  for (size_t i = 0; i < it->second.size(); i++) out[i] = it->second[i];
}

long awflref_state_size(void *p) {
  return (long)static_cast<RefHandle *>(p)->state.totElems();
}

void awflref_get_state(void *p, double *out) {
  RefHandle *h = static_cast<RefHandle *>(p);
  size_t n = h->state.totElems();
  for (size_t i = 0; i < n; i++) out[i] = h->state.data()[i];
}

void awflref_set_state(void *p, const double *in) {
  RefHandle *h = static_cast<RefHandle *>(p);
  size_t n = h->state.totElems();
  for (size_t i = 0; i < n; i++) h->state.data()[i] = in[i];
}

// Replace the theta perturbation by a bubble integrated with the same ord^3 GLL quadrature
// as initState (Spatial...h:428-485): state(idT) = sum wt*(rh*(th+tp) - rh*th).
// shape 0 = ellipsoid_linear(amp), 1 = ellipsoid_cosine(amp, pwr) (Profiles.h:49-72).
// Density and momenta perturbations are set to zero. Constant-theta background only.
void awflref_set_bubble(void *p, int shape, double x0, double y0, double z0,
                        double xrad, double yrad, double zrad, double amp, double pwr) {
  RefHandle *h = static_cast<RefHandle *>(p);
  Spatial &s = h->model.spaceOp;
  int const hs = Spatial::hs;
  auto state = h->state;
  for (int k = 0; k < s.nz; k++) {
    for (int j = 0; j < s.ny; j++) {
      for (int i = 0; i < s.nx; i++) {
        for (int l = 0; l < Spatial::numState; l++) state(l, hs + k, hs + j, hs + i) = 0;
        for (int kk = 0; kk < ord; kk++) {
          for (int jj = 0; jj < ord; jj++) {
            for (int ii = 0; ii < ord; ii++) {
              real zloc = (k + 0.5_fp) * s.dz + s.gllPts_ord(kk) * s.dz;
              real yloc;
              if (s.sim2d) { yloc = s.ylen / 2; }
              else         { yloc = (j + 0.5_fp) * s.dy + s.gllPts_ord(jj) * s.dy; }
              real xloc = (i + 0.5_fp) * s.dx + s.gllPts_ord(ii) * s.dx;
              real wt = s.gllWts_ord(kk) * s.gllWts_ord(jj) * s.gllWts_ord(ii);
              real th = 300;
              real rh = profiles::initConstTheta_density(th, zloc);
              real tp;
              if (shape == 0) tp = profiles::ellipsoid_linear(xloc, yloc, zloc, x0, y0, z0, xrad, yrad, zrad, amp);
              else            tp = profiles::ellipsoid_cosine(xloc, yloc, zloc, x0, y0, z0, xrad, yrad, zrad, amp, pwr);
              real t = th + tp;
              state(Spatial::idT, hs + k, hs + j, hs + i) += (rh * t - rh * th) * wt;
            }
          }
        }
      }
    }
  }
}

// Seeded uniform white noise on theta: n in [-amp, amp) per cell, added as
// state(idT) += hyDensCells(hs+k) * n. Cell (k,j,i) uses counter k*ny*nx + j*nx + i.
void awflref_add_theta_noise(void *p, unsigned long long seed, double amp) {
  RefHandle *h = static_cast<RefHandle *>(p);
  Spatial &s = h->model.spaceOp;
  int const hs = Spatial::hs;
  for (int k = 0; k < s.nz; k++)
    for (int j = 0; j < s.ny; j++)
      for (int i = 0; i < s.nx; i++) {
        uint64_t idx = ((uint64_t)k * s.ny + j) * s.nx + i;
        double n = (2.0 * unit_uniform(seed, idx) - 1.0) * amp;
        h->state(Spatial::idT, hs + k, hs + j, hs + i) += s.hyDensCells(hs + k) * n;
      }
}

double awflref_compute_dt(void *p, double cfl) {
  RefHandle *h = static_cast<RefHandle *>(p);
  return h->model.spaceOp.computeTimeStep(cfl, h->state);
}

// One reference time step (Temporal_ader.h:48-72): 3 splits of computeTendencies + apply.
void awflref_time_step(void *p, double dt) {
  RefHandle *h = static_cast<RefHandle *>(p);
  h->model.timeStep(h->state, h->tracers, dt);
}

// One split of computeTendencies (Spatial...h:565-594), tendencies copied out
// (numState,nz,ny,nx). Flips dimSwitch after split 2, exactly like the reference.
void awflref_compute_tendencies(void *p, double dt, int split, double *tend_out) {
  RefHandle *h = static_cast<RefHandle *>(p);
  real dtloc = dt;
  h->model.spaceOp.computeTendencies(h->state, h->model.stateTendArr, h->tracers,
                                     h->model.tracerTendArr, dtloc, split);
  size_t n = h->model.stateTendArr.totElems();
  for (size_t i = 0; i < n; i++) tend_out[i] = h->model.stateTendArr.data()[i];
}

int awflref_get_dimswitch(void *p) { return static_cast<RefHandle *>(p)->model.spaceOp.dimSwitch ? 1 : 0; }
void awflref_set_dimswitch(void *p, int v) { static_cast<RefHandle *>(p)->model.spaceOp.dimSwitch = (v != 0); }

// Constant tables as the reference's init builds them (Spatial...h:274-315).
// wenoRecon (ord,ord,ord), coefs_to_gll (ord,ngll), sten_to_gll (ord,ngll),
// derivMatrix (ngll,ngll), idl (hs+2), sigma, gll points/weights (ord) and (ngll).
void awflref_get_tables(void *p, double *wenoRecon, double *c2g, double *s2g, double *deriv,
                        double *idl, double *sigma, double *pts_ord, double *wts_ord,
                        double *pts_ngll, double *wts_ngll) {
  Spatial &s = static_cast<RefHandle *>(p)->model.spaceOp;
  for (int a = 0; a < ord; a++)
    for (int b = 0; b < ord; b++)
      for (int c = 0; c < ord; c++) wenoRecon[(a * ord + b) * ord + c] = s.wenoRecon(a, b, c);
  for (int a = 0; a < ord; a++)
    for (int b = 0; b < ngll; b++) {
      c2g[a * ngll + b] = s.coefs_to_gll(a, b);
      s2g[a * ngll + b] = s.sten_to_gll(a, b);
    }
  for (int a = 0; a < ngll; a++)
    for (int b = 0; b < ngll; b++) deriv[a * ngll + b] = s.derivMatrix(a, b);
  for (int a = 0; a < Spatial::hs + 2; a++) idl[a] = s.idl(a);
  *sigma = s.sigma;
  for (int a = 0; a < ord; a++) { pts_ord[a] = s.gllPts_ord(a); wts_ord[a] = s.gllWts_ord(a); }
  for (int a = 0; a < ngll; a++) { pts_ngll[a] = s.gllPts_ngll(a); wts_ngll[a] = s.gllWts_ngll(a); }
}

// Hydrostatic background (Spatial...h:371-425): cells (nz+2hs) and GLL (nz,ngll).
void awflref_get_background(void *p, double *dens_c, double *pres_c, double *theta_c,
                            double *denstheta_c, double *dens_g, double *pres_g,
                            double *theta_g, double *denstheta_g) {
  Spatial &s = static_cast<RefHandle *>(p)->model.spaceOp;
  for (int k = 0; k < s.nz + 2 * Spatial::hs; k++) {
    dens_c[k] = s.hyDensCells(k); pres_c[k] = s.hyPressureCells(k);
    theta_c[k] = s.hyThetaCells(k); denstheta_c[k] = s.hyDensThetaCells(k);
  }
  for (int k = 0; k < s.nz; k++)
    for (int g = 0; g < ngll; g++) {
      dens_g[k * ngll + g] = s.hyDensGLL(k, g); pres_g[k * ngll + g] = s.hyPressureGLL(k, g);
      theta_g[k * ngll + g] = s.hyThetaGLL(k, g); denstheta_g[k * ngll + g] = s.hyDensThetaGLL(k, g);
    }
}

// Single-function probes used to pin the oracle restatement function by function.
// TransformMatrices::coefs_to_tv for n = hs+1 or n = ord (TransformMatrices.h).
double awflref_coefs_to_tv(const double *a, int n) {
  int constexpr hs = Spatial::hs;
  if (n == hs + 1) {
    SArray<real, 1, hs + 1> v;
    for (int i = 0; i < hs + 1; i++) v(i) = a[i];
    return TransformMatrices::coefs_to_tv(v);
  }
  SArray<real, 1, ord> v;
  for (int i = 0; i < ord; i++) v(i) = a[i];
  return TransformMatrices::coefs_to_tv(v);
}

// weno::compute_weno_coefs (WenoLimiter.h:93-172) on one stencil.
void awflref_weno_coefs(void *p, const double *stencil, double *coefs_out) {
  Spatial &s = static_cast<RefHandle *>(p)->model.spaceOp;
  SArray<real, 1, ord> u, aw;
  for (int i = 0; i < ord; i++) u(i) = stencil[i];
  weno::compute_weno_coefs(s.wenoRecon, u, aw, s.idl, s.sigma);
  for (int i = 0; i < ord; i++) coefs_out[i] = aw(i);
}

}  // extern "C"
