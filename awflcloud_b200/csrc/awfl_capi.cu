// C ABI (include/awfl.h) of the AWFL Euler-3D ADER/WENO step: context, tables, background,
// argument checking, launches. Host code here is compiled with -ffp-contract=off so the
// init-time tables and background are bit-identical to the reference's CPU arithmetic.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "../../include/awfl.h"
#include "awfl_fp32_args.h"
#include "awfl_adj_split.h"
#include "awfl_internal.h"
#include "awfl_netcdf.h"
#include "awfl_tables.h"

using namespace awfl;

#define AWFL_VERSION_STRING "awflcloud_b200 0.1.0 (sm_100a)"

struct awfl_ctx {
  awfl_config cfg;
  int device = 0;
  int hs = 0, ngll = 0, sim2d = 0, dimswitch = 1, nsm = 148;
  double dx = 0, dy = 0, dz = 0;
  // tables (Spatial:274-315)
  std::vector<double> recon, c2g, s2g, deriv, idl, pts_ord, wts_ord, pts_ngll, wts_ngll;
  double sigma = 0;
  // hydrostatic background (Spatial:371-425)
  std::vector<double> dens_c, pres_c, theta_c, denstheta_c, dens_g, pres_g, theta_g, denstheta_g;
  double *d_bg = nullptr;  // device: dens_c | denstheta_c | dens_g | denstheta_g | pres_g | pres_c
  double *d_dens_c = nullptr, *d_denstheta_c = nullptr, *d_dens_g = nullptr, *d_denstheta_g = nullptr,
         *d_pres_g = nullptr;
  double *d_pres_c = nullptr;           // hydrostatic pressure cell averages (output)
  unsigned long long *d_cfl = nullptr;  // CFL reduction result (8 bytes)
  unsigned int *d_err = nullptr;        // a sweep's bounded wait gave up (the next 8 bytes)
  // FP32 form: FP32 copies of FP64 background constants (awfl_fp32_args.h)
  float *d_bg32 = nullptr;
  Bg32 bg32{};
  // discrete adjoint: split-start states of the recomputed window, and reverse scratch
  double *d_tape = nullptr;
  size_t tape_bytes = 0;
  double *d_adj = nullptr;
  size_t adj_bytes = 0;
  // diagnostics: 5 sums, a counter, then the block partials of the sums
  double *d_diag = nullptr;
  double *d_out = nullptr;  // output diagnostics (awfl_write_netcdf)
  size_t out_bytes = 0;
  double *d_trc = nullptr;  // tracer transport scratch (awfl_split_tracers)
  size_t trc_bytes = 0;
  size_t diag_bytes = 0;
  // a slab of a grid decomposed in x (awfl_create_slab): nslabs, this slab, the global x
  // index of its first cell, the grid's nx, and which ends border another slab
  int nslabs = 1, slab = 0, xoff = 0, nx_global = 0;
  bool xlo_ex = false, xhi_ex = false;
  // discrete adjoint: steps per recorded sub-window (0: the whole window at once)
  int adj_sub = 0;
  std::string err;
};

namespace {

thread_local std::string g_create_error;

int fail(awfl_ctx *c, int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  if (c) c->err = buf;
  else g_create_error = buf;
  return code;
}

}  // namespace

// Error message for entry points that have no context (read by awfl_last_error(NULL)).
void awfl::set_unbound_error(const char *msg) { g_create_error = msg; }

namespace {

int cuda_fail(awfl_ctx *c, cudaError_t e, const char *what) {
  return fail(c, AWFL_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

// phys_params.h:4-10
const double kGRAV = 9.81, kCP = 1004., kRD = 287., kP0 = 1.0e5;
const double kC0 = 27.5629410929725921310572974482;
const double kGAMMA = 1.40027894002789400278940027894;

// Profiles.h:8-46
double const_theta_density(double t0, double z) {
  double exner = 1. - kGRAV * z / (kCP * t0);
  double p = pow(exner, kCP / kRD) * kP0;
  double rt = pow(p / kC0, 1. / kGAMMA);
  return rt / t0;
}
double const_theta_pressure(double t0, double z) {
  double r = const_theta_density(t0, z);
  return kC0 * pow(r * t0, kGAMMA);
}
double bvf_pot_temp(double t0, double bvf, double z) { return t0 * exp(bvf * bvf * z / kGRAV); }
double bvf_density(double t0, double bvf, double z) {
  double t = bvf_pot_temp(t0, bvf, z);
  double exner = 1. - kGRAV * kGRAV / (kCP * bvf * bvf) * (t - t0) / (t * t0);
  double p = pow(exner, kCP / kRD) * kP0;
  double rt = pow(p / kC0, 1. / kGAMMA);
  return rt / t;
}
double bvf_pressure(double t0, double bvf, double z) {
  double t = bvf_pot_temp(t0, bvf, z);
  double r = bvf_density(t0, bvf, z);
  return kC0 * pow(r * t, kGAMMA);
}

// YAKL matmul_cr on (col,row) storage: out(c,r) = sum_k A(k,r)*B(c,k), k ascending.
void matmul_cr(const double *A, int K, int R, const double *B, int C, double *out) {
  for (int cc = 0; cc < C; cc++)
    for (int r = 0; r < R; r++) {
      double tmp = 0;
      for (int k = 0; k < K; k++) tmp += A[k * R + r] * B[cc * K + k];
      out[cc * R + r] = tmp;
    }
}

// WenoLimiter.h:20-25, 28-90
void convexify(double *w, int n) {
  double sum = 0.;
  const double eps = 1.0e-20;
  for (int i = 0; i < n; i++) sum += w[i];
  for (int i = 0; i < n; i++) w[i] /= (sum + eps);
}
void ideal_sigma(int ord, double *idl, double *sigma) {
  if (ord == 5) {
    *sigma = 0.73564225445964;
    idl[0] = 1.; idl[1] = 73.564225445964; idl[2] = 1.; idl[3] = 1584.89319246111;
  } else {
    *sigma = 0.0288539981181442;
    idl[0] = 1.; idl[1] = 2.15766927997459; idl[2] = 2.40224886796286;
    idl[3] = 2.15766927997459; idl[4] = 1.; idl[5] = 1136.12697719888;
  }
  convexify(idl, (ord - 1) / 2 + 2);
}

void build_tables(awfl_ctx *c) {
  const int o = c->cfg.ord, g = c->ngll, hs = c->hs;
  const double *rec, *s2c, *c2gl, *g2c, *c2d, *c2gn, *po, *wo, *pn, *wn;
  if (o == 5) {
    rec = awfl_weno_recon_o5; s2c = awfl_sten_to_coefs_o5; c2gl = awfl_coefs_to_gll_lower_o5;
    g2c = awfl_gll_to_coefs_n3_o5; c2d = awfl_coefs_to_deriv_n3_o5; c2gn = awfl_coefs_to_gll_n3_o5;
    po = awfl_gll_pts_ord_o5; wo = awfl_gll_wts_ord_o5; pn = awfl_gll_pts_ngll_o5; wn = awfl_gll_wts_ngll_o5;
  } else {
    rec = awfl_weno_recon_o9; s2c = awfl_sten_to_coefs_o9; c2gl = awfl_coefs_to_gll_lower_o9;
    g2c = awfl_gll_to_coefs_n5_o9; c2d = awfl_coefs_to_deriv_n5_o9; c2gn = awfl_coefs_to_gll_n5_o9;
    po = awfl_gll_pts_ord_o9; wo = awfl_gll_wts_ord_o9; pn = awfl_gll_pts_ngll_o9; wn = awfl_gll_wts_ngll_o9;
  }
  c->recon.assign(rec, rec + o * o * o);
  c->c2g.assign(c2gl, c2gl + o * g);
  c->s2g.assign(o * g, 0.0);
  matmul_cr(c2gl, o, g, s2c, o, c->s2g.data());  // sten_to_gll = matmul_cr(c2g_lower, s2c)
  std::vector<double> tmp(g * g);
  c->deriv.assign(g * g, 0.0);
  matmul_cr(c2d, g, g, g2c, g, tmp.data());        // derivMatrix = matmul_cr(c2g, matmul_cr(c2d, g2c))
  matmul_cr(c2gn, g, g, tmp.data(), g, c->deriv.data());
  c->idl.assign(hs + 2, 0.0);
  ideal_sigma(o, c->idl.data(), &c->sigma);
  c->pts_ord.assign(po, po + o); c->wts_ord.assign(wo, wo + o);
  c->pts_ngll.assign(pn, pn + g); c->wts_ngll.assign(wn, wn + g);
}

// Spatial:371-425 (hydrostatic background)
void build_background(awfl_ctx *c) {
  const int nz = c->cfg.nz, hs = c->hs, o = c->cfg.ord, g = c->ngll;
  const bool igw = c->cfg.data_spec == AWFL_DATA_IGW;
  c->dens_c.assign(nz + 2 * hs, 0.0); c->pres_c.assign(nz + 2 * hs, 0.0);
  c->theta_c.assign(nz + 2 * hs, 0.0); c->denstheta_c.assign(nz + 2 * hs, 0.0);
  for (int k = 0; k < nz + 2 * hs; k++) {
    for (int kk = 0; kk < o; kk++) {
      double zloc = (k - hs + 0.5) * c->dz + c->pts_ord[kk] * c->dz;
      double th, rh, ph;
      if (igw) {
        const double bvf = 0.01, t0 = 300;
        th = bvf_pot_temp(t0, bvf, zloc); rh = bvf_density(t0, bvf, zloc); ph = bvf_pressure(t0, bvf, zloc);
      } else {
        th = 300; rh = const_theta_density(th, zloc); ph = const_theta_pressure(th, zloc);
      }
      double wt = c->wts_ord[kk];
      c->dens_c[k] += rh * wt;
      c->theta_c[k] += th * wt;
      c->denstheta_c[k] += rh * th * wt;
      c->pres_c[k] += ph * wt;
    }
  }
  c->dens_g.assign(nz * g, 0.0); c->pres_g.assign(nz * g, 0.0);
  c->theta_g.assign(nz * g, 0.0); c->denstheta_g.assign(nz * g, 0.0);
  for (int k = 0; k < nz; k++)
    for (int kk = 0; kk < g; kk++) {
      double zloc = (k + 0.5) * c->dz + c->pts_ngll[kk] * c->dz;
      double th, rh, ph;
      if (igw) {
        const double bvf = 0.01, t0 = 300;
        th = bvf_pot_temp(t0, bvf, zloc); rh = bvf_density(t0, bvf, zloc); ph = bvf_pressure(t0, bvf, zloc);
      } else {
        th = 300; rh = const_theta_density(th, zloc); ph = const_theta_pressure(th, zloc);
      }
      c->dens_g[k * g + kk] = rh;
      c->theta_g[k * g + kk] = th;
      c->denstheta_g[k * g + kk] = rh * th;
      c->pres_g[k * g + kk] = ph;
    }
}

std::mutex g_tab_mutex;
unsigned g_tab_uploaded[256];  // per device: bit 0 = ord 5, bit 1 = ord 9

int ensure_tables(awfl_ctx *c) {
  std::lock_guard<std::mutex> lock(g_tab_mutex);
  const int bit = c->cfg.ord == 5 ? 1 : 2;
  if (c->device >= 0 && c->device < 256 && (g_tab_uploaded[c->device] & bit)) return AWFL_OK;
  cudaError_t e;
  if (c->cfg.ord == 5) {
    Tables<5> t;
    std::memcpy(t.recon, c->recon.data(), sizeof t.recon);
    std::memcpy(t.c2g, c->c2g.data(), sizeof t.c2g);
    std::memcpy(t.s2g, c->s2g.data(), sizeof t.s2g);
    std::memcpy(t.deriv, c->deriv.data(), sizeof t.deriv);
    std::memcpy(t.idl, c->idl.data(), sizeof t.idl);
    t.sigma = c->sigma;
    t.ridl = 1.0 / t.idl[t.HS + 1];
    std::memcpy(t.wts, c->wts_ngll.data(), sizeof t.wts);
    e = upload_tables_fp64(5, &t, sizeof t);
    if (e == cudaSuccess) e = upload_tables_adj(5, &t, sizeof t);
    if (e == cudaSuccess) e = upload_tables_tracers(5, &t, sizeof t);
    if (e == cudaSuccess) e = upload_tables_adjrev(5, &t, sizeof t);
    if (e == cudaSuccess) e = upload_tables_ens64(5, &t, sizeof t);
  } else {
    Tables<9> t;
    std::memcpy(t.recon, c->recon.data(), sizeof t.recon);
    std::memcpy(t.c2g, c->c2g.data(), sizeof t.c2g);
    std::memcpy(t.s2g, c->s2g.data(), sizeof t.s2g);
    std::memcpy(t.deriv, c->deriv.data(), sizeof t.deriv);
    std::memcpy(t.idl, c->idl.data(), sizeof t.idl);
    t.sigma = c->sigma;
    t.ridl = 1.0 / t.idl[t.HS + 1];
    std::memcpy(t.wts, c->wts_ngll.data(), sizeof t.wts);
    e = upload_tables_fp64(9, &t, sizeof t);
    if (e == cudaSuccess) e = upload_tables_adj(9, &t, sizeof t);
    if (e == cudaSuccess) e = upload_tables_tracers(9, &t, sizeof t);
    if (e == cudaSuccess) e = upload_tables_adjrev(9, &t, sizeof t);
    if (e == cudaSuccess) e = upload_tables_ens64(9, &t, sizeof t);
  }
  if (e != cudaSuccess) return cuda_fail(c, e, "upload of transform tables");
  e = upload_tables_fp32(c->cfg.ord, c->recon.data(), c->c2g.data(), c->s2g.data(), c->deriv.data(), c->idl.data(),
                         c->sigma, c->wts_ngll.data());
  if (e == cudaSuccess)
    e = upload_tables_ens32(c->cfg.ord, c->recon.data(), c->c2g.data(), c->s2g.data(), c->deriv.data(),
                            c->idl.data(), c->sigma, c->wts_ngll.data());
  if (e == cudaSuccess)
    e = upload_tables_tracers32(c->cfg.ord, c->recon.data(), c->c2g.data(), c->s2g.data(), c->deriv.data(),
                                c->idl.data(), c->sigma, c->wts_ngll.data());
  if (e != cudaSuccess) return cuda_fail(c, e, "upload of FP32 transform tables");
  if (c->device >= 0 && c->device < 256) g_tab_uploaded[c->device] |= bit;
  return AWFL_OK;
}

// FP32 background constants from the FP64 background (awfl_fp32_args.h): rows (nz+2hs) of
// rho_h, (rho theta)_h, its inverse and C0*(rho theta)_h^gamma; the same per GLL point and
// per z face. The top GLL point of cell k and the bottom point of cell k+1 are the same
// height, so both take the face value.
int build_bg32(awfl_ctx *c) {
  const int nz = c->cfg.nz, hs = c->hs, g = c->ngll;
  const size_t nr = nz + 2 * hs, ng = (size_t)nz * g, nf = nz + 1;
  std::vector<float> h(4 * (nr + ng + nf));
  float *rho_c = h.data(), *rt_c = rho_c + nr, *irt_c = rt_c + nr, *p_c = irt_c + nr;
  float *rho_g = p_c + nr, *rt_g = rho_g + ng, *irt_g = rt_g + ng, *p_g = irt_g + ng;
  float *rho_f = p_g + ng, *rt_f = rho_f + nf, *irt_f = rt_f + nf, *p_f = irt_f + nf;
  for (size_t k = 0; k < nr; k++) {
    rho_c[k] = (float)c->dens_c[k];
    rt_c[k] = (float)c->denstheta_c[k];
    irt_c[k] = (float)(1.0 / c->denstheta_c[k]);
    p_c[k] = (float)(kC0 * pow(c->denstheta_c[k], kGAMMA));
  }
  for (int f = 0; f <= nz; f++) {
    const size_t i = f < nz ? (size_t)f * g : (size_t)(nz - 1) * g + (g - 1);
    rho_f[f] = (float)c->dens_g[i];
    rt_f[f] = (float)c->denstheta_g[i];
    irt_f[f] = (float)(1.0 / c->denstheta_g[i]);
    p_f[f] = (float)c->pres_g[i];
  }
  for (int k = 0; k < nz; k++)
    for (int s = 0; s < g; s++) {
      const size_t i = (size_t)k * g + s;
      if (s == 0 || s == g - 1) {
        const int f = s == 0 ? k : k + 1;
        rho_g[i] = rho_f[f]; rt_g[i] = rt_f[f]; irt_g[i] = irt_f[f]; p_g[i] = p_f[f];
      } else {
        rho_g[i] = (float)c->dens_g[i];
        rt_g[i] = (float)c->denstheta_g[i];
        irt_g[i] = (float)(1.0 / c->denstheta_g[i]);
        p_g[i] = (float)c->pres_g[i];
      }
    }
  cudaError_t e = cudaMalloc(&c->d_bg32, h.size() * sizeof(float));
  if (e != cudaSuccess) return fail(c, AWFL_ERR_NOMEM, "cudaMalloc FP32 background: %s", cudaGetErrorString(e));
  e = cudaMemcpy(c->d_bg32, h.data(), h.size() * sizeof(float), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return cuda_fail(c, e, "upload FP32 background");
  float *d = c->d_bg32;
  auto at = [&](float *hp) { return d + (hp - h.data()); };
  c->bg32 = Bg32{at(rho_c), at(rt_c), at(irt_c), at(p_c), at(rho_g), at(rt_g), at(irt_g), at(p_g),
                 at(rho_f), at(rt_f), at(irt_f), at(p_f)};
  return AWFL_OK;
}

SweepArgs32 sweep_args32(awfl_ctx *c, void *state, void *tend, double dt, int dir, int mode) {
  SweepArgs32 A{};
  const long n = 5L * (c->cfg.nz + 2 * c->hs) * (c->cfg.ny + 2 * c->hs) * (c->cfg.nx + 2 * c->hs);
  A.state = (float *)state;
  A.comp = (float *)state + n;
  A.tend = (float *)tend;
  A.nx = c->cfg.nx; A.ny = c->cfg.ny; A.nz = c->cfg.nz;
  A.bc = dir == 0 ? c->cfg.bc_x : (dir == 1 ? c->cfg.bc_y : c->cfg.bc_z);
  A.weno_s = c->cfg.weno_scalars; A.weno_w = c->cfg.weno_winds; A.sim2d = c->sim2d; A.mode = mode;
  A.inv_dxd = (float)(1.0 / (dir == 0 ? c->dx : (dir == 1 ? c->dy : c->dz)));
  A.dt = (float)dt;
  A.bg = c->bg32;
  A.tma = 0;  // a single-grid sweep launch encodes its own tensor map (awfl_sweep.cuh)
  A.err = c->d_err;
  return A;
}

int set_device(awfl_ctx *c) {
  if (c->device < 0) return fail(c, AWFL_ERR_ARG, "host-only context (created with device < 0) cannot run device work");
  int cur = -1;
  cudaError_t e = cudaGetDevice(&cur);
  if (e != cudaSuccess) return cuda_fail(c, e, "cudaGetDevice");
  if (cur != c->device) {
    e = cudaSetDevice(c->device);
    if (e != cudaSuccess) return cuda_fail(c, e, "cudaSetDevice");
  }
  return AWFL_OK;
}

SweepArgs sweep_args(awfl_ctx *c, void *state, void *tend, double dt, int dir, int mode) {
  SweepArgs A{};
  A.state = (double *)state;
  A.tend = (double *)tend;
  A.nx = c->cfg.nx; A.ny = c->cfg.ny; A.nz = c->cfg.nz;
  A.bc = dir == 0 ? c->cfg.bc_x : (dir == 1 ? c->cfg.bc_y : c->cfg.bc_z);
  A.weno_s = c->cfg.weno_scalars; A.weno_w = c->cfg.weno_winds; A.sim2d = c->sim2d; A.mode = mode;
  A.dxd = dir == 0 ? c->dx : (dir == 1 ? c->dy : c->dz);
  A.rdxd = 1.0 / A.dxd;
  A.dt = dt;
  A.plane = 0;
  A.dens_c = c->d_dens_c; A.denstheta_c = c->d_denstheta_c;
  A.dens_g = c->d_dens_g; A.denstheta_g = c->d_denstheta_g; A.pres_g = c->d_pres_g;
  return A;
}

bool bad_ptr(const void *p) { return p == nullptr || (reinterpret_cast<uintptr_t>(p) & 7) != 0; }

bool fp32(const awfl_ctx *c) { return c->cfg.precision == AWFL_FP32; }

long state_plane(const awfl_ctx *c) {
  return 5L * (c->cfg.nz + 2 * c->hs) * (c->cfg.ny + 2 * c->hs) * (c->cfg.nx + 2 * c->hs);
}

}  // namespace

namespace {

// Grows a device buffer owned by the context (contents are not kept).
int ensure_buffer(awfl_ctx *c, double **buf, size_t *have, size_t need, const char *what) {
  if (*have >= need) return AWFL_OK;
  if (*buf) {
    cudaFree(*buf);
    *buf = nullptr;
    *have = 0;
  }
  cudaError_t e = cudaMalloc(buf, need);
  if (e != cudaSuccess) {
    *buf = nullptr;
    cudaGetLastError();
    return fail(c, AWFL_ERR_NOMEM, "cudaMalloc %s (%zu bytes): %s", what, need, cudaGetErrorString(e));
  }
  *have = need;
  return AWFL_OK;
}

int ensure_diag(awfl_ctx *c, int nblk) {
  return ensure_buffer(c, &c->d_diag, &c->diag_bytes, sizeof(double) * (size_t)(8 + 5 * nblk), "diagnostics scratch");
}

}  // namespace

// Accessors for the library's other host translation unit (awfl_ensemble.cu).
namespace awfl {
namespace host {
const awfl_config &ctx_cfg(const awfl_ctx *c) { return c->cfg; }
int ctx_hs(const awfl_ctx *c) { return c->hs; }
int ctx_sim2d(const awfl_ctx *c) { return c->sim2d; }
int ctx_nsm(const awfl_ctx *c) { return c->nsm; }
int ctx_device(const awfl_ctx *c) { return c->device; }
int ctx_set_device(awfl_ctx *c) { return set_device(c); }
long ctx_state_elems(const awfl_ctx *c) { return (fp32(c) ? 2L : 1L) * state_plane(c); }
SweepArgs ctx_sweep_args64(awfl_ctx *c, void *state, double dt, int dir) {
  return sweep_args(c, state, nullptr, dt, dir, MODE_APPLY);
}
SweepArgs32 ctx_sweep_args32(awfl_ctx *c, void *state, double dt, int dir) {
  return sweep_args32(c, state, nullptr, dt, dir, MODE_APPLY);
}
}  // namespace host
}  // namespace awfl

extern "C" {

const char *awfl_version(void) { return AWFL_VERSION_STRING; }

const char *awfl_last_error(const awfl_ctx *ctx) {
  if (!ctx) return g_create_error.c_str();
  return ctx->err.c_str();
}

int awfl_create(const awfl_config *cfg, int device, awfl_ctx **out) {
  if (!cfg || !out) return fail(nullptr, AWFL_ERR_ARG, "awfl_create: NULL argument");
  *out = nullptr;
  if (cfg->ord != 5 && cfg->ord != 9) return fail(nullptr, AWFL_ERR_ARG, "ord must be 5 or 9 (got %d)", cfg->ord);
  if (cfg->precision != AWFL_FP64 && cfg->precision != AWFL_FP32)
    return fail(nullptr, AWFL_ERR_NOT_BUILT, "precision %d is not available in this build", cfg->precision);
  const int hs = (cfg->ord - 1) / 2;
  if (cfg->nx < 1 || cfg->ny < 1 || cfg->nz < 1) return fail(nullptr, AWFL_ERR_ARG, "nx, ny, nz must be >= 1");
  // the kernels lay y and z along grid dimensions of at most 65535 blocks
  if (cfg->ny > 65535 || cfg->nz > 65535) return fail(nullptr, AWFL_ERR_ARG, "ny and nz must be <= 65535");
  if (!(cfg->xlen > 0) || !(cfg->ylen > 0) || !(cfg->zlen > 0))
    return fail(nullptr, AWFL_ERR_ARG, "xlen, ylen, zlen must be > 0");
  const int bcs[3] = {cfg->bc_x, cfg->bc_y, cfg->bc_z};
  const int ns[3] = {cfg->nx, cfg->ny, cfg->nz};
  const char *nm[3] = {"x", "y", "z"};
  for (int d = 0; d < 3; d++) {
    if (bcs[d] != AWFL_BC_PERIODIC && bcs[d] != AWFL_BC_WALL)
      return fail(nullptr, AWFL_ERR_ARG, "bc_%s must be periodic (0) or wall (1)", nm[d]);
    const bool swept = !(d == 1 && cfg->ny == 1);
    if (swept && bcs[d] == AWFL_BC_PERIODIC && ns[d] < hs)
      return fail(nullptr, AWFL_ERR_ARG, "periodic n%s = %d is smaller than the halo width %d", nm[d], ns[d], hs);
  }
  if (cfg->data_spec < AWFL_DATA_THERMAL || cfg->data_spec > AWFL_DATA_IGW)
    return fail(nullptr, AWFL_ERR_ARG, "data_spec must be 1..4");
  long long cells = (long long)(cfg->nx + 2 * hs) * (cfg->ny + 2 * hs) * (cfg->nz + 2 * hs);
  if (cells * 5 > (1LL << 40)) return fail(nullptr, AWFL_ERR_ARG, "grid too large");

  awfl_ctx *c = new (std::nothrow) awfl_ctx();
  if (!c) return fail(nullptr, AWFL_ERR_NOMEM, "host allocation failed");
  c->cfg = *cfg;
  c->device = device;
  c->hs = hs;
  c->ngll = cfg->ord == 5 ? 3 : 5;
  c->sim2d = cfg->ny == 1;
  c->dx = cfg->xlen / cfg->nx;
  c->dy = cfg->ylen / cfg->ny;
  c->dz = cfg->zlen / cfg->nz;
  build_tables(c);
  build_background(c);
  if (device < 0) {  // host-only context: tables and background, no device resources
    *out = c;
    return AWFL_OK;
  }

  int rc = set_device(c);
  if (rc) { g_create_error = c->err; delete c; return rc; }
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) == cudaSuccess) c->nsm = prop.multiProcessorCount;
  rc = ensure_tables(c);
  if (rc) { g_create_error = c->err; delete c; return rc; }
  const int nz = cfg->nz, g = c->ngll;
  const size_t nbg = (size_t)3 * (nz + 2 * hs) + (size_t)3 * nz * g;
  cudaError_t e = cudaMalloc(&c->d_bg, nbg * sizeof(double) + 64);
  if (e != cudaSuccess) { fail(nullptr, AWFL_ERR_NOMEM, "cudaMalloc background: %s", cudaGetErrorString(e)); delete c; return AWFL_ERR_NOMEM; }
  c->d_dens_c = c->d_bg;
  c->d_denstheta_c = c->d_dens_c + (nz + 2 * hs);
  c->d_dens_g = c->d_denstheta_c + (nz + 2 * hs);
  c->d_denstheta_g = c->d_dens_g + nz * g;
  c->d_pres_g = c->d_denstheta_g + nz * g;
  c->d_pres_c = c->d_pres_g + nz * g;
  c->d_cfl = reinterpret_cast<unsigned long long *>(c->d_pres_c + (nz + 2 * hs));
  c->d_err = reinterpret_cast<unsigned int *>(c->d_cfl + 1);
  std::vector<double> h;
  h.reserve(nbg);
  h.insert(h.end(), c->dens_c.begin(), c->dens_c.end());
  h.insert(h.end(), c->denstheta_c.begin(), c->denstheta_c.end());
  h.insert(h.end(), c->dens_g.begin(), c->dens_g.end());
  h.insert(h.end(), c->denstheta_g.begin(), c->denstheta_g.end());
  h.insert(h.end(), c->pres_g.begin(), c->pres_g.end());
  h.insert(h.end(), c->pres_c.begin(), c->pres_c.end());
  e = cudaMemcpy(c->d_bg, h.data(), nbg * sizeof(double), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(c->d_err, 0, sizeof(unsigned int));
  if (e != cudaSuccess) { cuda_fail(nullptr, e, "upload background"); g_create_error = "upload background: " + std::string(cudaGetErrorString(e)); cudaFree(c->d_bg); delete c; return AWFL_ERR_CUDA; }
  if (cfg->precision == AWFL_FP32) {
    rc = build_bg32(c);
    warm_tma_encoder();
    if (rc) { g_create_error = c->err; cudaFree(c->d_bg); if (c->d_bg32) cudaFree(c->d_bg32); delete c; return rc; }
  }
  *out = c;
  return AWFL_OK;
}

int awfl_destroy(awfl_ctx *c) {
  if (!c) return AWFL_OK;
  if (c->d_bg && c->device >= 0) {
    set_device(c);
    cudaFree(c->d_bg);
    if (c->d_bg32) cudaFree(c->d_bg32);
    if (c->d_tape) cudaFree(c->d_tape);
    if (c->d_adj) cudaFree(c->d_adj);
    if (c->d_diag) cudaFree(c->d_diag);
    if (c->d_out) cudaFree(c->d_out);
    if (c->d_trc) cudaFree(c->d_trc);
  }
  delete c;
  return AWFL_OK;
}

int awfl_sizes(const awfl_ctx *c, long *state_elems, long *tend_elems, int *hs) {
  if (!c) return AWFL_ERR_ARG;
  const int h = c->hs;
  // FP32 contexts: value plane followed by the Kahan compensation plane
  if (state_elems) *state_elems = (fp32(c) ? 2L : 1L) * 5L * (c->cfg.nz + 2 * h) * (c->cfg.ny + 2 * h) * (c->cfg.nx + 2 * h);
  if (tend_elems) *tend_elems = 5L * c->cfg.nz * c->cfg.ny * c->cfg.nx;
  if (hs) *hs = h;
  return AWFL_OK;
}

int awfl_get_dimswitch(const awfl_ctx *c, int *value) {
  if (!c || !value) return AWFL_ERR_ARG;
  *value = c->dimswitch;
  return AWFL_OK;
}

int awfl_set_dimswitch(awfl_ctx *c, int value) {
  if (!c) return AWFL_ERR_ARG;
  c->dimswitch = value != 0;
  return AWFL_OK;
}

int awfl_init_state(awfl_ctx *c, void *d_state, const awfl_init_spec *spec, void *stream) {
  if (!c) return AWFL_ERR_ARG;
  if (bad_ptr(d_state)) return fail(c, AWFL_ERR_ARG, "awfl_init_state: state pointer is NULL or misaligned");
  if (spec && spec->kind != AWFL_INIT_REFERENCE && spec->kind != AWFL_INIT_BUBBLE)
    return fail(c, AWFL_ERR_ARG, "awfl_init_state: unknown kind %d", spec->kind);
  if (spec && spec->kind == AWFL_INIT_BUBBLE && c->cfg.data_spec == AWFL_DATA_IGW)
    return fail(c, AWFL_ERR_ARG, "awfl_init_state: bubble initial data needs a constant-theta background");
  int rc = set_device(c);
  if (rc) return rc;
  InitLaunch L{};
  std::memset(&L, 0, sizeof L);
  L.state = d_state;
  if (fp32(c)) {
    L.state32 = (float *)d_state;
    L.comp32 = (float *)d_state + state_plane(c);
  }
  L.nx = c->cfg.nx; L.ny = c->cfg.ny; L.nz = c->cfg.nz; L.hs = c->hs; L.ord = c->cfg.ord;
  L.xoff = c->xoff; L.nx_global = c->nx_global > 0 ? c->nx_global : c->cfg.nx;
  L.dx = c->dx; L.dy = c->dy; L.dz = c->dz; L.xlen = c->cfg.xlen; L.ylen = c->cfg.ylen; L.zlen = c->cfg.zlen;
  L.data_spec = c->cfg.data_spec; L.sim2d = c->sim2d;
  if (spec) {
    L.kind = spec->kind; L.shape = spec->shape;
    L.x0 = spec->x0; L.y0 = spec->y0; L.z0 = spec->z0; L.xrad = spec->xrad; L.yrad = spec->yrad; L.zrad = spec->zrad;
    L.amp = spec->amp; L.pwr = spec->pwr; L.noise_amp = spec->noise_amp; L.seed = spec->noise_seed;
    L.noise_kind = spec->noise_kind;
  }
  L.dens_c = c->d_dens_c;
  for (int m = 0; m < c->cfg.ord; m++) { L.pts[m] = c->pts_ord[m]; L.wts[m] = c->wts_ord[m]; }
  cudaError_t e = launch_init_state_fp64(L, (cudaStream_t)stream);
  if (e != cudaSuccess) return cuda_fail(c, e, "init_state kernel");
  return AWFL_OK;
}

int awfl_state_sums(awfl_ctx *c, const void *d_state, double *sums, void *stream) {
  if (!c || !sums) return AWFL_ERR_ARG;
  if (bad_ptr(d_state)) return fail(c, AWFL_ERR_ARG, "awfl_state_sums: state pointer is NULL or misaligned");
  int rc = set_device(c);
  if (rc) return rc;
  const int nblk = c->nsm * 2;
  rc = ensure_diag(c, nblk);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e = launch_state_sums(d_state, fp32(c), state_plane(c), c->cfg.nx, c->cfg.ny, c->cfg.nz, c->hs,
                                    c->dx * c->dy * c->dz, c->d_diag + 8, nblk, c->d_diag, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(sums, c->d_diag, 5 * sizeof(double), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_fail(c, e, "awfl_state_sums");
  return AWFL_OK;
}

int awfl_output_fields(awfl_ctx *c, const void *d_state, double *d_fields, void *stream) {
  if (!c) return AWFL_ERR_ARG;
  if (bad_ptr(d_state)) return fail(c, AWFL_ERR_ARG, "awfl_output_fields: state pointer is NULL or misaligned");
  if (bad_ptr(d_fields)) return fail(c, AWFL_ERR_ARG, "awfl_output_fields: fields pointer is NULL or misaligned");
  int rc = set_device(c);
  if (rc) return rc;
  cudaError_t e = launch_output_fields(d_state, fp32(c), state_plane(c), c->d_dens_c, c->d_denstheta_c, c->d_pres_c,
                                       c->cfg.nx, c->cfg.ny, c->cfg.nz, c->hs, c->nsm, d_fields,
                                       (cudaStream_t)stream);
  if (e != cudaSuccess) return cuda_fail(c, e, "awfl_output_fields");
  return AWFL_OK;
}

int awfl_output_tracer_fields(awfl_ctx *c, const void *d_state, const double *d_tracers, int ntracers,
                              double *d_fields, void *stream) {
  if (!c) return AWFL_ERR_ARG;
  if (ntracers < 0) return fail(c, AWFL_ERR_ARG, "awfl_output_tracer_fields: ntracers < 0");
  if (ntracers == 0) return AWFL_OK;
  if (bad_ptr(d_state) || bad_ptr(d_tracers) || bad_ptr(d_fields))
    return fail(c, AWFL_ERR_ARG, "awfl_output_tracer_fields: a pointer is NULL or misaligned");
  int rc = set_device(c);
  if (rc) return rc;
  cudaError_t e = launch_tracer_fields(d_state, fp32(c), state_plane(c), c->d_dens_c, d_tracers, ntracers, c->cfg.nx,
                                       c->cfg.ny, c->cfg.nz, c->hs, c->nsm, d_fields, (cudaStream_t)stream);
  if (e != cudaSuccess) return cuda_fail(c, e, "awfl_output_tracer_fields");
  return AWFL_OK;
}

int awfl_write_netcdf_fields_tracers(awfl_ctx *c, const char *path, const double *h_fields, int ntracers,
                                     const char *const *names, double etime) {
  if (!c) return AWFL_ERR_ARG;
  if (!path || !h_fields) return fail(c, AWFL_ERR_ARG, "awfl_write_netcdf_fields: path or fields is NULL");
  if (ntracers < 0 || (ntracers > 0 && !names))
    return fail(c, AWFL_ERR_ARG, "awfl_write_netcdf: ntracers < 0, or tracer names missing");
  std::vector<std::string> tn;
  for (int t = 0; t < ntracers; t++) {
    if (!names[t] || !names[t][0]) return fail(c, AWFL_ERR_ARG, "awfl_write_netcdf: tracer %d has no name", t);
    tn.emplace_back(names[t]);
  }
  std::string err;
  if (nc::write(path, c->cfg.nx, c->cfg.ny, c->cfg.nz, c->dx, c->dy, c->dz, c->hs, c->dens_c.data(),
                c->pres_c.data(), c->theta_c.data(), h_fields, etime, &err, tn) != 0)
    return fail(c, AWFL_ERR_IO, "awfl_write_netcdf: %s", err.c_str());
  return AWFL_OK;
}

int awfl_write_netcdf_fields(awfl_ctx *c, const char *path, const double *h_fields, double etime) {
  return awfl_write_netcdf_fields_tracers(c, path, h_fields, 0, nullptr, etime);
}

int awfl_write_netcdf_tracers(awfl_ctx *c, const char *path, const void *d_state, const double *d_tracers,
                              int ntracers, const char *const *names, double etime, void *stream) {
  if (!c) return AWFL_ERR_ARG;
  if (!path) return fail(c, AWFL_ERR_ARG, "awfl_write_netcdf: path is NULL");
  if (bad_ptr(d_state)) return fail(c, AWFL_ERR_ARG, "awfl_write_netcdf: state pointer is NULL or misaligned");
  if (ntracers < 0 || (ntracers > 0 && (!names || bad_ptr(d_tracers))))
    return fail(c, AWFL_ERR_ARG, "awfl_write_netcdf: ntracers < 0, or tracers / names missing");
  int rc = set_device(c);
  if (rc) return rc;
  const size_t cells = (size_t)c->cfg.nx * c->cfg.ny * c->cfg.nz;
  const size_t n = (6 + (size_t)ntracers) * cells;
  rc = ensure_buffer(c, &c->d_out, &c->out_bytes, n * sizeof(double), "output fields");
  if (rc) return rc;
  rc = awfl_output_fields(c, d_state, c->d_out, stream);
  if (rc) return rc;
  rc = awfl_output_tracer_fields(c, d_state, d_tracers, ntracers, c->d_out + 6 * cells, stream);
  if (rc) return rc;
  std::vector<double> h(n);
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e = cudaMemcpyAsync(h.data(), c->d_out, n * sizeof(double), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_fail(c, e, "awfl_write_netcdf");
  return awfl_write_netcdf_fields_tracers(c, path, h.data(), ntracers, names, etime);
}

int awfl_write_netcdf(awfl_ctx *c, const char *path, const void *d_state, double etime, void *stream) {
  return awfl_write_netcdf_tracers(c, path, d_state, nullptr, 0, nullptr, etime, stream);
}

int awfl_init_tracers(awfl_ctx *c, double *d_tracers, int ntracers, void *stream) {
  if (!c) return AWFL_ERR_ARG;
  if (ntracers < 0) return fail(c, AWFL_ERR_ARG, "awfl_init_tracers: ntracers < 0");
  if (ntracers == 0) return AWFL_OK;
  if (bad_ptr(d_tracers)) return fail(c, AWFL_ERR_ARG, "awfl_init_tracers: tracer pointer is NULL or misaligned");
  int rc = set_device(c);
  if (rc) return rc;
  InitLaunch L{};
  std::memset(&L, 0, sizeof L);
  L.state = d_tracers;
  L.nx = c->cfg.nx; L.ny = c->cfg.ny; L.nz = c->cfg.nz; L.hs = c->hs; L.ord = c->cfg.ord;
  L.xoff = c->xoff; L.nx_global = c->nx_global > 0 ? c->nx_global : c->cfg.nx;
  L.dx = c->dx; L.dy = c->dy; L.dz = c->dz; L.xlen = c->cfg.xlen; L.ylen = c->cfg.ylen; L.zlen = c->cfg.zlen;
  L.sim2d = c->sim2d;
  for (int m = 0; m < c->cfg.ord; m++) { L.pts[m] = c->pts_ord[m]; L.wts[m] = c->wts_ord[m]; }
  cudaError_t e = launch_init_tracers_fp64(L, ntracers, (cudaStream_t)stream);
  if (e != cudaSuccess) return cuda_fail(c, e, "init_tracers kernel");
  return AWFL_OK;
}

int awfl_check_state(awfl_ctx *c, const void *d_state, long *bad_cells, void *stream) {
  if (!c) return AWFL_ERR_ARG;
  if (bad_ptr(d_state)) return fail(c, AWFL_ERR_ARG, "awfl_check_state: state pointer is NULL or misaligned");
  int rc = set_device(c);
  if (rc) return rc;
  rc = ensure_diag(c, c->nsm * 2);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  unsigned long long *cnt = reinterpret_cast<unsigned long long *>(c->d_diag + 5);
  unsigned long long h = 0;
  cudaError_t e = cudaMemsetAsync(cnt, 0, sizeof *cnt, st);
  if (e == cudaSuccess)
    e = launch_check_state(d_state, fp32(c), state_plane(c), c->d_dens_c, c->cfg.nx, c->cfg.ny, c->cfg.nz, c->hs,
                           c->nsm, cnt, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&h, cnt, sizeof h, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_fail(c, e, "awfl_check_state");
  if (bad_cells) *bad_cells = (long)h;
  if (h) return fail(c, AWFL_ERR_STATE, "%llu cells with a non-finite value or a non-positive density", h);
  unsigned int werr = 0;  // a sweep whose bounded wait for its staged rows gave up
  e = cudaMemcpy(&werr, c->d_err, sizeof werr, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_fail(c, e, "awfl_check_state");
  if (werr) return fail(c, AWFL_ERR_TIMEOUT, "a sweep gave up waiting for its staged stencil rows");
  return AWFL_OK;
}

int awfl_cfl(awfl_ctx *c, const void *d_state, double cfl, double *h_dt, void *stream) {
  if (!c || !h_dt) return AWFL_ERR_ARG;
  if (bad_ptr(d_state)) return fail(c, AWFL_ERR_ARG, "awfl_cfl: state pointer is NULL or misaligned");
  if (!(cfl > 0)) return fail(c, AWFL_ERR_ARG, "awfl_cfl: cfl must be > 0");
  int rc = set_device(c);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  static const unsigned long long inf_bits = 0x7ff0000000000000ULL;
  cudaError_t e = cudaMemcpyAsync(c->d_cfl, &inf_bits, sizeof inf_bits, cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) return cuda_fail(c, e, "awfl_cfl init");
  if (fp32(c))
    e = launch_cfl_fp32((const float *)d_state, c->d_dens_c, c->d_denstheta_c, cfl, c->dx, c->dy, c->dz, c->cfg.nx,
                        c->cfg.ny, c->cfg.nz, c->hs, c->nsm, c->d_cfl, st);
  else
    e = launch_cfl_fp64((const double *)d_state, c->d_dens_c, c->d_denstheta_c, cfl, c->dx, c->dy, c->dz, c->cfg.nx,
                        c->cfg.ny, c->cfg.nz, c->hs, c->nsm, c->d_cfl, st);
  if (e != cudaSuccess) return cuda_fail(c, e, "cfl kernel");
  unsigned long long bits = 0;
  e = cudaMemcpyAsync(&bits, c->d_cfl, sizeof bits, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_fail(c, e, "awfl_cfl readback");
  double dt;
  std::memcpy(&dt, &bits, sizeof dt);
  if (!(dt > 0) || !std::isfinite(dt)) return fail(c, AWFL_ERR_STATE, "awfl_cfl: non-finite or non-positive time step (%g)", dt);
  *h_dt = dt;
  return AWFL_OK;
}

int awfl_compute_tendencies(awfl_ctx *c, void *d_state, void *d_tend, double dt, int dir, void *stream) {
  if (!c) return AWFL_ERR_ARG;
  if (dir < 0 || dir > 2) return fail(c, AWFL_ERR_ARG, "dir must be 0, 1 or 2");
  if (dir == 0 && (c->xlo_ex || c->xhi_ex))
    return fail(c, AWFL_ERR_ARG, "the x split of a slab needs its neighbours' columns (awfl_split_slab)");
  if (bad_ptr(d_state) || bad_ptr(d_tend)) return fail(c, AWFL_ERR_ARG, "state/tend pointer is NULL or misaligned");
  int rc = set_device(c);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e;
  if (dir == 1 && c->sim2d) {  // Spatial:573-576: the Y tendency is zero in 2-D
    e = cudaMemsetAsync(d_tend, 0, (fp32(c) ? sizeof(float) : sizeof(double)) * 5L * c->cfg.nz * c->cfg.ny * c->cfg.nx, st);
  } else if (fp32(c)) {
    e = launch_sweep_fp32(c->cfg.ord, dir, sweep_args32(c, d_state, d_tend, dt, dir, MODE_TEND), st);
  } else {
    e = launch_sweep_fp64(c->cfg.ord, dir, sweep_args(c, d_state, d_tend, dt, dir, MODE_TEND), st);
  }
  if (e != cudaSuccess) return cuda_fail(c, e, "compute_tendencies");
  return AWFL_OK;
}

int awfl_apply_tendencies(awfl_ctx *c, void *d_state, const void *d_tend, double dt, void *stream) {
  if (!c) return AWFL_ERR_ARG;
  if (bad_ptr(d_state) || bad_ptr(d_tend)) return fail(c, AWFL_ERR_ARG, "state/tend pointer is NULL or misaligned");
  int rc = set_device(c);
  if (rc) return rc;
  cudaError_t e;
  if (fp32(c))
    e = launch_apply_fp32((float *)d_state, (float *)d_state + state_plane(c), (const float *)d_tend, (float)dt,
                          c->cfg.nx, c->cfg.ny, c->cfg.nz, c->hs, c->nsm, (cudaStream_t)stream);
  else
    e = launch_apply_fp64((double *)d_state, (const double *)d_tend, dt, c->cfg.nx, c->cfg.ny, c->cfg.nz, c->hs,
                          c->nsm, (cudaStream_t)stream);
  if (e != cudaSuccess) return cuda_fail(c, e, "apply_tendencies");
  return AWFL_OK;
}

int awfl_split(awfl_ctx *c, void *d_state, double dt, int dir, void *stream) {
  if (!c) return AWFL_ERR_ARG;
  if (dir < 0 || dir > 2) return fail(c, AWFL_ERR_ARG, "dir must be 0, 1 or 2");
  if (dir == 0 && (c->xlo_ex || c->xhi_ex))
    return fail(c, AWFL_ERR_ARG, "the x split of a slab needs its neighbours' columns (awfl_split_slab)");
  if (bad_ptr(d_state)) return fail(c, AWFL_ERR_ARG, "state pointer is NULL or misaligned");
  int rc = set_device(c);
  if (rc) return rc;
  if (dir == 1 && c->sim2d) {  // zero tendencies (Spatial:572-575)
    // FP64: state += dt*0 as the reference applies them (no value changes; a -0 becomes
    // +0); the FP32 form's compensated update is left out, its state is unchanged
    if (fp32(c)) return AWFL_OK;
    cudaError_t e = launch_add_zero_fp64((double *)d_state, 5, c->cfg.nx, c->cfg.ny, c->cfg.nz, c->hs, c->nsm,
                                         (cudaStream_t)stream);
    return e == cudaSuccess ? AWFL_OK : cuda_fail(c, e, "split");
  }
  cudaError_t e = fp32(c)
                      ? launch_sweep_fp32(c->cfg.ord, dir, sweep_args32(c, d_state, nullptr, dt, dir, MODE_APPLY),
                                          (cudaStream_t)stream)
                      : launch_sweep_fp64(c->cfg.ord, dir, sweep_args(c, d_state, nullptr, dt, dir, MODE_APPLY),
                                          (cudaStream_t)stream);
  if (e != cudaSuccess) return cuda_fail(c, e, "split");
  return AWFL_OK;
}

int awfl_step(awfl_ctx *c, void *d_state, double dt, void *stream) {
  if (!c) return AWFL_ERR_ARG;
  if (c->xlo_ex || c->xhi_ex)
    return fail(c, AWFL_ERR_ARG, "a slab's step exchanges columns between its x split's slabs (awfl_split_slab)");
  for (int spl = 0; spl < 3; spl++) {
    const int dir = c->dimswitch ? spl : 2 - spl;
    int rc = awfl_split(c, d_state, dt, dir, stream);
    if (rc) return rc;
  }
  c->dimswitch = !c->dimswitch;
  return AWFL_OK;
}

int awfl_create_slab(const awfl_config *global, int nslabs, int slab, int device, awfl_ctx **out) {
  if (!global || !out) return fail(nullptr, AWFL_ERR_ARG, "awfl_create_slab: NULL argument");
  *out = nullptr;
  if (global->ord != 5 && global->ord != 9) return fail(nullptr, AWFL_ERR_ARG, "ord must be 5 or 9 (got %d)", global->ord);
  const int hs = (global->ord - 1) / 2;
  if (nslabs < 1 || slab < 0 || slab >= nslabs)
    return fail(nullptr, AWFL_ERR_ARG, "awfl_create_slab: slab %d of %d", slab, nslabs);
  if (global->nx < (long)nslabs * (hs + 1))
    return fail(nullptr, AWFL_ERR_ARG, "awfl_create_slab: nx = %d leaves a slab of %d slabs narrower than %d cells",
                global->nx, nslabs, hs + 1);
  const int base = global->nx / nslabs, extra = global->nx % nslabs;
  awfl_config local = *global;
  local.nx = base + (slab < extra ? 1 : 0);
  int rc = awfl_create(&local, device, out);
  if (rc) return rc;
  awfl_ctx *c = *out;
  c->nslabs = nslabs;
  c->slab = slab;
  c->xoff = slab * base + (slab < extra ? slab : extra);
  c->nx_global = global->nx;
  c->dx = global->xlen / global->nx;  // the grid's spacing, as the undivided grid computes it
  if (nslabs > 1) {
    const bool periodic = global->bc_x == AWFL_BC_PERIODIC;
    c->xlo_ex = periodic || slab > 0;
    c->xhi_ex = periodic || slab < nslabs - 1;
  }
  return AWFL_OK;
}

int awfl_slab_info(const awfl_ctx *c, int *nslabs, int *slab, int *xoff, int *nx_global, long *halo_elems) {
  if (!c) return AWFL_ERR_ARG;
  if (nslabs) *nslabs = c->nslabs;
  if (slab) *slab = c->slab;
  if (xoff) *xoff = c->xoff;
  if (nx_global) *nx_global = c->nx_global > 0 ? c->nx_global : c->cfg.nx;
  if (halo_elems) *halo_elems = 2L * 5 * c->cfg.nz * c->cfg.ny * (c->hs + 1);
  return AWFL_OK;
}

int awfl_slab_pack(awfl_ctx *c, const void *d_state, void *d_send, void *stream) {
  if (!c) return AWFL_ERR_ARG;
  if (bad_ptr(d_state) || (reinterpret_cast<uintptr_t>(d_send) & 7) != 0 || !d_send)
    return fail(c, AWFL_ERR_ARG, "awfl_slab_pack: state or send pointer is NULL or misaligned");
  if (c->cfg.nx < c->hs + 1) return fail(c, AWFL_ERR_ARG, "awfl_slab_pack: the slab is narrower than hs+1 cells");
  int rc = set_device(c);
  if (rc) return rc;
  cudaError_t e = launch_slab_pack(d_state, fp32(c) ? 4 : 8, c->cfg.nx, c->cfg.ny, c->cfg.nz, c->hs, d_send,
                                   (cudaStream_t)stream);
  if (e != cudaSuccess) return cuda_fail(c, e, "slab_pack");
  return AWFL_OK;
}

int awfl_split_slab(awfl_ctx *c, void *d_state, const void *d_recv, double dt, void *stream) {
  if (!c) return AWFL_ERR_ARG;
  if (bad_ptr(d_state)) return fail(c, AWFL_ERR_ARG, "state pointer is NULL or misaligned");
  if ((c->xlo_ex || c->xhi_ex) && (!d_recv || (reinterpret_cast<uintptr_t>(d_recv) & 7) != 0))
    return fail(c, AWFL_ERR_ARG, "awfl_split_slab: the received columns are NULL or misaligned");
  int rc = set_device(c);
  if (rc) return rc;
  const long side = 5L * c->cfg.nz * c->cfg.ny * (c->hs + 1);
  cudaError_t e;
  if (fp32(c)) {
    SweepArgs32 A = sweep_args32(c, d_state, nullptr, dt, 0, MODE_APPLY);
    A.xh[0] = c->xlo_ex ? (const float *)d_recv : nullptr;
    A.xh[1] = c->xhi_ex ? (const float *)d_recv + side : nullptr;
    e = launch_sweep_fp32(c->cfg.ord, 0, A, (cudaStream_t)stream);
  } else {
    SweepArgs A = sweep_args(c, d_state, nullptr, dt, 0, MODE_APPLY);
    A.xh[0] = c->xlo_ex ? (const double *)d_recv : nullptr;
    A.xh[1] = c->xhi_ex ? (const double *)d_recv + side : nullptr;
    e = launch_sweep_fp64(c->cfg.ord, 0, A, (cudaStream_t)stream);
  }
  if (e != cudaSuccess) return cuda_fail(c, e, "split_slab");
  return AWFL_OK;
}

// One tracer split; io: TRC_IN_DIVIDED -- the tracers arrive divided by the current
// density (the previous split of the same step left them so); TRC_OUT_DIVIDED -- leave
// the interior divided by the post-split density for the next split. Either way the
// values are the ones the undivided round trip gives, bit for bit.
static int split_tracers_io(awfl_ctx *c, void *d_state, double *d_tracers, int ntracers, const int *pos, double dt,
                            int dir, int io, void *stream) {
  if (!c) return AWFL_ERR_ARG;
  if (c->nslabs > 1) return fail(c, AWFL_ERR_ARG, "tracer transport is not available on a slab");
  if (dir < 0 || dir > 2) return fail(c, AWFL_ERR_ARG, "dir must be 0, 1 or 2");
  if (ntracers < 0 || ntracers > 64) return fail(c, AWFL_ERR_ARG, "ntracers must be in [0, 64]");
  if (ntracers == 0) return awfl_split(c, d_state, dt, dir, stream);
  if (bad_ptr(d_state) || bad_ptr(d_tracers)) return fail(c, AWFL_ERR_ARG, "state or tracer pointer is NULL or misaligned");
  if (!pos) return fail(c, AWFL_ERR_ARG, "pos (positive-definite flags) is NULL");
  // (every stencil index maps into the line for any length: a wall copies cell 0 or n-1;
  // periodic directions shorter than hs are refused by awfl_create)
  int rc = set_device(c);
  if (rc) return rc;
  if (dir == 1 && c->sim2d) {  // zero tendencies (Spatial:572-575)
    // FP64: state and tracers += dt*0 as the reference applies them (no value changes; a
    // -0 becomes +0; tracers held divided between splits are -0 exactly where rho*tracer
    // is); the FP32 form leaves both unchanged
    if (fp32(c)) return AWFL_OK;
    cudaError_t e = launch_add_zero_fp64((double *)d_state, 5, c->cfg.nx, c->cfg.ny, c->cfg.nz, c->hs, c->nsm,
                                         (cudaStream_t)stream);
    if (e == cudaSuccess)
      e = launch_add_zero_fp64(d_tracers, ntracers, c->cfg.nx, c->cfg.ny, c->cfg.nz, c->hs, c->nsm,
                               (cudaStream_t)stream);
    return e == cudaSuccess ? AWFL_OK : cuda_fail(c, e, "split_tracers");
  }
  unsigned long long mask = 0;
  for (int l = 0; l < ntracers; l++)
    if (pos[l]) mask |= 1ull << l;
  const size_t need =
      tracer_scratch_bytes(c->cfg.ord, c->cfg.nx, c->cfg.ny, c->cfg.nz, ntracers, fp32(c) ? 4 : 8);
  rc = ensure_buffer(c, &c->d_trc, &c->trc_bytes, need, "tracer scratch");
  if (rc) return rc;
  cudaError_t e;
  if (fp32(c)) {
    SweepArgs32 A = sweep_args32(c, d_state, nullptr, dt, dir, MODE_APPLY);
    const double dxd = dir == 0 ? c->dx : (dir == 1 ? c->dy : c->dz);
    e = launch_split_tracers32(c->cfg.ord, dir, A, c->d_dens_c, dt, dxd, d_tracers, ntracers, mask,
                               reinterpret_cast<float *>(c->d_trc), io, (cudaStream_t)stream);
  } else {
    SweepArgs A = sweep_args(c, d_state, nullptr, dt, dir, MODE_APPLY);
    e = launch_split_tracers(c->cfg.ord, dir, A, d_tracers, ntracers, mask, c->d_trc, io, (cudaStream_t)stream);
  }
  if (e != cudaSuccess) return cuda_fail(c, e, "split_tracers");
  return AWFL_OK;
}

int awfl_split_tracers(awfl_ctx *c, void *d_state, double *d_tracers, int ntracers, const int *pos, double dt,
                       int dir, void *stream) {
  return split_tracers_io(c, d_state, d_tracers, ntracers, pos, dt, dir, 0, stream);
}

int awfl_step_tracers(awfl_ctx *c, void *d_state, double *d_tracers, int ntracers, const int *pos, double dt,
                      void *stream) {
  if (!c) return AWFL_ERR_ARG;
  // the tracers stay divided by the density from one split to the next (the division the
  // next split would start with is done by the previous one's update); the y split of a
  // sim2d context changes neither state nor tracers, and it is never the last
  for (int spl = 0; spl < 3; spl++) {
    const int dir = c->dimswitch ? spl : 2 - spl;
    const int io = (spl > 0 ? TRC_IN_DIVIDED : 0) | (spl < 2 ? TRC_OUT_DIVIDED : 0);
    int rc = split_tracers_io(c, d_state, d_tracers, ntracers, pos, dt, dir, io, stream);
    if (rc) return rc;
  }
  c->dimswitch = !c->dimswitch;
  return AWFL_OK;
}

int awfl_step_tlm(awfl_ctx *c, void *d_state_tangent, double dt, void *stream) {
  if (!c) return AWFL_ERR_ARG;
  if (c->nslabs > 1) return fail(c, AWFL_ERR_ARG, "the tangent-linear step is not available on a slab");
  if (fp32(c)) return fail(c, AWFL_ERR_ARG, "awfl_step_tlm needs an FP64 context");
  if (bad_ptr(d_state_tangent)) return fail(c, AWFL_ERR_ARG, "state pointer is NULL or misaligned");
  int rc = set_device(c);
  if (rc) return rc;
  for (int spl = 0; spl < 3; spl++) {
    const int dir = c->dimswitch ? spl : 2 - spl;
    if (dir == 1 && c->sim2d) continue;
    SweepArgs A = sweep_args(c, d_state_tangent, nullptr, dt, dir, MODE_APPLY);
    A.plane = state_plane(c);
    cudaError_t e = launch_sweep_tlm(c->cfg.ord, dir, A, (cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(c, e, "step_tlm");
  }
  c->dimswitch = !c->dimswitch;
  return AWFL_OK;
}



namespace {

// The split directions of `nsteps` steps from dimSwitch value ds (sim2d drops Y).
std::vector<int> split_dirs(const awfl_ctx *c, int nsteps, int ds) {
  std::vector<int> dirs;
  for (int n = 0; n < nsteps; n++) {
    for (int spl = 0; spl < 3; spl++) {
      const int dir = ds ? spl : 2 - spl;
      if (dir == 1 && c->sim2d) continue;
      dirs.push_back(dir);
    }
    ds = !ds;
  }
  return dirs;
}

// Device memory (doubles) of awfl_step_adjoint for a window of nsteps steps: the split-
// start states and records of the recorded stretch (the whole window, or one sub-window),
// the sub-window start states, and the reverse scratch.
long adjoint_doubles(const awfl_ctx *c, int nsteps) {
  const long per_step = c->sim2d ? 2L : 3L;
  const long ncell = (long)c->cfg.nx * c->cfg.ny * c->cfg.nz;
  const long nface = (long)(c->cfg.nx + 1) * (c->cfg.ny + 1) * (c->cfg.nz + 1);
  const long rec = (5L * c->ngll + 10L) * ncell;  // per split: level-0 values + edges
  const int m = c->adj_sub > 0 && c->adj_sub < nsteps ? c->adj_sub : nsteps;  // recorded steps
  const long nsub = m > 0 ? (nsteps + m - 1) / m : 0;
  const long nspl = per_step * m;
  const long tape = nspl > 0 ? (nspl + 1) * state_plane(c) + nspl * rec : 0;
  const long starts = nsub > 1 ? (nsub - 1) * state_plane(c) : 0;
  return tape + starts + 10L * nface + 5L * (c->cfg.ord + c->ngll) * ncell;
}

}  // namespace

int awfl_adjoint_tape_bytes(const awfl_ctx *c, int nsteps, long *bytes) {
  if (!c || nsteps < 0 || !bytes) return AWFL_ERR_ARG;
  *bytes = (long)sizeof(double) * adjoint_doubles(c, nsteps);
  return AWFL_OK;
}

int awfl_set_adjoint_subwindow(awfl_ctx *c, int steps) {
  if (!c || steps < 0) return AWFL_ERR_ARG;
  c->adj_sub = steps;
  return AWFL_OK;
}

int awfl_step_adjoint(awfl_ctx *c, const void *d_state_ckpt, void *d_lambda, int nsteps, double dt, void *stream) {
  if (c && c->nslabs > 1) return fail(c, AWFL_ERR_ARG, "the adjoint is not available on a slab");
  if (!c) return AWFL_ERR_ARG;
  if (fp32(c)) return fail(c, AWFL_ERR_ARG, "awfl_step_adjoint needs an FP64 context");
  if (bad_ptr(d_state_ckpt) || bad_ptr(d_lambda)) return fail(c, AWFL_ERR_ARG, "state or lambda pointer is NULL or misaligned");
  if (d_state_ckpt == d_lambda) return fail(c, AWFL_ERR_ARG, "state and lambda must be distinct buffers");
  if (nsteps < 0) return fail(c, AWFL_ERR_ARG, "nsteps must be >= 0");
  if (!(dt > 0.0) || !std::isfinite(dt)) return fail(c, AWFL_ERR_ARG, "dt must be positive and finite");
  int rc = set_device(c);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  const int nx = c->cfg.nx, ny = c->cfg.ny, nz = c->cfg.nz, ord = c->cfg.ord;
  const long plane = state_plane(c);
  const long ncell = (long)nx * ny * nz;
  const long nface = (long)(nx + 1) * (ny + 1) * (nz + 1);
  if (nsteps == 0) {
    cudaError_t e = launch_zero_halo((double *)d_lambda, nx, ny, nz, c->hs, c->nsm, st);
    return e == cudaSuccess ? AWFL_OK : cuda_fail(c, e, "adjoint reverse sweep");
  }
  // Sub-windows of m steps (the whole window when the context's sub-window length is 0 or
  // not shorter): pass 1 steps from the checkpoint with the plain sweep (bit-identical to
  // the recording one) and keeps the state at each sub-window's start; pass 2, last
  // sub-window first, recomputes the sub-window with the recording sweep (split-start
  // states and records) and runs its reverse sweeps, last split first.
  const int m = c->adj_sub > 0 && c->adj_sub < nsteps ? c->adj_sub : nsteps;
  const int nsub = (nsteps + m - 1) / m;
  const long per_step = c->sim2d ? 2L : 3L;
  const long rec = (5L * c->ngll + 10L) * ncell;  // per split: level-0 values + edges
  const long mspl = per_step * m;
  rc = ensure_buffer(c, &c->d_tape, &c->tape_bytes,
                     sizeof(double) * (size_t)((mspl + 1) * plane + mspl * rec + (long)(nsub - 1) * plane),
                     "adjoint tape");
  if (rc) return rc;
  rc = ensure_buffer(c, &c->d_adj, &c->adj_bytes, sizeof(double) * (size_t)(10 * nface + 5L * (ord + c->ngll) * ncell),
                     "adjoint scratch");
  if (rc) return rc;
  double *states = c->d_tape, *recs = c->d_tape + (mspl + 1) * plane;
  double *starts = recs + mspl * rec;  // sub-window g >= 1 starts at starts + (g-1)*plane
  auto start_of = [&](int g) -> const double * {
    return g == 0 ? (const double *)d_state_ckpt : starts + (long)(g - 1) * plane;
  };
  // dimSwitch at each sub-window start (the context's value is the checkpoint's)
  std::vector<int> ds_at(nsub);
  {
    int ds = c->dimswitch;
    for (int g = 0; g < nsub; g++) {
      ds_at[g] = ds;
      if (m % 2) ds = !ds;
    }
  }
  cudaError_t e = cudaSuccess;
  // pass 1: the sub-window start states
  for (int g = 1; g < nsub && e == cudaSuccess; g++) {
    double *dst = starts + (long)(g - 1) * plane;
    e = cudaMemcpyAsync(dst, start_of(g - 1), sizeof(double) * plane, cudaMemcpyDeviceToDevice, st);
    const std::vector<int> dirs = split_dirs(c, m, ds_at[g - 1]);
    for (size_t s = 0; s < dirs.size() && e == cudaSuccess; s++)
      e = launch_sweep_fp64(ord, dirs[s], sweep_args(c, dst, nullptr, dt, dirs[s], MODE_APPLY), st);
  }
  if (e != cudaSuccess) return cuda_fail(c, e, "adjoint forward recomputation");
  // pass 2: each sub-window recorded and reversed, last first
  for (int g = nsub - 1; g >= 0 && e == cudaSuccess; g--) {
    const int mg = (g == nsub - 1) ? nsteps - g * m : m;
    const std::vector<int> dirs = split_dirs(c, mg, ds_at[g]);
    const long nspl = (long)dirs.size();
    if (nspl == 0) continue;
    // forward recomputation: state s = state at the start of split s (s = 0..nspl), and the
    // record of split s (its level-0 values and edges) taken by the recording sweep
    e = cudaMemcpyAsync(states, start_of(g), sizeof(double) * plane, cudaMemcpyDeviceToDevice, st);
    for (long s = 0; s < nspl && e == cudaSuccess; s++) {
      double *dst = states + (s + 1) * plane;
      e = cudaMemcpyAsync(dst, states + s * plane, sizeof(double) * plane, cudaMemcpyDeviceToDevice, st);
      if (e == cudaSuccess)
        e = launch_sweep_rec(ord, dirs[s], sweep_args(c, dst, recs + s * rec, dt, dirs[s], MODE_APPLY), st);
    }
    if (e != cudaSuccess) return cuda_fail(c, e, "adjoint forward recomputation");
    // reverse sweeps, last split first
    for (long s = nspl - 1; s >= 0 && e == cudaSuccess; s--) {
      const int dir = dirs[s];
      adj::SplitArgs A{};
      A.state = states + s * plane;
      A.q0 = recs + s * rec;
      A.edges = A.q0 + 5L * c->ngll * ncell;
      A.lq = c->d_adj;
      A.ls = c->d_adj + 10 * nface;
      A.lq0 = A.ls + 5L * ord * ncell;
      A.lam = (double *)d_lambda;
      A.nx = nx; A.ny = ny; A.nz = nz; A.hs = c->hs;
      A.sim2d = c->sim2d;
      A.ca.nz = nz;
      A.ca.bc = dir == 0 ? c->cfg.bc_x : (dir == 1 ? c->cfg.bc_y : c->cfg.bc_z);
      A.ca.weno_s = c->cfg.weno_scalars; A.ca.weno_w = c->cfg.weno_winds;
      A.ca.dxd = dir == 0 ? c->dx : (dir == 1 ? c->dy : c->dz);
      A.ca.dt = dt;
      A.ca.dens_c = c->d_dens_c; A.ca.denstheta_c = c->d_denstheta_c;
      A.ca.dens_g = c->d_dens_g; A.ca.denstheta_g = c->d_denstheta_g; A.ca.pres_g = c->d_pres_g;
      e = launch_adjoint_split(ord, dir, A, 0, c->nsm, st);
    }
  }
  if (e == cudaSuccess) e = launch_zero_halo((double *)d_lambda, nx, ny, nz, c->hs, c->nsm, st);
  if (e != cudaSuccess) return cuda_fail(c, e, "adjoint reverse sweep");
  return AWFL_OK;
}

int awfl_get_tables(const awfl_ctx *c, double *weno_recon, double *coefs_to_gll, double *sten_to_gll, double *deriv,
                    double *idl, double *sigma, double *gll_pts_ord, double *gll_wts_ord, double *gll_pts_ngll,
                    double *gll_wts_ngll) {
  if (!c) return AWFL_ERR_ARG;
  auto cp = [](double *dst, const std::vector<double> &v) {
    if (dst) std::memcpy(dst, v.data(), v.size() * sizeof(double));
  };
  cp(weno_recon, c->recon); cp(coefs_to_gll, c->c2g); cp(sten_to_gll, c->s2g); cp(deriv, c->deriv);
  cp(idl, c->idl);
  if (sigma) *sigma = c->sigma;
  cp(gll_pts_ord, c->pts_ord); cp(gll_wts_ord, c->wts_ord); cp(gll_pts_ngll, c->pts_ngll); cp(gll_wts_ngll, c->wts_ngll);
  return AWFL_OK;
}

int awfl_get_background(const awfl_ctx *c, double *dens_c, double *pres_c, double *theta_c, double *denstheta_c,
                        double *dens_g, double *pres_g, double *theta_g, double *denstheta_g) {
  if (!c) return AWFL_ERR_ARG;
  auto cp = [](double *dst, const std::vector<double> &v) {
    if (dst) std::memcpy(dst, v.data(), v.size() * sizeof(double));
  };
  cp(dens_c, c->dens_c); cp(pres_c, c->pres_c); cp(theta_c, c->theta_c); cp(denstheta_c, c->denstheta_c);
  cp(dens_g, c->dens_g); cp(pres_g, c->pres_g); cp(theta_g, c->theta_g); cp(denstheta_g, c->denstheta_g);
  return AWFL_OK;
}

int awfl_selftest_pow(const void *d_x, double y, void *d_out, long n, int mode, void *stream) {
  if (n < 0 || mode < 0 || mode > 4 || (n > 0 && (bad_ptr(d_x) || bad_ptr(d_out)))) return AWFL_ERR_ARG;
  cudaError_t e = launch_selftest_pow((const double *)d_x, y, (double *)d_out, n, mode, (cudaStream_t)stream);
  return e == cudaSuccess ? AWFL_OK : AWFL_ERR_CUDA;
}

int awfl_measure_fma_peak(int precision, int device, double *tflops) {
  if (!tflops || (precision != AWFL_FP64 && precision != AWFL_FP32 && precision != AWFL_PEAK_FP32_PAIRED))
    return AWFL_ERR_ARG;
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return AWFL_ERR_CUDA;
  int nsm = 148;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) == cudaSuccess) nsm = prop.multiProcessorCount;
  e = run_fma_peak(precision == AWFL_FP64 ? 0 : (precision == AWFL_FP32 ? 1 : 2), nsm, tflops);
  return e == cudaSuccess ? AWFL_OK : AWFL_ERR_CUDA;
}

int awfl_device_alloc(void **d_ptr, long bytes) {
  if (!d_ptr || bytes < 0) return AWFL_ERR_ARG;
  cudaError_t e = cudaMalloc(d_ptr, bytes > 0 ? (size_t)bytes : 1);
  if (e != cudaSuccess) { g_create_error = cudaGetErrorString(e); return AWFL_ERR_NOMEM; }
  return AWFL_OK;
}
int awfl_device_free(void *d_ptr) {
  cudaError_t e = cudaFree(d_ptr);
  return e == cudaSuccess ? AWFL_OK : AWFL_ERR_CUDA;
}
int awfl_copy_h2d(void *d_dst, const void *h_src, long bytes, void *stream) {
  if (bytes < 0) return AWFL_ERR_ARG;
  cudaError_t e = cudaMemcpyAsync(d_dst, h_src, (size_t)bytes, cudaMemcpyHostToDevice, (cudaStream_t)stream);
  return e == cudaSuccess ? AWFL_OK : AWFL_ERR_CUDA;
}
int awfl_copy_d2h(void *h_dst, const void *d_src, long bytes, void *stream) {
  if (bytes < 0) return AWFL_ERR_ARG;
  cudaError_t e = cudaMemcpyAsync(h_dst, d_src, (size_t)bytes, cudaMemcpyDeviceToHost, (cudaStream_t)stream);
  return e == cudaSuccess ? AWFL_OK : AWFL_ERR_CUDA;
}
int awfl_memset_device(void *d_ptr, int value, long bytes, void *stream) {
  if (bytes < 0) return AWFL_ERR_ARG;
  cudaError_t e = cudaMemsetAsync(d_ptr, value, (size_t)bytes, (cudaStream_t)stream);
  return e == cudaSuccess ? AWFL_OK : AWFL_ERR_CUDA;
}
int awfl_stream_synchronize(void *stream) {
  cudaError_t e = cudaStreamSynchronize((cudaStream_t)stream);
  return e == cudaSuccess ? AWFL_OK : AWFL_ERR_CUDA;
}
int awfl_device_synchronize(void) {
  cudaError_t e = cudaDeviceSynchronize();
  return e == cudaSuccess ? AWFL_OK : AWFL_ERR_CUDA;
}

}  // extern "C"
