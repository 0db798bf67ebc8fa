/* CPU restatement (test oracle) of the AWFL Euler-3D ADER/WENO finite-volume step.
 *
 * TEST INFRASTRUCTURE ONLY -- see awfl_oracle.h. Every function names the reference
 * lines it restates; arithmetic is written in the reference's evaluation order so that,
 * compiled without FMA contraction against the same libm, results are bit-identical.
 *
 * Reference files (paths within mrnorman/awflCloud):
 *   Spatial_euler3d_cons_expl_cart_fv_Agrid.h  ("Spatial" below)
 *   WenoLimiter.h, TransformMatrices.h, Temporal_ader.h, Profiles.h, phys_params.h
 */
#define _GNU_SOURCE
#include "awfl_oracle.h"

#include <math.h>
#include <tgmath.h> /* pow/exp/sqrt/... follow the argument type (oreal) */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../awflcloud_b200/csrc/awfl_tables.h"

/* ORACLE_CR_POW builds the variant whose pow calls in the time step and the CFL time step
 * are correctly rounded (awfl_pow_cr.h) instead of glibc's, like the GPU FP64 kernels.
 * The hydrostatic profiles (init-time, computed on the host by the library as well) keep
 * glibc's pow/exp. */
#if defined(ORACLE_CR_POW) && defined(ORACLE_LONG_DOUBLE)
#error "ORACLE_CR_POW is a double-precision variant"
#endif
#ifdef ORACLE_CR_POW
#include "awfl_pow_cr.h"
#define OPOW(x, y) awfl_test_pow_cr((x), (y))
#define OEXP(x) awfl_test_exp_cr((x))
#else
#define OPOW(x, y) pow((x), (y))
#define OEXP(x) exp((x))
#endif

#ifndef ORACLE_ORD
#define ORACLE_ORD 5
#endif
#ifndef ORACLE_NGLL
#define ORACLE_NGLL 3
#endif

#define ORD ORACLE_ORD
#define NGLL ORACLE_NGLL
#define NADER NGLL
#define HS ((ORD - 1) / 2)
#define NUMSTATE 5

#if ORD == 5
#define TBL(name) name##_o5
#define TV_LO_N AWFL_TV_LO_O5_NTERM
#define TV_HI_N AWFL_TV_HI_O5_NTERM
#define TVS(part, name) awfl_tv_##part##_o5_##name
#elif ORD == 9
#define TBL(name) name##_o9
#define TV_LO_N AWFL_TV_LO_O9_NTERM
#define TV_HI_N AWFL_TV_HI_O9_NTERM
#define TVS(part, name) awfl_tv_##part##_o9_##name
#else
#error "oracle supports ORD 5 (NGLL 3) and ORD 9 (NGLL 5)"
#endif

/* phys_params.h:4-10 */
static const oreal GRAV = 9.81;
static const oreal CP = 1004.;
static const oreal RD = 287.;
static const oreal P0 = 1.0e5;
static const oreal C0 = 27.5629410929725921310572974482;
static const oreal GAMMA = 1.40027894002789400278940027894;

enum { idR = 0, idU = 1, idV = 2, idW = 3, idT = 4 };
/* BC_GIVEN (x only; test infrastructure for slab decompositions): the caller supplies the
 * x halos (no halo fill); the line ends' edge values are copied as at a wall. */
enum { BC_PERIODIC = 0, BC_WALL = 1, BC_GIVEN = 2 };
enum { DATA_THERMAL = 1, DATA_COLLISION = 2, DATA_STRAKA = 3, DATA_IGW = 4 };

struct oracle_ctx {
  int nx, ny, nz;
  oreal xlen, ylen, zlen, dx, dy, dz;
  int bc[3];
  int weno_scalars, weno_winds, sim2d, data_spec, dimswitch;
  /* tables (Spatial:274-315) */
  oreal recon[ORD][ORD][ORD];
  oreal c2g[ORD][NGLL];   /* coefs_to_gll(col=s, row=ii) */
  oreal s2g[ORD][NGLL];   /* sten_to_gll */
  oreal deriv[NGLL][NGLL];
  oreal idl[HS + 2];
  oreal sigma;
  oreal pts_ord[ORD], wts_ord[ORD], pts_ngll[NGLL], wts_ngll[NGLL];
  /* hydrostatic background (Spatial:371-425) */
  oreal *hyDensCells, *hyPressureCells, *hyThetaCells, *hyDensThetaCells; /* nz+2hs */
  oreal *hyDensGLL, *hyPressureGLL, *hyThetaGLL, *hyDensThetaGLL;         /* nz*ngll */
  /* scratch (Spatial:327-330) */
  oreal *limits; /* (5,2,nz+1,ny+1,nx+1) */
  oreal *flux;   /* (5,nz+1,ny+1,nx+1) */
  /* tracer transport (Spatial:624-627, 760-809, 826-835, 891-935, 948-955 and the y/z
   * equivalents): set by oracle_tracer_step for the duration of one call */
  int ntr;
  const int *trpos;
  oreal *tr, *ttend;        /* (ntr,nz+2hs,ny+2hs,nx+2hs), (ntr,nz,ny,nx) */
  oreal *tlimits, *tflux, *tflux_lim;  /* (ntr,2,...), (ntr,...), (ntr,...) */
  /* faces of the last tracer split whose limited flux differs from the one computed with
   * every face read unscaled (the serial order's chains; oracle_limiter_chained_faces) */
  long lim_chained;
};

/* ---------------------------------------------------------------- indexing */
static inline long sidx(const oracle_ctx *c, int l, int k, int j, int i) {
  return (((long)l * (c->nz + 2 * HS) + k) * (c->ny + 2 * HS) + j) * (c->nx + 2 * HS) + i;
}
static inline long tidx(const oracle_ctx *c, int l, int k, int j, int i) {
  return (((long)l * c->nz + k) * c->ny + j) * c->nx + i;
}
static inline long lidx(const oracle_ctx *c, int l, int side, int k, int j, int i) {
  return ((((long)l * 2 + side) * (c->nz + 1) + k) * (c->ny + 1) + j) * (c->nx + 1) + i;
}
static inline long fidx(const oracle_ctx *c, int l, int k, int j, int i) {
  return (((long)l * (c->nz + 1) + k) * (c->ny + 1) + j) * (c->nx + 1) + i;
}

static inline oreal dmax(oreal a, oreal b) { return a > b ? a : b; }
static inline oreal dmin(oreal a, oreal b) { return a < b ? a : b; }

/* ---------------------------------------------------------------- WENO */
/* TransformMatrices::coefs_to_tv: ordered quadratic form, c*(a*a) or (c*a_m)*a_q. */
static oreal tv_eval(const oreal *a, int nterm, const int *m, const int *q, const double *cf) {
  oreal r = 0;
  for (int t = 0; t < nterm; t++) {
    oreal term = (m[t] == q[t]) ? cf[t] * (a[q[t]] * a[q[t]]) : cf[t] * a[m[t]] * a[q[t]];
    r = (t == 0) ? term : r + term;
  }
  return r;
}
static oreal tv_lo(const oreal *a) {
  return tv_eval(a, TV_LO_N, TVS(lo, m), TVS(lo, q), TVS(lo, c));
}
static oreal tv_hi(const oreal *a) {
  return tv_eval(a, TV_HI_N, TVS(hi, m), TVS(hi, q), TVS(hi, c));
}

/* WenoLimiter.h:20-25 */
static void convexify(oreal *wts) {
  oreal sum = 0.;
  const oreal eps = 1.0e-20;
  for (int i = 0; i < HS + 2; i++) sum += wts[i];
  for (int i = 0; i < HS + 2; i++) wts[i] /= (sum + eps);
}

/* WenoLimiter.h:12-17 */
static void map_weights(const oreal *idl, oreal *wts) {
  for (int i = 0; i < HS + 2; i++) {
    wts[i] = wts[i] * (idl[i] + idl[i] * idl[i] - 3. * idl[i] * wts[i] + wts[i] * wts[i]) /
             (idl[i] * idl[i] + wts[i] * (1. - 2. * idl[i]));
  }
}

/* WenoLimiter.h:28-90 (ord 5 and 9 rows) */
static void weno_set_ideal_sigma(oreal *idl, oreal *sigma) {
#if ORD == 5
  *sigma = 0.73564225445964;
  idl[0] = 1.; idl[1] = 73.564225445964; idl[2] = 1.; idl[3] = 1584.89319246111;
#else
  *sigma = 0.0288539981181442;
  idl[0] = 1.; idl[1] = 2.15766927997459; idl[2] = 2.40224886796286;
  idl[3] = 2.15766927997459; idl[4] = 1.; idl[5] = 1136.12697719888;
#endif
  convexify(idl);
}

/* WenoLimiter.h:93-172 */
static void weno_coefs(const oracle_ctx *c, const oreal *u, oreal *aw) {
  oreal tv[HS + 2], wts[HS + 2], a[HS + 2][ORD], lotmp[HS + 1], hitmp[ORD];
  const oreal eps = 1.0e-20;
  for (int j = 0; j < HS + 2; j++)
    for (int i = 0; i < ORD; i++) a[j][i] = 0.;
  for (int i = 0; i < HS + 1; i++)
    for (int ii = 0; ii < HS + 1; ii++)
      for (int s = 0; s < HS + 1; s++) a[i][ii] += c->recon[i][s][ii] * u[i + s];
  for (int ii = 0; ii < ORD; ii++)
    for (int s = 0; s < ORD; s++) a[HS + 1][ii] += c->recon[HS + 1][s][ii] * u[s];
  for (int i = 0; i < HS + 1; i++)
    for (int ii = 0; ii < HS + 1; ii++) a[HS + 1][ii] -= c->idl[i] * a[i][ii];
  for (int ii = 0; ii < ORD; ii++) a[HS + 1][ii] /= c->idl[HS + 1];
  for (int i = 0; i < HS + 1; i++) {
    for (int ii = 0; ii < HS + 1; ii++) lotmp[ii] = a[i][ii];
    tv[i] = tv_lo(lotmp);
  }
  for (int ii = 0; ii < ORD; ii++) hitmp[ii] = a[HS + 1][ii];
  tv[HS + 1] = tv_hi(hitmp);
  oreal lo_avg = 0.;
  for (int i = 0; i < HS + 1; i++) lo_avg += tv[i];
  lo_avg /= HS + 1;
  tv[HS + 1] = lo_avg + (tv[HS + 1] - lo_avg) * c->sigma;
  for (int i = 0; i < HS + 2; i++) wts[i] = c->idl[i] / (tv[i] * tv[i] + eps);
  convexify(wts);
  map_weights(c->idl, wts);
  convexify(wts);
  for (int i = 0; i < ORD; i++) aw[i] = 0.;
  for (int i = 0; i < HS + 2; i++)
    for (int ii = 0; ii < ORD; ii++) aw[ii] += wts[i] * a[i][ii];
}

/* Spatial:1800-1833 */
static void reconstruct_gll(const oracle_ctx *c, const oreal *stencil, oreal *out, int doweno) {
  if (doweno) {
    oreal wc[ORD];
    weno_coefs(c, stencil, wc);
    for (int ii = 0; ii < NGLL; ii++) {
      oreal tmp = 0;
      for (int s = 0; s < ORD; s++) tmp += c->c2g[s][ii] * wc[s];
      out[ii] = tmp;
    }
  } else {
    for (int ii = 0; ii < NGLL; ii++) {
      oreal tmp = 0;
      for (int s = 0; s < ORD; s++) tmp += c->s2g[s][ii] * stencil[s];
      out[ii] = tmp;
    }
  }
}

/* ---------------------------------------------------------------- ADER */
/* Per-cell ADER arrays: q[v][kt][ii] for v = r, ru, rv, rw, rt; f[x][kt][ii] for the
 * four normal-momentum flux products (normal*u, normal*v, normal*w, normal*t)/r, and the
 * (rho*theta)^gamma series g. dir selects the normal momentum (1+dir). */
typedef struct {
  oreal q[NUMSTATE][NADER][NGLL];
  oreal f[4][NADER][NGLL];
  oreal g[NADER][NGLL];
  oreal src[NADER][NGLL];
} ader_t;

/* diffTransformEulerConsX/Y/Z (Spatial:1837-1916, 1920-2000, 2004-2091). */
static void diff_transform(const oracle_ctx *c, ader_t *A, int dir, oreal dxd, int k) {
  const int nm = 1 + dir; /* normal momentum index */
  for (int kt = 1; kt < NADER; kt++)
    for (int ii = 0; ii < NGLL; ii++) {
      for (int x = 0; x < 4; x++) A->f[x][kt][ii] = 0;
      A->g[kt][ii] = 0;
    }
  for (int kt = 0; kt < NADER - 1; kt++) {
    for (int ii = 0; ii < NGLL; ii++) {
      oreal dq[NUMSTATE] = {0, 0, 0, 0, 0};
      for (int s = 0; s < NGLL; s++) {
        oreal D = c->deriv[s][ii];
        dq[idR] += D * (A->q[nm][kt][s]);
        for (int v = 1; v <= 3; v++) {
          if (v == nm) {
            if (dir == 2 && kt == 0) {
              dq[v] += D * (A->f[v - 1][kt][s] + C0 * A->g[kt][s] - c->hyPressureGLL[k * NGLL + s]);
            } else if (kt == 0) {
              dq[v] += D * (A->f[v - 1][kt][s] + C0 * A->g[kt][s]);
            } else {
              dq[v] += D * (A->f[v - 1][kt][s] + C0 * A->g[kt][s] / 2);
            }
          } else {
            dq[v] += D * (A->f[v - 1][kt][s]);
          }
        }
        dq[idT] += D * (A->f[3][kt][s]);
      }
      for (int v = 0; v < NUMSTATE; v++) A->q[v][kt + 1][ii] = -dq[v] / dxd / (kt + 1.);
      if (dir == 2) {
        A->q[idW][kt + 1][ii] = -dq[idW] / dxd / (kt + 1.) + A->src[kt][ii] / (kt + 1.);
        if (c->bc[2] == BC_WALL) {
          if (k == c->nz - 1) A->q[idW][kt + 1][NGLL - 1] = 0;
          if (k == 0) A->q[idW][kt + 1][0] = 0;
        }
        A->src[kt + 1][ii] = -A->q[idR][kt + 1][ii] * GRAV;
      }
    }
    for (int ii = 0; ii < NGLL; ii++) {
      oreal tot[4] = {0, 0, 0, 0};
      for (int ir = 0; ir <= kt + 1; ir++) {
        for (int x = 0; x < 4; x++) {
          int xv = x + 1; /* u->ru(1), v->rv(2), w->rw(3), t->rt(4) */
          tot[x] += A->q[nm][ir][ii] * A->q[xv][kt + 1 - ir][ii] - A->q[idR][ir][ii] * A->f[x][kt + 1 - ir][ii];
        }
      }
      for (int x = 0; x < 4; x++) A->f[x][kt + 1][ii] = tot[x] / A->q[idR][0][ii];
      oreal tg = 0;
      for (int ir = 0; ir <= kt; ir++) {
        tg += (kt + 1. - ir) * (GAMMA * A->g[ir][ii] * A->q[idT][kt + 1 - ir][ii] -
                                A->q[idT][ir][ii] * A->g[kt + 1 - ir][ii]);
      }
      A->g[kt + 1][ii] = (GAMMA * A->g[0][ii] * A->q[idT][kt + 1][ii] + tg / (kt + 1.)) / A->q[idT][0][ii];
    }
  }
  for (int kt = 1; kt < NADER; kt++)
    for (int ii = 0; ii < NGLL; ii++) A->g[kt][ii] /= 2;
}

/* diffTransformTracer (Spatial:2095-2125): rho*tracer time derivatives from the density
 * and normal-momentum series r, ru; rut is the normal tracer flux series. */
static void diff_transform_tracer(const oracle_ctx *c, oreal r[NADER][NGLL], oreal ru[NADER][NGLL],
                                  oreal rt[NADER][NGLL], oreal rut[NADER][NGLL], oreal dxd) {
  for (int kt = 1; kt < NADER; kt++)
    for (int ii = 0; ii < NGLL; ii++) rut[kt][ii] = 0;
  for (int kt = 0; kt < NADER - 1; kt++) {
    for (int ii = 0; ii < NGLL; ii++) {
      oreal df_dx = 0;
      for (int s = 0; s < NGLL; s++) df_dx += c->deriv[s][ii] * rut[kt][s];
      rt[kt + 1][ii] = -df_dx / dxd / (kt + 1.);
    }
    for (int ii = 0; ii < NGLL; ii++) {
      oreal tot = 0;
      for (int ir = 0; ir <= kt + 1; ir++) tot += ru[ir][ii] * rt[kt + 1 - ir][ii] - r[ir][ii] * rut[kt + 1 - ir][ii];
      rut[kt + 1][ii] = tot / r[0][ii];
    }
  }
}

/* compute_timeAvg_edges (Spatial:2153-2177): edge points only. */
static void time_avg_edges(oreal dts[NADER][NGLL], oreal dt) {
  oreal dtmult = dt;
  for (int kt = 1; kt < NADER; kt++) {
    dts[0][0] += dts[kt][0] * dtmult / (kt + 1.);
    dts[0][NGLL - 1] += dts[kt][NGLL - 1] * dtmult / (kt + 1.);
    dtmult *= dt;
  }
}

/* compute_timeAvg (Spatial:2130-2138): all points. */
static void time_avg_full(oreal dts[NADER][NGLL], oreal dt) {
  oreal dtmult = dt;
  for (int kt = 1; kt < NADER; kt++) {
    for (int ii = 0; ii < NGLL; ii++) dts[0][ii] += dts[kt][ii] * dtmult / (kt + 1.);
    dtmult *= dt;
  }
}

/* ---------------------------------------------------------------- halos */
/* Spatial:631-662 (x), 994-1025 (y), 1351-1382 (z). */
static void fill_halos(const oracle_ctx *c, oreal *st, int dir) {
  const int nx = c->nx, ny = c->ny, nz = c->nz;
  if (dir == 0 && c->bc[0] == BC_GIVEN) return;
  if (dir == 0) {
#pragma omp parallel for collapse(2)
    for (int k = 0; k < nz; k++)
      for (int j = 0; j < ny; j++)
        for (int ii = 0; ii < HS; ii++)
          for (int l = 0; l < NUMSTATE; l++) {
            if (c->bc[0] == BC_PERIODIC) {
              st[sidx(c, l, HS + k, HS + j, ii)] = st[sidx(c, l, HS + k, HS + j, nx + ii)];
              st[sidx(c, l, HS + k, HS + j, HS + nx + ii)] = st[sidx(c, l, HS + k, HS + j, HS + ii)];
            } else if (l == idU) {
              st[sidx(c, l, HS + k, HS + j, ii)] = 0;
              st[sidx(c, l, HS + k, HS + j, HS + nx + ii)] = 0;
            } else {
              st[sidx(c, l, HS + k, HS + j, ii)] = st[sidx(c, l, HS + k, HS + j, HS)];
              st[sidx(c, l, HS + k, HS + j, HS + nx + ii)] = st[sidx(c, l, HS + k, HS + j, HS + nx - 1)];
            }
          }
  } else if (dir == 1) {
#pragma omp parallel for collapse(2)
    for (int k = 0; k < nz; k++)
      for (int i = 0; i < nx; i++)
        for (int jj = 0; jj < HS; jj++)
          for (int l = 0; l < NUMSTATE; l++) {
            if (c->bc[1] == BC_PERIODIC) {
              st[sidx(c, l, HS + k, jj, HS + i)] = st[sidx(c, l, HS + k, ny + jj, HS + i)];
              st[sidx(c, l, HS + k, HS + ny + jj, HS + i)] = st[sidx(c, l, HS + k, HS + jj, HS + i)];
            } else if (l == idV) {
              st[sidx(c, l, HS + k, jj, HS + i)] = 0;
              st[sidx(c, l, HS + k, HS + ny + jj, HS + i)] = 0;
            } else {
              st[sidx(c, l, HS + k, jj, HS + i)] = st[sidx(c, l, HS + k, HS, HS + i)];
              st[sidx(c, l, HS + k, HS + ny + jj, HS + i)] = st[sidx(c, l, HS + k, HS + ny - 1, HS + i)];
            }
          }
  } else {
#pragma omp parallel for collapse(2)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++)
        for (int kk = 0; kk < HS; kk++)
          for (int l = 0; l < NUMSTATE; l++) {
            if (c->bc[2] == BC_PERIODIC) {
              st[sidx(c, l, kk, HS + j, HS + i)] = st[sidx(c, l, nz + kk, HS + j, HS + i)];
              st[sidx(c, l, HS + nz + kk, HS + j, HS + i)] = st[sidx(c, l, HS + kk, HS + j, HS + i)];
            } else if (l == idW) {
              st[sidx(c, l, kk, HS + j, HS + i)] = 0;
              st[sidx(c, l, HS + nz + kk, HS + j, HS + i)] = 0;
            } else {
              st[sidx(c, l, kk, HS + j, HS + i)] = st[sidx(c, l, HS, HS + j, HS + i)];
              st[sidx(c, l, HS + nz + kk, HS + j, HS + i)] = st[sidx(c, l, HS + nz - 1, HS + j, HS + i)];
            }
          }
  }
}

/* ---------------------------------------------------------------- tendencies */
/* computeTendenciesX/Y/Z (Spatial:598-957, 961-1311, 1315-1697), one direction. */
void oracle_compute_tendencies_dir(oracle_ctx *c, oreal *st, oreal *tend, oreal dt, int dir) {
  const int nx = c->nx, ny = c->ny, nz = c->nz;
  const int nm = 1 + dir;
  const oreal dxd = dir == 0 ? c->dx : (dir == 1 ? c->dy : c->dz);
  const int bc = c->bc[dir];
  const int ntr = c->ntr;
  oreal *tr = c->tr;

  /* tracers /= (rho' + rho_h) inside the domain (Spatial:624-627, 985-990, 1342-1347) */
#pragma omp parallel for collapse(3)
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++)
        for (int l = 0; l < ntr; l++)
          tr[sidx(c, l, HS + k, HS + j, HS + i)] /= (st[sidx(c, idR, HS + k, HS + j, HS + i)] + c->hyDensCells[HS + k]);

  fill_halos(c, st, dir);
  /* tracer halos: periodic copy, or the edge cell at a wall (Spatial:637-642, 655-660 and
   * the y/z equivalents) */
  if (ntr > 0) {
    const int n = dir == 0 ? nx : (dir == 1 ? ny : nz);
    const int na = dir == 2 ? ny : nz, nb = dir == 0 ? ny : nx;
    for (int a = 0; a < na; a++)
      for (int b2 = 0; b2 < nb; b2++)
        for (int h = 0; h < HS; h++)
          for (int l = 0; l < ntr; l++) {
#define TIDX(p) (dir == 0 ? sidx(c, l, HS + a, HS + b2, (p)) : (dir == 1 ? sidx(c, l, HS + a, (p), HS + b2) : sidx(c, l, (p), HS + a, HS + b2)))
            if (bc == BC_PERIODIC) {
              tr[TIDX(h)] = tr[TIDX(n + h)];
              tr[TIDX(HS + n + h)] = tr[TIDX(HS + h)];
            } else {
              tr[TIDX(h)] = tr[TIDX(HS)];
              tr[TIDX(HS + n + h)] = tr[TIDX(HS + n - 1)];
            }
#undef TIDX
          }
  }

  /* Reconstruct + ADER + time average; store cell-edge states (K2). */
#pragma omp parallel for collapse(3)
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++) {
        ader_t A;
        oreal stencil[ORD];
        for (int v = 0; v < NUMSTATE; v++) {
          for (int s = 0; s < ORD; s++) {
            if (dir == 0) stencil[s] = st[sidx(c, v, HS + k, HS + j, i + s)];
            else if (dir == 1) stencil[s] = st[sidx(c, v, HS + k, j + s, HS + i)];
            else stencil[s] = st[sidx(c, v, k + s, HS + j, HS + i)];
          }
          int doweno = (v == idR || v == idT) ? c->weno_scalars : c->weno_winds;
          reconstruct_gll(c, stencil, A.q[v][0], doweno);
          if (v == idR) {
            for (int ii = 0; ii < NGLL; ii++)
              A.q[idR][0][ii] += (dir == 2) ? c->hyDensGLL[k * NGLL + ii] : c->hyDensCells[HS + k];
          }
          if (dir == 2 && v == idW && bc == BC_WALL) { /* Spatial:1413-1416 */
            if (k == nz - 1) A.q[idW][0][NGLL - 1] = 0;
            if (k == 0) A.q[idW][0][0] = 0;
          }
          if (v == idT) {
            for (int ii = 0; ii < NGLL; ii++)
              A.q[idT][0][ii] += (dir == 2) ? c->hyDensThetaGLL[k * NGLL + ii] : c->hyDensThetaCells[HS + k];
          }
        }
        /* level-0 flux products (Spatial:704-715 and per-direction equivalents) */
        oreal srcfill = 0;
        for (int ii = 0; ii < NGLL; ii++) {
          oreal r = A.q[idR][0][ii];
          oreal u = A.q[idU][0][ii] / r;
          oreal v = A.q[idV][0][ii] / r;
          oreal w = A.q[idW][0][ii] / r;
          oreal t = A.q[idT][0][ii] / r;
          oreal vn = nm == 1 ? u : (nm == 2 ? v : w);
          A.f[0][0][ii] = r * vn * u;
          A.f[1][0][ii] = r * vn * v;
          A.f[2][0][ii] = r * vn * w;
          A.f[3][0][ii] = r * vn * t;
          A.g[0][ii] = OPOW(r * t, GAMMA);
          if (dir == 2) srcfill = -(A.q[idR][0][ii] - c->hyDensGLL[k * NGLL + ii]) * GRAV;
        }
        if (dir == 2) { /* SArray scalar assignment fills every entry (Spatial:1439) */
          for (int kt = 0; kt < NADER; kt++)
            for (int ii = 0; ii < NGLL; ii++) A.src[kt][ii] = srcfill;
        }
        if (NADER > 1) diff_transform(c, &A, dir, dxd, k);
        oreal rser[NADER][NGLL], ruser[NADER][NGLL]; /* "still exist and are computed" (Spatial:762) */
        memcpy(rser, A.q[idR], sizeof rser);
        memcpy(ruser, A.q[nm], sizeof ruser);
        for (int v = 0; v < NUMSTATE; v++) time_avg_edges(A.q[v], dt);
        int kl = k, jl = j, il = i, kr = k, jr = j, ir = i;
        if (dir == 0) ir = i + 1;
        else if (dir == 1) jr = j + 1;
        else kr = k + 1;
        /* tracers (Spatial:760-809, 1123-1170, 1500-1548) */
        for (int l = 0; l < ntr; l++) {
          oreal rt[NADER][NGLL], rut[NADER][NGLL], sten[ORD];
          for (int s2 = 0; s2 < ORD; s2++) {
            if (dir == 0) sten[s2] = tr[sidx(c, l, HS + k, HS + j, i + s2)];
            else if (dir == 1) sten[s2] = tr[sidx(c, l, HS + k, j + s2, HS + i)];
            else sten[s2] = tr[sidx(c, l, k + s2, HS + j, HS + i)];
          }
          reconstruct_gll(c, sten, rt[0], c->weno_scalars);
          for (int ii = 0; ii < NGLL; ii++) rt[0][ii] *= rser[0][ii];
          if (c->trpos[l])
            for (int ii = 0; ii < NGLL; ii++) rt[0][ii] = dmax(0., rt[0][ii]);
          for (int ii = 0; ii < NGLL; ii++) rut[0][ii] = rt[0][ii] * ruser[0][ii] / rser[0][ii];
          if (NADER > 1) diff_transform_tracer(c, rser, ruser, rt, rut, dxd);
          time_avg_edges(rt, dt);
          if (c->trpos[l]) {
            rt[0][0] = dmax(0., rt[0][0]);
            rt[0][NGLL - 1] = dmax(0., rt[0][NGLL - 1]);
          }
          c->tlimits[lidx(c, l, 1, kl, jl, il)] = rt[0][0];
          c->tlimits[lidx(c, l, 0, kr, jr, ir)] = rt[0][NGLL - 1];
        }
        for (int v = 0; v < NUMSTATE; v++) {
          c->limits[lidx(c, v, 1, kl, jl, il)] = A.q[v][0][0];
          c->limits[lidx(c, v, 0, kr, jr, ir)] = A.q[v][0][NGLL - 1];
        }
        if (dir == 2) { /* gravity source (Spatial:1459-1499) */
          time_avg_full(A.src, dt);
          oreal src_avg = 0;
          for (int ii = 0; ii < NGLL; ii++) src_avg += A.src[0][ii] * c->wts_ngll[ii];
          tend[tidx(c, idR, k, j, i)] = 0;
          tend[tidx(c, idU, k, j, i)] = 0;
          tend[tidx(c, idV, k, j, i)] = 0;
          tend[tidx(c, idW, k, j, i)] = src_avg;
          tend[tidx(c, idT, k, j, i)] = 0;
        }
      }

  /* Edge-value BCs (K3: Spatial:816-837, 1176-1197, 1557-1578). */
  {
    int n = dir == 0 ? nx : (dir == 1 ? ny : nz);
    int na = dir == 2 ? ny : nz;   /* outer */
    int nb = dir == 0 ? ny : nx;   /* inner */
    for (int a = 0; a < na; a++)
      for (int b = 0; b < nb; b++)
        for (int l = 0; l < NUMSTATE; l++) {
          long i0, in, i0s1, ins0;
#define LIM(side, f) (dir == 0 ? lidx(c, l, side, a, b, f) : (dir == 1 ? lidx(c, l, side, a, f, b) : lidx(c, l, side, f, a, b)))
          i0 = LIM(0, 0); in = LIM(1, n); i0s1 = LIM(1, 0); ins0 = LIM(0, n);
#undef LIM
          if (bc == BC_PERIODIC) {
            c->limits[i0] = c->limits[ins0];
            c->limits[in] = c->limits[i0s1];
          } else {
            c->limits[i0] = c->limits[i0s1];
            c->limits[in] = c->limits[ins0];
          }
        }
    for (int a = 0; a < na; a++) /* tracers (Spatial:826-835, 1186-1195, 1567-1576) */
      for (int b = 0; b < nb; b++)
        for (int l = 0; l < ntr; l++) {
#define LIM(side, f) (dir == 0 ? lidx(c, l, side, a, b, f) : (dir == 1 ? lidx(c, l, side, a, f, b) : lidx(c, l, side, f, a, b)))
          long i0 = LIM(0, 0), in = LIM(1, n), i0s1 = LIM(1, 0), ins0 = LIM(0, n);
#undef LIM
          if (bc == BC_PERIODIC) {
            c->tlimits[i0] = c->tlimits[ins0];
            c->tlimits[in] = c->tlimits[i0s1];
          } else {
            c->tlimits[i0] = c->tlimits[i0s1];
            c->tlimits[in] = c->tlimits[ins0];
          }
        }
  }

  /* Upwind Riemann flux (K4: Spatial:842-902, 1202-1260, 1583-1644). */
  {
    int ek = nz + (dir == 2), ej = ny + (dir == 1), ei = nx + (dir == 0);
#pragma omp parallel for collapse(3)
    for (int k = 0; k < ek; k++)
      for (int j = 0; j < ej; j++)
        for (int i = 0; i < ei; i++) {
          oreal qL[5], qR[5];
          for (int l = 0; l < 5; l++) {
            qL[l] = c->limits[lidx(c, l, 0, k, j, i)];
            qR[l] = c->limits[lidx(c, l, 1, k, j, i)];
          }
          oreal r, vel[3], t;
          r = 0.5 * (qL[0] + qR[0]);
          if (dir == 1) { /* y: averages are NOT divided by density (Spatial:1210-1214) */
            vel[0] = 0.5 * (qL[1] + qR[1]);
            vel[1] = 0.5 * (qL[2] + qR[2]);
            vel[2] = 0.5 * (qL[3] + qR[3]);
            t = 0.5 * (qL[4] + qR[4]);
          } else {
            vel[0] = 0.5 * (qL[1] / qL[0] + qR[1] / qR[0]);
            vel[1] = 0.5 * (qL[2] / qL[0] + qR[2] / qR[0]);
            vel[2] = 0.5 * (qL[3] / qL[0] + qR[3] / qR[0]);
            t = 0.5 * (qL[4] / qL[0] + qR[4] / qR[0]);
          }
          oreal p = C0 * OPOW(r * t, GAMMA);
          oreal cs2 = GAMMA * p / r;
          oreal cs = sqrt(cs2);
          /* tangential indices in increasing order */
          int ta = dir == 0 ? 1 : 0, tb = dir == 2 ? 1 : 2; /* velocity slots */
          oreal vn = vel[dir], va = vel[ta], vb = vel[tb];
          int qn = 1 + dir, qa = 1 + ta, qb = 1 + tb;
          oreal w1, w2, w3;
          if (vn > 0) {
            w1 = qL[0] - qL[4] / t;
            w2 = qL[qa] - va * qL[4] / t;
            w3 = qL[qb] - vb * qL[4] / t;
          } else {
            w1 = qR[0] - qR[4] / t;
            w2 = qR[qa] - va * qR[4] / t;
            w3 = qR[qb] - vb * qR[4] / t;
          }
          oreal w5 = vn * qR[0] / (2 * cs) - qR[qn] / (2 * cs) + qR[4] / (2 * t);
          oreal w6 = -vn * qL[0] / (2 * cs) + qL[qn] / (2 * cs) + qL[4] / (2 * t);
          oreal q[5];
          q[0] = w1 + w5 + w6;
          q[qn] = vn * w1 + (vn - cs) * w5 + (vn + cs) * w6;
          q[qa] = w2 + va * w5 + va * w6;
          q[qb] = w3 + vb * w5 + vb * w6;
          q[4] = t * w5 + t * w6;
          oreal F[5];
          F[0] = q[qn];
          F[qn] = q[qn] * q[qn] / q[0] + C0 * OPOW(q[4], GAMMA);
          F[qa] = q[qn] * q[qa] / q[0];
          F[qb] = q[qn] * q[qb] / q[0];
          F[4] = q[qn] * q[4] / q[0];
          if (dir == 2) {
            if (k < nz) F[idW] -= c->hyPressureGLL[k * NGLL + 0];
            if (k == nz) F[idW] -= c->hyPressureGLL[(nz - 1) * NGLL + NGLL - 1];
          }
          for (int l = 0; l < 5; l++) c->flux[fidx(c, l, k, j, i)] = F[l];
          /* upwind tracer fluxes (Spatial:891-901, 1249-1259, 1633-1643) */
          for (int l = 0; l < ntr; l++) {
            if (vn > 0) c->tflux[fidx(c, l, k, j, i)] = F[0] * c->tlimits[lidx(c, l, 0, k, j, i)] / qL[0];
            else c->tflux[fidx(c, l, k, j, i)] = F[0] * c->tlimits[lidx(c, l, 1, k, j, i)] / qR[0];
          }
        }
  }

  /* Positivity limiter of the tracer fluxes (Spatial:904-935, 1262-1293, 1646-1677), in the
   * reference's serial loop order: the reference scales tracerFlux in place inside a
   * parallel_for whose other iterations read it, so its one defined result is the serial
   * one (its CPU build run in order), which this restates: along each line the faces are
   * visited in increasing order and each is scaled in place by its upwind cell's factor,
   * computed from that cell's two faces as they stand at that moment (the face behind
   * already scaled, the face itself and the ones ahead not yet). The y branch for v < 0
   * reads the faces along y (the reference indexes tracerFlux(tr,k,j,ind_j) there,
   * Spatial:1285-1286, with j and i swapped), and a periodic z wraps like x and y (the
   * reference reads outside the array there). */
  if (ntr > 0) {
    const int n = dir == 0 ? nx : (dir == 1 ? ny : nz);
    const oreal eps = 1.e-10;
    const int la = dir == 2 ? ny : nz, lb = dir == 0 ? ny : nx;  /* the lines: (la, lb) */
    const long nflim = (long)ntr * (nz + 1) * (ny + 1) * (nx + 1);
    memcpy(c->tflux_lim, c->tflux, sizeof(oreal) * (size_t)nflim);
#pragma omp parallel for collapse(3)
    for (int l = 0; l < ntr; l++)
      for (int a = 0; a < la; a++)
        for (int b = 0; b < lb; b++) {
          if (!c->trpos[l]) continue;
          /* the line's cell at index p along dir */
#define LK(p) (dir == 2 ? (p) : a)
#define LJ(p) (dir == 1 ? (p) : (dir == 2 ? a : b))
#define LI(p) (dir == 0 ? (p) : b)
          oreal *TF = c->tflux_lim;
          long chained = 0;
          for (int f = 0; f <= n; f++) {
            const long fi = fidx(c, l, LK(f), LJ(f), LI(f));
            const oreal un = 0.5 * (c->limits[lidx(c, nm, 0, LK(f), LJ(f), LI(f))] +
                                    c->limits[lidx(c, nm, 1, LK(f), LJ(f), LI(f))]);
            int ind;
            if (un > 0) { ind = f - 1; if (ind == -1) ind = n - 1; }
            else if (un < 0) { ind = f; if (ind == n) ind = 0; }
            else continue;
            const oreal f1 = dmin(TF[fidx(c, l, LK(ind), LJ(ind), LI(ind))], 0.);
            const oreal f2 = dmax(TF[fidx(c, l, LK(ind + 1), LJ(ind + 1), LI(ind + 1))], 0.);
            const oreal fluxOut = dt * (f2 - f1) / dxd;
            const oreal dens = st[sidx(c, idR, HS + LK(ind), HS + LJ(ind), HS + LI(ind))] + c->hyDensCells[HS + LK(ind)];
            const oreal q = tr[sidx(c, l, HS + LK(ind), HS + LJ(ind), HS + LI(ind))];
            TF[fi] *= dmin(1., q * dens / (fluxOut + eps));
            /* the same face with both of its cell's faces read unscaled */
            const oreal u1 = dmin(c->tflux[fidx(c, l, LK(ind), LJ(ind), LI(ind))], 0.);
            const oreal u2 = dmax(c->tflux[fidx(c, l, LK(ind + 1), LJ(ind + 1), LI(ind + 1))], 0.);
            if (!(c->tflux[fi] * dmin(1., q * dens / (dt * (u2 - u1) / dxd + eps)) == TF[fi])) chained++;
          }
#pragma omp atomic
          c->lim_chained += chained;
#undef LK
#undef LJ
#undef LI
        }
  }

  /* Flux divergence (K5: Spatial:940-956, 1298-1310, 1680-1696). */
#pragma omp parallel for collapse(3)
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++)
        for (int l = 0; l < NUMSTATE; l++) {
          oreal fl = c->flux[fidx(c, l, k, j, i)];
          oreal fr = dir == 0 ? c->flux[fidx(c, l, k, j, i + 1)]
                    : (dir == 1 ? c->flux[fidx(c, l, k, j + 1, i)] : c->flux[fidx(c, l, k + 1, j, i)]);
          long ti = tidx(c, l, k, j, i);
          if (dir == 0) {
            tend[ti] = (c->sim2d && l == idV) ? 0 : -(fr - fl) / dxd;
          } else if (dir == 1) {
            tend[ti] = -(fr - fl) / dxd;
          } else {
            if (c->sim2d && l == idV) tend[ti] = 0;
            else tend[ti] += -(fr - fl) / dxd;
          }
        }
  /* tracer tendencies, and density multiplied back onto the tracers (Spatial:948-955,
   * 1302-1309, 1688-1695) */
#pragma omp parallel for collapse(3)
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++)
        for (int l = 0; l < ntr; l++) {
          oreal fl = c->tflux_lim[fidx(c, l, k, j, i)];
          oreal fr = dir == 0 ? c->tflux_lim[fidx(c, l, k, j, i + 1)]
                    : (dir == 1 ? c->tflux_lim[fidx(c, l, k, j + 1, i)] : c->tflux_lim[fidx(c, l, k + 1, j, i)]);
          c->ttend[tidx(c, l, k, j, i)] = -(fr - fl) / dxd;
          tr[sidx(c, l, HS + k, HS + j, HS + i)] *= (st[sidx(c, idR, HS + k, HS + j, HS + i)] + c->hyDensCells[HS + k]);
        }
}

/* One split of Temporal_ader::timeStep (Temporal_ader.h:50-70) with the tracer transport
 * compiled in: computeTendencies along dir on state and tracers, then state += dt*tend
 * and tracers += dt*tracerTend. sim2d's y split zeroes both tendencies (Spatial:572-575). */
void oracle_split_tracers(oracle_ctx *c, oreal *st, oreal *tr, int ntr, const int *pos, oreal dt, int dir) {
  const long nf = (long)(c->nz + 1) * (c->ny + 1) * (c->nx + 1);
  const long ncell = (long)c->nz * c->ny * c->nx;
  oreal *tend = (oreal *)calloc((size_t)NUMSTATE * ncell, sizeof(oreal));
  c->ntr = ntr;
  c->trpos = pos;
  c->tr = tr;
  c->lim_chained = 0;
  c->ttend = (oreal *)calloc((size_t)ntr * ncell + 1, sizeof(oreal));
  c->tlimits = (oreal *)calloc((size_t)ntr * 2 * nf + 1, sizeof(oreal));
  c->tflux = (oreal *)calloc((size_t)ntr * nf + 1, sizeof(oreal));
  c->tflux_lim = (oreal *)calloc((size_t)ntr * nf + 1, sizeof(oreal));
  if (!(dir == 1 && c->sim2d)) oracle_compute_tendencies_dir(c, st, tend, dt, dir);
  oracle_apply(c, st, tend, dt);
  for (int k = 0; k < c->nz; k++)
    for (int j = 0; j < c->ny; j++)
      for (int i = 0; i < c->nx; i++)
        for (int l = 0; l < ntr; l++)
          tr[sidx(c, l, HS + k, HS + j, HS + i)] += dt * c->ttend[tidx(c, l, k, j, i)];
  free(tend); free(c->ttend); free(c->tlimits); free(c->tflux); free(c->tflux_lim);
  c->ntr = 0; c->trpos = NULL; c->tr = NULL; c->ttend = NULL;
  c->tlimits = c->tflux = c->tflux_lim = NULL;
}

/* Temporal_ader::timeStep (Temporal_ader.h:48-72) with the tracer transport compiled in:
 * oracle_split_tracers for each split in the dimSwitch order. */
void oracle_time_step_tracers(oracle_ctx *c, oreal *st, oreal *tr, int ntr, const int *pos, oreal dt) {
  for (int split = 0; split < 3; split++) {
    const int dir = c->dimswitch ? split : 2 - split;
    oracle_split_tracers(c, st, tr, ntr, pos, dt, dir);
  }
  c->dimswitch = !c->dimswitch;
}

/* Spatial:565-594 */
void oracle_compute_tendencies(oracle_ctx *c, oreal *st, oreal *tend, oreal dt, int split) {
  int dir;
  if (c->dimswitch) dir = split == 0 ? 0 : (split == 1 ? 1 : 2);
  else dir = split == 0 ? 2 : (split == 1 ? 1 : 0);
  if (dir == 1 && c->sim2d) {
    long n = (long)NUMSTATE * c->nz * c->ny * c->nx;
    for (long i = 0; i < n; i++) tend[i] = 0.;
  } else {
    oracle_compute_tendencies_dir(c, st, tend, dt, dir);
  }
  if (split == 2) c->dimswitch = !c->dimswitch;
}

/* Temporal_ader.h:63-65 */
void oracle_apply(const oracle_ctx *c, oreal *st, const oreal *tend, oreal dt) {
#pragma omp parallel for collapse(3)
  for (int l = 0; l < NUMSTATE; l++)
    for (int k = 0; k < c->nz; k++)
      for (int j = 0; j < c->ny; j++)
        for (int i = 0; i < c->nx; i++)
          st[sidx(c, l, HS + k, HS + j, HS + i)] += dt * tend[tidx(c, l, k, j, i)];
}

/* Temporal_ader.h:48-72 */
void oracle_time_step(oracle_ctx *c, oreal *st, oreal dt) {
  long n = (long)NUMSTATE * c->nz * c->ny * c->nx;
  oreal *tend = (oreal *)calloc((size_t)n, sizeof(oreal));
  for (int spl = 0; spl < 3; spl++) {
    oracle_compute_tendencies(c, st, tend, dt, spl);
    oracle_apply(c, st, tend, dt);
  }
  free(tend);
}

int oracle_get_dimswitch(const oracle_ctx *c) { return c->dimswitch; }
long oracle_limiter_chained_faces(const oracle_ctx *c) { return c->lim_chained; }
void oracle_set_dimswitch(oracle_ctx *c, int v) { c->dimswitch = v != 0; }

/* ---------------------------------------------------------------- CFL */
/* Spatial:159-187 */
oreal oracle_compute_dt(const oracle_ctx *c, const oreal *st, oreal cfl) {
  oreal best = INFINITY;
  int first = 1;
  for (int k = 0; k < c->nz; k++)
    for (int j = 0; j < c->ny; j++)
      for (int i = 0; i < c->nx; i++) {
        oreal r = st[sidx(c, idR, HS + k, HS + j, HS + i)] + c->hyDensCells[HS + k];
        oreal u = st[sidx(c, idU, HS + k, HS + j, HS + i)] / r;
        oreal v = st[sidx(c, idV, HS + k, HS + j, HS + i)] / r;
        oreal w = st[sidx(c, idW, HS + k, HS + j, HS + i)] / r;
        oreal t = (st[sidx(c, idT, HS + k, HS + j, HS + i)] + c->hyDensThetaCells[HS + k]) / r;
        oreal p = C0 * OPOW(r * t, GAMMA);
        oreal cs = sqrt(GAMMA * p / r);
        oreal udt = cfl * c->dx / dmax(fabs(u - cs), fabs(u + cs));
        oreal vdt = cfl * c->dy / dmax(fabs(v - cs), fabs(v + cs));
        oreal wdt = cfl * c->dz / dmax(fabs(w - cs), fabs(w + cs));
        oreal d = dmin(dmin(udt, vdt), wdt);
        if (first || d < best) { best = d; first = 0; }
      }
  return best;
}

/* ---------------------------------------------------------------- profiles */
/* Profiles.h:8-46 */
static oreal const_theta_density(oreal t0, oreal z) {
  oreal exner = 1. - GRAV * z / (CP * t0);
  oreal p = pow(exner, CP / RD) * P0;
  oreal rt = pow(p / C0, 1. / GAMMA);
  return rt / t0;
}
static oreal const_theta_pressure(oreal t0, oreal z) {
  oreal r = const_theta_density(t0, z);
  return C0 * pow(r * t0, GAMMA);
}
static oreal bvf_pot_temp(oreal t0, oreal bvf, oreal z) { return t0 * exp(bvf * bvf * z / GRAV); }
static oreal bvf_density(oreal t0, oreal bvf, oreal z) {
  oreal t = bvf_pot_temp(t0, bvf, z);
  oreal exner = 1. - GRAV * GRAV / (CP * bvf * bvf) * (t - t0) / (t * t0);
  oreal p = pow(exner, CP / RD) * P0;
  oreal rt = pow(p / C0, 1. / GAMMA);
  return rt / t;
}
static oreal bvf_pressure(oreal t0, oreal bvf, oreal z) {
  oreal t = bvf_pot_temp(t0, bvf, z);
  oreal r = bvf_density(t0, bvf, z);
  return C0 * pow(r * t, GAMMA);
}
/* Profiles.h:49-81 */
static oreal ellipsoid_linear(oreal x, oreal y, oreal z, oreal x0, oreal y0, oreal z0,
                               oreal xrad, oreal yrad, oreal zrad, oreal amp) {
  oreal xn = (x - x0) / xrad, yn = (y - y0) / yrad, zn = (z - z0) / zrad;
  oreal dist = sqrt(xn * xn + yn * yn + zn * zn);
  return amp * dmax(1. - dist, 0.);
}
static oreal ellipsoid_cosine(oreal x, oreal y, oreal z, oreal x0, oreal y0, oreal z0,
                               oreal xrad, oreal yrad, oreal zrad, oreal amp, oreal pwr) {
  oreal val = 0;
  oreal xn = (x - x0) / xrad, yn = (y - y0) / yrad, zn = (z - z0) / zrad;
  oreal dist = sqrt(xn * xn + yn * yn + zn * zn);
  if (dist <= 1.) val = amp * pow((cos(M_PI * dist) + 1) / 2, pwr);
  return val;
}
static oreal igw_prof(oreal x, oreal y, oreal z, oreal x0, oreal y0, oreal hr, oreal zlen, oreal amp) {
  oreal xn = (x - x0) / hr, yn = (y - y0) / hr;
  return amp * sin(M_PI * z / zlen) / sqrt(1 + xn * xn + yn * yn);
}

/* Spatial:371-425 */
static void init_background(oracle_ctx *c) {
  const int nz = c->nz;
  for (int k = 0; k < nz + 2 * HS; k++) {
    c->hyDensCells[k] = 0; c->hyPressureCells[k] = 0; c->hyThetaCells[k] = 0; c->hyDensThetaCells[k] = 0;
    for (int kk = 0; kk < ORD; kk++) {
      oreal zloc = (k - HS + 0.5) * c->dz + c->pts_ord[kk] * c->dz;
      oreal th, rh, ph;
      if (c->data_spec == DATA_IGW) {
        const oreal bvf = 0.01, t0 = 300;
        th = bvf_pot_temp(t0, bvf, zloc); rh = bvf_density(t0, bvf, zloc); ph = bvf_pressure(t0, bvf, zloc);
      } else {
        th = 300; rh = const_theta_density(th, zloc); ph = const_theta_pressure(th, zloc);
      }
      oreal wt = c->wts_ord[kk];
      c->hyDensCells[k] += rh * wt;
      c->hyThetaCells[k] += th * wt;
      c->hyDensThetaCells[k] += rh * th * wt;
      c->hyPressureCells[k] += ph * wt;
    }
  }
  for (int k = 0; k < nz; k++)
    for (int kk = 0; kk < NGLL; kk++) {
      oreal zloc = (k + 0.5) * c->dz + c->pts_ngll[kk] * c->dz;
      oreal th, rh, ph;
      if (c->data_spec == DATA_IGW) {
        const oreal bvf = 0.01, t0 = 300;
        th = bvf_pot_temp(t0, bvf, zloc); rh = bvf_density(t0, bvf, zloc); ph = bvf_pressure(t0, bvf, zloc);
      } else {
        th = 300; rh = const_theta_density(th, zloc); ph = const_theta_pressure(th, zloc);
      }
      c->hyDensGLL[k * NGLL + kk] = rh;
      c->hyThetaGLL[k * NGLL + kk] = th;
      c->hyDensThetaGLL[k * NGLL + kk] = rh * th;
      c->hyPressureGLL[k * NGLL + kk] = ph;
    }
}

/* Spatial:428-485 */
void oracle_init_state(oracle_ctx *c, oreal *st) {
  const int nx = c->nx, ny = c->ny, nz = c->nz;
#pragma omp parallel for collapse(3)
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++) {
        for (int l = 0; l < NUMSTATE; l++) st[sidx(c, l, HS + k, HS + j, HS + i)] = 0;
        for (int kk = 0; kk < ORD; kk++)
          for (int jj = 0; jj < ORD; jj++)
            for (int ii = 0; ii < ORD; ii++) {
              oreal zloc = (k + 0.5) * c->dz + c->pts_ord[kk] * c->dz;
              oreal yloc = c->sim2d ? c->ylen / 2 : (j + 0.5) * c->dy + c->pts_ord[jj] * c->dy;
              oreal xloc = (i + 0.5) * c->dx + c->pts_ord[ii] * c->dx;
              oreal wt = c->wts_ord[kk] * c->wts_ord[jj] * c->wts_ord[ii];
              long it = sidx(c, idT, HS + k, HS + j, HS + i);
              if (c->data_spec == DATA_THERMAL) {
                oreal th = 300, rh = const_theta_density(th, zloc);
                oreal tp = ellipsoid_linear(xloc, yloc, zloc, c->xlen / 2, c->ylen / 2, 2000, 2000, 2000, 2000, 2);
                oreal t = th + tp;
                st[it] += (rh * t - rh * th) * wt;
              } else if (c->data_spec == DATA_COLLISION) {
                oreal th = 300, rh = const_theta_density(th, zloc);
                oreal tp = ellipsoid_linear(xloc, yloc, zloc, c->xlen / 2, c->ylen / 2, 2000, 2000, 2000, 2000, 20);
                tp += ellipsoid_linear(xloc, yloc, zloc, c->xlen / 2, c->ylen / 2, 8000, 2000, 2000, 2000, -20);
                oreal t = th + tp;
                st[it] += (rh * t - rh * th) * wt;
              } else if (c->data_spec == DATA_STRAKA) {
                oreal th = 300, rh = const_theta_density(th, zloc);
                oreal tp = ellipsoid_cosine(xloc, yloc, zloc, c->xlen / 2, c->ylen / 2, 3000, 4000, 2000, 2000, -15, 1);
                oreal t = th + tp;
                st[it] += (rh * t - rh * th) * wt;
              } else if (c->data_spec == DATA_IGW) {
                if (c->sim2d) yloc = c->ylen / 3;
                const oreal t0 = 300, bvf = 0.01;
                oreal rh = bvf_density(t0, bvf, zloc);
                oreal th = bvf_pot_temp(t0, bvf, zloc);
                oreal tp = igw_prof(xloc, yloc, zloc, c->xlen / 3, c->ylen / 3, 5000, c->zlen, 0.01);
                oreal t = th + tp;
                st[it] += (rh * t - rh * th) * wt;
                st[sidx(c, idU, HS + k, HS + j, HS + i)] += 20 * rh * wt;
                if (!c->sim2d) st[sidx(c, idV, HS + k, HS + j, HS + i)] += 20 * rh * wt;
              }
            }
      }
}

/* Spatial:505-560 (initTracers; not under NO_TRACERS, so the reference runs it): ord^3 GLL
 * quadrature of rho_h * tval per tracer, with tval = 1 (tracer 0), the 2 K linear ellipsoid
 * of radius 2 km at (xlen/2, ylen/2, 2 km) (tracer 1) or the block indicator of
 * k in [nz/10, 3nz/10), i in [4nx/10, 6nx/10), j in [4ny/10, 6ny/10) unless sim2d (tracer 2)
 * (integer division); any further tracer is zero. tr: (ntr, nz+2hs, ny+2hs, nx+2hs), only
 * the interior is written. */
void oracle_init_tracers(oracle_ctx *c, oreal *tr, int ntr) {
  const int nx = c->nx, ny = c->ny, nz = c->nz;
#pragma omp parallel for collapse(3)
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++)
        for (int l = 0; l < ntr; l++) {
          long it = sidx(c, l, HS + k, HS + j, HS + i);
          tr[it] = 0;
          for (int kk = 0; kk < ORD; kk++)
            for (int jj = 0; jj < ORD; jj++)
              for (int ii = 0; ii < ORD; ii++) {
                oreal zloc = (k + 0.5) * c->dz + c->pts_ord[kk] * c->dz;
                oreal yloc = c->sim2d ? c->ylen / 2 : (j + 0.5) * c->dy + c->pts_ord[jj] * c->dy;
                oreal xloc = (i + 0.5) * c->dx + c->pts_ord[ii] * c->dx;
                oreal wt = c->wts_ord[kk] * c->wts_ord[jj] * c->wts_ord[ii];
                oreal th = 300, rh = const_theta_density(th, zloc);
                if (l == 0) {
                  tr[it] += rh * 1 * wt;
                } else if (l == 1) {
                  oreal tval = ellipsoid_linear(xloc, yloc, zloc, c->xlen / 2, c->ylen / 2, 2000, 2000, 2000, 2000, 2);
                  tr[it] += rh * tval * wt;
                } else if (l == 2) {
                  int inside = k >= 1 * nz / 10 && k < 3 * nz / 10 && i >= 4 * nx / 10 && i < 6 * nx / 10;
                  if (!c->sim2d) inside = inside && j >= 4 * ny / 10 && j < 6 * ny / 10;
                  oreal tval = inside ? 1 : 0;
                  tr[it] += rh * tval * wt;
                }
              }
        }
}

void oracle_set_bubble(oracle_ctx *c, oreal *st, int shape, oreal x0, oreal y0, oreal z0,
                       oreal xrad, oreal yrad, oreal zrad, oreal amp, oreal pwr) {
  const int nx = c->nx, ny = c->ny, nz = c->nz;
#pragma omp parallel for collapse(3)
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++) {
        for (int l = 0; l < NUMSTATE; l++) st[sidx(c, l, HS + k, HS + j, HS + i)] = 0;
        for (int kk = 0; kk < ORD; kk++)
          for (int jj = 0; jj < ORD; jj++)
            for (int ii = 0; ii < ORD; ii++) {
              oreal zloc = (k + 0.5) * c->dz + c->pts_ord[kk] * c->dz;
              oreal yloc = c->sim2d ? c->ylen / 2 : (j + 0.5) * c->dy + c->pts_ord[jj] * c->dy;
              oreal xloc = (i + 0.5) * c->dx + c->pts_ord[ii] * c->dx;
              oreal wt = c->wts_ord[kk] * c->wts_ord[jj] * c->wts_ord[ii];
              oreal th = 300, rh = const_theta_density(th, zloc);
              oreal tp = shape == 0 ? ellipsoid_linear(xloc, yloc, zloc, x0, y0, z0, xrad, yrad, zrad, amp)
                                     : ellipsoid_cosine(xloc, yloc, zloc, x0, y0, z0, xrad, yrad, zrad, amp, pwr);
              oreal t = th + tp;
              st[sidx(c, idT, HS + k, HS + j, HS + i)] += (rh * t - rh * th) * wt;
            }
      }
}

static inline uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ULL;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
  return x ^ (x >> 31);
}

void oracle_add_theta_noise(oracle_ctx *c, oreal *st, unsigned long long seed, oreal amp) {
  for (int k = 0; k < c->nz; k++)
    for (int j = 0; j < c->ny; j++)
      for (int i = 0; i < c->nx; i++) {
        uint64_t idx = ((uint64_t)k * c->ny + j) * c->nx + i;
        oreal u = (oreal)(splitmix64(seed * 0x100000001B3ULL + idx) >> 11) * (1.0 / 9007199254740992.0);
        oreal n = (2.0 * u - 1.0) * amp;
        st[sidx(c, idT, HS + k, HS + j, HS + i)] += c->hyDensCells[HS + k] * n;
      }
}

/* ---------------------------------------------------------------- setup */
static void copy_tab(oreal *dst, const double *src, int n) {
  for (int i = 0; i < n; i++) dst[i] = src[i];
}

/* matmul_cr: C(col,row) = sum_k A(k,row) * B(col,k), k ascending. */
static void matmul_cr(const oreal *A, int K, int R, const oreal *B, int C, oreal *out) {
  for (int cc = 0; cc < C; cc++)
    for (int r = 0; r < R; r++) {
      oreal tmp = 0;
      for (int k = 0; k < K; k++) tmp += A[k * R + r] * B[cc * K + k];
      out[cc * R + r] = tmp;
    }
}

/* Grid spacing set directly (a slab of a larger grid keeps the whole grid's dx). */
void oracle_set_spacing(oracle_ctx *c, oreal dx, oreal dy, oreal dz) {
  c->dx = dx; c->dy = dy; c->dz = dz;
}

oracle_ctx *oracle_create(int nx, int ny, int nz, oreal xlen, oreal ylen, oreal zlen,
                          int bc_x, int bc_y, int bc_z, int weno_scalars, int weno_winds,
                          int data_spec) {
  oracle_ctx *c = (oracle_ctx *)calloc(1, sizeof(oracle_ctx));
  c->nx = nx; c->ny = ny; c->nz = nz;
  c->xlen = xlen; c->ylen = ylen; c->zlen = zlen;
  c->bc[0] = bc_x; c->bc[1] = bc_y; c->bc[2] = bc_z;
  c->weno_scalars = weno_scalars; c->weno_winds = weno_winds;
  c->sim2d = ny == 1;
  c->data_spec = data_spec;
  c->dimswitch = 1;
  c->dx = xlen / nx; c->dy = ylen / ny; c->dz = zlen / nz;
  /* Spatial:274-315 (the generated tables are doubles; copied element by element so that
   * the long-double variant holds the same values) */
  copy_tab((oreal *)c->recon, TBL(awfl_weno_recon), ORD * ORD * ORD);
  copy_tab((oreal *)c->c2g, TBL(awfl_coefs_to_gll_lower), ORD * NGLL);
  {
    oreal a[ORD * NGLL], b[ORD * ORD];
    copy_tab(a, TBL(awfl_coefs_to_gll_lower), ORD * NGLL);
    copy_tab(b, TBL(awfl_sten_to_coefs), ORD * ORD);
    matmul_cr(a, ORD, NGLL, b, ORD, (oreal *)c->s2g);
  }
  {
    oreal tmp[NGLL * NGLL], d[NGLL * NGLL], g2c[NGLL * NGLL], c2g[NGLL * NGLL];
#if ORD == 5
    copy_tab(d, awfl_coefs_to_deriv_n3_o5, NGLL * NGLL);
    copy_tab(g2c, awfl_gll_to_coefs_n3_o5, NGLL * NGLL);
    copy_tab(c2g, awfl_coefs_to_gll_n3_o5, NGLL * NGLL);
#else
    copy_tab(d, awfl_coefs_to_deriv_n5_o9, NGLL * NGLL);
    copy_tab(g2c, awfl_gll_to_coefs_n5_o9, NGLL * NGLL);
    copy_tab(c2g, awfl_coefs_to_gll_n5_o9, NGLL * NGLL);
#endif
    matmul_cr(d, NGLL, NGLL, g2c, NGLL, tmp);
    matmul_cr(c2g, NGLL, NGLL, tmp, NGLL, (oreal *)c->deriv);
  }
  copy_tab(c->pts_ord, TBL(awfl_gll_pts_ord), ORD);
  copy_tab(c->wts_ord, TBL(awfl_gll_wts_ord), ORD);
  copy_tab(c->pts_ngll, TBL(awfl_gll_pts_ngll), NGLL);
  copy_tab(c->wts_ngll, TBL(awfl_gll_wts_ngll), NGLL);
  weno_set_ideal_sigma(c->idl, &c->sigma);

  int nzc = nz + 2 * HS;
  c->hyDensCells = (oreal *)calloc(nzc, sizeof(oreal));
  c->hyPressureCells = (oreal *)calloc(nzc, sizeof(oreal));
  c->hyThetaCells = (oreal *)calloc(nzc, sizeof(oreal));
  c->hyDensThetaCells = (oreal *)calloc(nzc, sizeof(oreal));
  c->hyDensGLL = (oreal *)calloc((size_t)nz * NGLL, sizeof(oreal));
  c->hyPressureGLL = (oreal *)calloc((size_t)nz * NGLL, sizeof(oreal));
  c->hyThetaGLL = (oreal *)calloc((size_t)nz * NGLL, sizeof(oreal));
  c->hyDensThetaGLL = (oreal *)calloc((size_t)nz * NGLL, sizeof(oreal));
  c->limits = (oreal *)calloc((size_t)5 * 2 * (nz + 1) * (ny + 1) * (nx + 1), sizeof(oreal));
  c->flux = (oreal *)calloc((size_t)5 * (nz + 1) * (ny + 1) * (nx + 1), sizeof(oreal));
  init_background(c);
  return c;
}

void oracle_destroy(oracle_ctx *c) {
  if (!c) return;
  free(c->hyDensCells); free(c->hyPressureCells); free(c->hyThetaCells); free(c->hyDensThetaCells);
  free(c->hyDensGLL); free(c->hyPressureGLL); free(c->hyThetaGLL); free(c->hyDensThetaGLL);
  free(c->limits); free(c->flux);
  free(c);
}

int oracle_ord(void) { return ORD; }
int oracle_ngll(void) { return NGLL; }
int oracle_hs(void) { return HS; }
long oracle_state_size(const oracle_ctx *c) {
  return (long)NUMSTATE * (c->nz + 2 * HS) * (c->ny + 2 * HS) * (c->nx + 2 * HS);
}

void oracle_get_tables(const oracle_ctx *c, oreal *s2g, oreal *deriv, oreal *idl, oreal *sigma) {
  memcpy(s2g, c->s2g, sizeof(c->s2g));
  memcpy(deriv, c->deriv, sizeof(c->deriv));
  memcpy(idl, c->idl, sizeof(c->idl));
  *sigma = c->sigma;
}

void oracle_get_background(const oracle_ctx *c, oreal *dens_c, oreal *pres_c, oreal *theta_c,
                           oreal *denstheta_c, oreal *dens_g, oreal *pres_g, oreal *theta_g,
                           oreal *denstheta_g) {
  int nzc = c->nz + 2 * HS;
  memcpy(dens_c, c->hyDensCells, nzc * sizeof(oreal));
  memcpy(pres_c, c->hyPressureCells, nzc * sizeof(oreal));
  memcpy(theta_c, c->hyThetaCells, nzc * sizeof(oreal));
  memcpy(denstheta_c, c->hyDensThetaCells, nzc * sizeof(oreal));
  memcpy(dens_g, c->hyDensGLL, (size_t)c->nz * NGLL * sizeof(oreal));
  memcpy(pres_g, c->hyPressureGLL, (size_t)c->nz * NGLL * sizeof(oreal));
  memcpy(theta_g, c->hyThetaGLL, (size_t)c->nz * NGLL * sizeof(oreal));
  memcpy(denstheta_g, c->hyDensThetaGLL, (size_t)c->nz * NGLL * sizeof(oreal));
}

oreal oracle_coefs_to_tv(const oreal *a, int n) {
  if (n == HS + 1) return tv_lo(a);
  return tv_hi(a);
}

void oracle_weno_coefs(const oracle_ctx *c, const oreal *stencil, oreal *coefs_out) {
  weno_coefs(c, stencil, coefs_out);
}
