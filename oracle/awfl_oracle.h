/* CPU restatement (test oracle) of the AWFL Euler-3D ADER/WENO finite-volume step.
 *
 * TEST INFRASTRUCTURE ONLY: used by tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline leg as the checker. The shipped library never links or calls it.
 *
 * Parity pin: every function is checked bit-for-bit against the reference's own code
 * (oracle/_ref, the unmodified reference headers built on project-written stand-ins for
 * the absent YAKL/yaml-cpp/netCDF dependencies) through the fixtures in tests/golden/.
 *
 * Compile-time order: ORACLE_ORD / ORACLE_NGLL (5/3 or 9/5), like the reference's
 * ORD/NGLL macros (const.h:21-27). FP64, compiled without FMA contraction (or the
 * long-double variant, see oreal below).
 */
#ifndef AWFL_ORACLE_H
#define AWFL_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* The arithmetic type: oreal (the parity oracle), or long oreal (x87 80-bit) when built
 * with ORACLE_LONG_DOUBLE -- the same restatement evaluated with 11 more bits, used only as
 * a finite-difference reference for the discrete adjoint. */
#ifdef ORACLE_LONG_DOUBLE
typedef long double oreal;
#else
typedef double oreal;
#endif

typedef struct oracle_ctx oracle_ctx;

/* bc: 0 periodic, 1 wall. data_spec: 1 thermal, 2 collision, 3 straka, 4 igw
 * (Spatial_euler3d_cons_expl_cart_fv_Agrid.h:75-78). */
oracle_ctx *oracle_create(int nx, int ny, int nz, oreal xlen, oreal ylen, oreal zlen,
                          int bc_x, int bc_y, int bc_z, int weno_scalars, int weno_winds,
                          int data_spec);
/* Grid spacing set directly (a slab of a larger grid keeps the whole grid's dx). */
void oracle_set_spacing(oracle_ctx *c, oreal dx, oreal dy, oreal dz);
void oracle_destroy(oracle_ctx *c);
int oracle_ord(void);
int oracle_ngll(void);
int oracle_hs(void);
long oracle_state_size(const oracle_ctx *c);

/* Hydrostatic background + reference initial data (Spatial...h:345-485). */
void oracle_init_state(oracle_ctx *c, oreal *state);
/* Bubble replacing the theta perturbation (shape 0 linear, 1 cosine) and seeded noise. */
void oracle_set_bubble(oracle_ctx *c, oreal *state, int shape, oreal x0, oreal y0,
                       oreal z0, oreal xrad, oreal yrad, oreal zrad, oreal amp, oreal pwr);
void oracle_add_theta_noise(oracle_ctx *c, oreal *state, unsigned long long seed, oreal amp);
/* Spatial::initTracers (Spatial...h:505-560): the driver's three tracers (uniform, theta
 * replica, block) as rho_h-weighted GLL cell averages; tracers beyond the third are zero.
 * tracers: (ntr, nz+2hs, ny+2hs, nx+2hs), interior written. */
void oracle_init_tracers(oracle_ctx *c, oreal *tracers, int ntr);

/* CFL time step (Spatial...h:159-187), NOT cached here. */
oreal oracle_compute_dt(const oracle_ctx *c, const oreal *state, oreal cfl);

/* One directional split: halo fill (in place on state) + tendencies (5,nz,ny,nx).
 * dir: 0 = x, 1 = y, 2 = z. */
void oracle_compute_tendencies_dir(oracle_ctx *c, oreal *state, oreal *tend, oreal dt, int dir);
/* computeTendencies(split) with the reference's dimSwitch alternation (Spatial...h:565-594). */
void oracle_compute_tendencies(oracle_ctx *c, oreal *state, oreal *tend, oreal dt, int split);
/* state(l,hs+k,hs+j,hs+i) += dt * tend(l,k,j,i)  (Temporal_ader.h:63-65). */
void oracle_apply(const oracle_ctx *c, oreal *state, const oreal *tend, oreal dt);
/* One full time step: 3 splits (Temporal_ader.h:48-72). */
void oracle_time_step(oracle_ctx *c, oreal *state, oreal dt);
/* The same step with the reference's tracer transport compiled in (its code under
 * #ifndef NO_TRACERS, Spatial...h:624-955 and the y/z equivalents; the reference itself
 * defines NO_TRACERS, Spatial...h:10). tracers: (ntr, nz+2hs, ny+2hs, nx+2hs) rho*q;
 * pos[l] != 0 marks a positive-definite tracer (limited). Decisions where the reference's
 * code is not well defined are stated at the limiter. */
void oracle_time_step_tracers(oracle_ctx *c, oreal *state, oreal *tracers, int ntr, const int *pos, oreal dt);
/* One split of that step along dir (0/1/2). */
void oracle_split_tracers(oracle_ctx *c, oreal *state, oreal *tracers, int ntr, const int *pos, oreal dt, int dir);
int oracle_get_dimswitch(const oracle_ctx *c);
/* Faces of the last oracle_split_tracers / oracle_time_step_tracers split whose limited
 * flux differs from the value computed with every face read before scaling: the faces where
 * the serial order of the limiter matters. */
long oracle_limiter_chained_faces(const oracle_ctx *c);
void oracle_set_dimswitch(oracle_ctx *c, int v);

/* Derived tables and background, for pinning against the reference. */
void oracle_get_tables(const oracle_ctx *c, oreal *s2g, oreal *deriv, oreal *idl, oreal *sigma);
void oracle_get_background(const oracle_ctx *c, oreal *dens_c, oreal *pres_c, oreal *theta_c,
                           oreal *denstheta_c, oreal *dens_g, oreal *pres_g, oreal *theta_g,
                           oreal *denstheta_g);
/* Single-function probes. */
oreal oracle_coefs_to_tv(const oreal *a, int n);
void oracle_weno_coefs(const oracle_ctx *c, const oreal *stencil, oreal *coefs_out);

#ifdef __cplusplus
}
#endif
#endif
