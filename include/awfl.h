/* awfl.h -- C ABI of the B200-native AWFL Euler-3D ADER/WENO finite-volume step.
 *
 * This is the boundary that replaces the reference's YAKL parallel_for kernels behind its
 * Spatial/Temporal operator interface (mrnorman/awflCloud):
 *   Spatial_euler3d_cons_expl_cart_fv_Agrid.h (the spatial operator, "Spatial" below)
 *   Temporal_ader.h                            (the ADER time stepper)
 * The C++ drop-in headers in awflcloud_b200/dropin/ implement that interface on top of
 * these entry points; any other host (ctypes, JNI, cgo) can bind them directly.
 *
 * Conventions
 *   - Plain pointers and sizes only. Device pointers are CUDA device addresses; streams
 *     are passed as void* (a cudaStream_t; NULL = the legacy default stream).
 *   - State arrays are C-order (5, nz+2hs, ny+2hs, nx+2hs), x fastest, variables
 *     (rho', rho*u, rho*v, rho*w, (rho*theta)') -- Spatial:129-131, :69-73.
 *     Tendency arrays are C-order (5, nz, ny, nx) -- Spatial:141-143.
 *   - Element type is double for AWFL_FP64 contexts and float for AWFL_FP32 contexts.
 *     An FP32 state buffer holds two such planes back to back: the values, then the Kahan
 *     compensation of the stage updates (zeroed by awfl_init_state); awfl_sizes reports
 *     the total. The library cannot see allocation sizes: buffers must be at least that
 *     large.
 *   - Every function returns AWFL_OK (0) or a negative awfl_status; nothing throws
 *     across the ABI. awfl_last_error() gives the message of the last failure.
 *   - A context is used by one host thread at a time; all work is ordered on the
 *     stream passed in. Separate contexts are independent.
 */
#ifndef AWFL_H
#define AWFL_H

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  AWFL_OK = 0,
  AWFL_ERR_ARG = -1,       /* invalid argument or unsupported configuration */
  AWFL_ERR_CUDA = -2,      /* a CUDA runtime call failed */
  AWFL_ERR_NOMEM = -3,     /* device allocation failed */
  AWFL_ERR_STATE = -4,     /* device-side check failed (NaN / non-positive density) */
  AWFL_ERR_TIMEOUT = -5,   /* a bounded device wait gave up */
  AWFL_ERR_NOT_BUILT = -6, /* the requested variant is not compiled into this library */
  AWFL_ERR_IO = -7         /* an output file could not be written, or is not this grid's */
} awfl_status;

enum { AWFL_BC_PERIODIC = 0, AWFL_BC_WALL = 1 };           /* Spatial:80-81 */
enum { AWFL_FP64 = 0, AWFL_FP32 = 1 };
enum { AWFL_DATA_THERMAL = 1, AWFL_DATA_COLLISION = 2,      /* Spatial:83-86 */
       AWFL_DATA_STRAKA = 3, AWFL_DATA_IGW = 4 };
enum { AWFL_DIR_X = 0, AWFL_DIR_Y = 1, AWFL_DIR_Z = 2 };

/* The YAML keys read by Spatial::init (Spatial:197-272) plus the compile-time order
 * (const.h:21-27: ord in {5, 9}, ngll = 3 or 5) and the arithmetic precision. */
typedef struct {
  int nx, ny, nz;
  double xlen, ylen, zlen;
  int bc_x, bc_y, bc_z;
  int weno_scalars, weno_winds;
  int data_spec;   /* selects the hydrostatic background: constant theta, or constant
                      Brunt-Vaisala frequency for AWFL_DATA_IGW (Spatial:371-425) */
  int ord;         /* 5 or 9 */
  int precision;   /* AWFL_FP64 or AWFL_FP32 */
} awfl_config;

/* Initial-data recipe for awfl_init_state. kind AWFL_INIT_REFERENCE reproduces
 * Spatial::initState for the context's data_spec (Spatial:428-485); AWFL_INIT_BUBBLE
 * replaces the theta perturbation by an ellipsoid (shape 0 linear / 1 cosine, Profiles.h
 * 49-72) integrated with the same ord^3 GLL quadrature. noise_amp > 0 then adds seeded
 * theta noise n as state(rho*theta) += hyDensCells(k) * n, cell = (k*ny + j)*nx + i:
 *   noise_kind AWFL_NOISE_UNIFORM: n = (2u-1)*amp, u = top 53 bits of
 *     splitmix64(seed*0x100000001B3 + cell)/2^53;
 *   noise_kind AWFL_NOISE_NORMAL: n = amp*sqrt(-2 ln u1)*cos(2 pi u2) (Box-Muller), u1 =
 *     (top 53 bits of splitmix64(seed*0x100000001B3 + 2 cell) + 1)/2^53, u2 likewise from
 *     2 cell + 1: normal noise of standard deviation amp. */
enum { AWFL_INIT_REFERENCE = 0, AWFL_INIT_BUBBLE = 1 };
enum { AWFL_NOISE_UNIFORM = 0, AWFL_NOISE_NORMAL = 1 };
typedef struct {
  int kind;
  int shape;
  double x0, y0, z0, xrad, yrad, zrad, amp, pwr;
  double noise_amp;
  unsigned long long noise_seed;
  int noise_kind;
} awfl_init_spec;

typedef struct awfl_ctx awfl_ctx;

/* Spatial::init (Spatial:192-340) + the background of Spatial::initState (:371-425):
 * validates the configuration, builds the transform tables and the hydrostatic
 * background on `device`, uploads them. device < 0 makes a host-only context: tables and
 * background are built (awfl_get_tables / awfl_get_background work) but every entry point
 * that runs device work returns AWFL_ERR_ARG. */
int awfl_create(const awfl_config *cfg, int device, awfl_ctx **out);
int awfl_destroy(awfl_ctx *ctx);
const char *awfl_last_error(const awfl_ctx *ctx);
/* Library version string (never NULL). */
const char *awfl_version(void);

/* Sizes (elements) of the state (with halos) and tendency arrays; the halo width hs. */
int awfl_sizes(const awfl_ctx *ctx, long *state_elems, long *tend_elems, int *hs);

/* Spatial::initState (Spatial:345-500) on the device; writes the interior of d_state. */
int awfl_init_state(awfl_ctx *ctx, void *d_state, const awfl_init_spec *spec, void *stream);

/* Sums over the interior of the five conserved variables times the cell volume, in FP64
 * (FP32 contexts: the value plane minus the Kahan compensation): sums[0] = sum rho' dV
 * (the perturbation mass), sums[1..3] the momenta, sums[4] = sum (rho theta)' dV. Fixed
 * reduction order, so the result is reproducible bit for bit. Synchronises the stream.
 * (The reference has no such diagnostic; its run only prints dt and etime.) */
int awfl_state_sums(awfl_ctx *ctx, const void *d_state, double *sums, void *stream);

/* Device-side state check: counts interior cells with a non-finite value or a
 * non-positive total density; AWFL_ERR_STATE if any (count in *bad_cells, may be NULL).
 * AWFL_ERR_TIMEOUT if a sweep of this context ever gave up its bounded wait for staged
 * stencil rows (the state is then not to be trusted). Synchronises the stream. */
int awfl_check_state(awfl_ctx *ctx, const void *d_state, long *bad_cells, void *stream);

/* The diagnostics of Spatial::output (Spatial:1744-1778) on the device, FP64, from either
 * state form: d_fields = [6][nz][ny][nx] doubles, in the order dens_pert, u, v, w,
 * pot_temp_pert, pressure_pert (rho', rho*u/rho, ..., theta - theta_h, C0*(rho*theta)^gamma
 * - p_h), with the reference's operations. Asynchronous on the stream. */
int awfl_output_fields(awfl_ctx *ctx, const void *d_state, double *d_fields, void *stream);

/* Spatial::output (Spatial:1705-1791) without the netCDF library: writes the reference's
 * output file with a project-written writer of the netCDF classic data model (64-bit
 * offset format, readable by any netCDF reader). etime == 0 creates the file (coordinates
 * x, y, z; hyDens, hyPressure, hyTheta; record 0 of t and the six fields); any other etime
 * appends a record to a file this grid created. Synchronises the stream; allocates (once
 * per context) a device buffer for the fields. AWFL_ERR_IO on a file error. */
int awfl_write_netcdf(awfl_ctx *ctx, const char *path, const void *d_state, double etime, void *stream);

/* The same file from host-side fields ([6][nz][ny][nx] doubles, as awfl_output_fields
 * gives them); needs no device (host-only contexts too). */
int awfl_write_netcdf_fields(awfl_ctx *ctx, const char *path, const double *h_fields, double etime);

/* Spatial::initTracers (Spatial:505-560; the reference runs it although its tracer
 * transport is compiled out by NO_TRACERS, Spatial:10): d_tracers = double
 * (ntracers, nz+2hs, ny+2hs, nx+2hs), interior written, for either context precision.
 * Tracer 0 = rho_h (uniform 1), 1 = rho_h x the 2 K linear ellipsoid of radius 2 km at
 * (xlen/2, ylen/2, 2 km), 2 = rho_h x the block indicator, as ord^3 GLL cell averages;
 * tracers beyond the third are zero (the reference's loop leaves them so). Asynchronous. */
int awfl_init_tracers(awfl_ctx *ctx, double *d_tracers, int ntracers, void *stream);

/* The tracer fields of Spatial::output (Spatial:1778-1783): d_fields = [ntracers][nz][ny][nx]
 * doubles, tracers(t, hs+k, hs+j, hs+i) / (rho' + hyDensCells(hs+k)). Asynchronous. */
int awfl_output_tracer_fields(awfl_ctx *ctx, const void *d_state, const double *d_tracers, int ntracers,
                              double *d_fields, void *stream);

/* awfl_write_netcdf with the reference's tracer record variables "tracer_<name>"
 * (Spatial:1778-1783) after the six diagnostics; names holds ntracers non-empty C strings.
 * Appending needs the same tracer names as the call that created the file. */
int awfl_write_netcdf_tracers(awfl_ctx *ctx, const char *path, const void *d_state, const double *d_tracers,
                              int ntracers, const char *const *names, double etime, void *stream);
/* The same from host-side fields ([6 + ntracers][nz][ny][nx] doubles). */
int awfl_write_netcdf_fields_tracers(awfl_ctx *ctx, const char *path, const double *h_fields, int ntracers,
                                     const char *const *names, double etime);

/* Tracer transport: the reference's tracer code (Spatial:624-955 and the y/z equivalents),
 * which the reference itself compiles out (NO_TRACERS, Spatial:10), built in, for both
 * precisions: an FP32 context reconstructs, fluxes and limits the tracers in FP32 beside
 * its FP32 state split and keeps the tracers FP64 (division by the density and the update
 * in FP64). One split (dir = 0/1/2) of state AND tracers: the state as awfl_split
 * advances it (FP64: bit for bit), and the tracers -- divided by the pre-split density,
 * reconstructed, advanced by their ADER series along the state's density and normal
 * momentum, upwind fluxes from the state's Riemann mass flux, the positivity limiter for
 * tracers with pos[l] != 0, then tracers = (tracers/rho)*rho + dt*tend in place.
 * ntracers <= 64 (0: awfl_split); tracers as for awfl_init_tracers (rho*tracer). The halo
 * cells along dir are left holding tracer/rho, as the reference's in-place halo fill leaves
 * them. Allocates (once per context, grown when ntracers grows) a scratch buffer of
 * (2*ngll*(ngll-1) + ngll + 1) values per cell and (2*ntracers + 5) per face (doubles; floats in
 * an FP32 context) and two ints per line. Decisions
 * where the reference's code is not well defined: the limiter scales the faces of a line
 * in place in increasing order, as the reference's loop does when it runs serially (it
 * scales in place while other iterations read, Spatial:904-935); the y limiter's v < 0
 * branch reads the y faces (the reference swaps j and i there, :1285-1286); a periodic z
 * wraps (the reference reads outside its flux array there). */
int awfl_split_tracers(awfl_ctx *ctx, void *d_state, double *d_tracers, int ntracers, const int *pos, double dt,
                       int dir, void *stream);
/* One time step with tracers (Temporal_ader::timeStep with the tracer code compiled in):
 * awfl_split_tracers for each split in the dimSwitch order; between two splits the
 * tracers' interior stays divided by the density (each split's update does the division
 * the next would start with), which gives the same values bit for bit. After an error the
 * tracer array may be left divided. */
int awfl_step_tracers(awfl_ctx *ctx, void *d_state, double *d_tracers, int ntracers, const int *pos, double dt,
                      void *stream);

/* Spatial::computeTimeStep without the caching (Spatial:159-187): the acoustic CFL time
 * step, min over all cells, returned in *h_dt (synchronises the stream). */
int awfl_cfl(awfl_ctx *ctx, const void *d_state, double cfl, double *h_dt, void *stream);

/* Spatial::computeTendenciesX/Y/Z for dir = 0/1/2 (Spatial:598-957, 961-1311,
 * 1315-1697): fills the dir-halos of d_state in place (as the reference does) and writes
 * the dt-time-averaged tendencies to d_tend. The interior of d_state is not modified. */
int awfl_compute_tendencies(awfl_ctx *ctx, void *d_state, void *d_tend, double dt, int dir,
                            void *stream);

/* Temporal_ader's apply (Temporal_ader.h:63-65): state(l,hs+k,hs+j,hs+i) += dt*tend(l,k,j,i). */
int awfl_apply_tendencies(awfl_ctx *ctx, void *d_state, const void *d_tend, double dt,
                          void *stream);

/* One split fused: compute_tendencies(dir) followed by apply_tendencies, in one kernel,
 * without a tendency array. Same results as the two calls. */
int awfl_split(awfl_ctx *ctx, void *d_state, double dt, int dir, void *stream);

/* Temporal_ader::timeStep (Temporal_ader.h:48-72): three fused splits in the order
 * X,Y,Z or Z,Y,X (the reference's dimSwitch, Spatial:568-593, kept in the context and
 * flipped after every step). sim2d (ny == 1) skips the Y split, whose tendency the
 * reference sets to zero. */
int awfl_step(awfl_ctx *ctx, void *d_state, double dt, void *stream);

/* ---- x-slab decomposition of one grid over several GPUs: no counterpart in the active
 * reference, whose single domain lives in one process; its legacy model decomposes x/y
 * with MPI halo exchanges (qjrmsCode/Exchange.cpp:106-176) and an MPI_Allreduce(MIN) of dt
 * (qjrmsCode/Initializer.cpp:263). Slab s of n owns the x cells [xoff, xoff + nx_s) of the
 * grid `global` (nx split as evenly as possible, every slab at least hs+1 cells) with the
 * whole y and z extent; its context works on its own state (awfl_sizes: nx_s in x) with
 * the grid's dx, places initial data by global cell (awfl_init_state), and runs y and z
 * splits alone (awfl_split). Before each x split the slabs trade hs+1 columns:
 *   awfl_slab_pack   copies the slab's first and last hs+1 interior columns of every
 *                    variable into d_send = [2][5][nz][ny][hs+1] (side 0: first columns,
 *                    for the slab below; side 1: last columns, for the slab above);
 *   (the caller moves side 1 of slab s to side 0 of d_recv of slab s+1, and side 0 of
 *   slab s to side 1 of d_recv of slab s-1: NCCL send/recv, a copy, ...; a periodic x
 *   wraps from the last slab to the first);
 *   awfl_split_slab  the fused x split with the neighbours' columns (d_recv, same layout:
 *                    side 0 = the slab below's last columns, side 1 = the slab above's
 *                    first); an end at a wall of the grid ignores its side.
 * The interior cells then advance bit for bit as in the undivided grid. The CFL time step
 * of the grid is the minimum of the slabs' awfl_cfl. Tracer transport, the tangent-linear
 * step and the adjoint refuse slab contexts, and so do awfl_step, awfl_split and
 * awfl_compute_tendencies for the x direction when an end borders another slab. */
int awfl_create_slab(const awfl_config *global, int nslabs, int slab, int device, awfl_ctx **out);
/* The slab's place: slab count, index, global x index of its first cell, the grid's nx,
 * and the elements of one d_send / d_recv buffer (2*5*nz*ny*(hs+1)). Any pointer may be
 * NULL; a context made by awfl_create is slab 0 of 1. */
int awfl_slab_info(const awfl_ctx *ctx, int *nslabs, int *slab, int *xoff, int *nx_global, long *halo_elems);
int awfl_slab_pack(awfl_ctx *ctx, const void *d_state, void *d_send, void *stream);
int awfl_split_slab(awfl_ctx *ctx, void *d_state, const void *d_recv, double dt, void *stream);

/* Tangent-linear time step (FP64 contexts): d_state_tangent holds two FP64 state planes,
 * the state then a perturbation direction. The state advances exactly like awfl_step
 * (bit-identical) and the second plane becomes the derivative of the new state along the
 * direction (forward-mode differentiation of the same arithmetic; dt is held fixed).
 * Flips dimSwitch like awfl_step. */
int awfl_step_tlm(awfl_ctx *ctx, void *d_state_tangent, double dt, void *stream);

/* Discrete adjoint of nsteps time steps (FP64 contexts; no counterpart in the reference,
 * whose time loop is Temporal_ader.h:48-72). d_state_ckpt is the state at the start of
 * the window (a checkpoint; not modified) and the context's dimSwitch must hold its value
 * at that checkpoint (awfl_set_dimswitch); it is left unchanged. On entry d_lambda holds
 * the adjoint of the state after the nsteps steps (dJ/dS_end), on return the adjoint of
 * the checkpoint state (dJ/dS_ckpt), dt held fixed. Halo entries of d_lambda are ignored
 * on entry and zero on return. The window is recomputed forward from the checkpoint and
 * its split-start states and per-split records kept on a device tape owned by the context
 * (see awfl_adjoint_tape_bytes); a caller checkpointing every k steps calls this once per
 * segment, last segment first. With a sub-window length m set (awfl_set_adjoint_subwindow)
 * the window is taken m steps at a time: one plain forward pass keeps the state at every
 * m-th step, then each sub-window, last first, is recomputed with its records and
 * reversed -- a tape of about nsteps/m + 3m states and 3m records instead of 3*nsteps + 1
 * states and 3*nsteps records, for one more forward pass over the window. The result is
 * the same either way. Stream-ordered on `stream`. */
int awfl_step_adjoint(awfl_ctx *ctx, const void *d_state_ckpt, void *d_lambda, int nsteps, double dt,
                      void *stream);

/* Device memory awfl_step_adjoint holds for a window of nsteps steps (tape + scratch). */
int awfl_adjoint_tape_bytes(const awfl_ctx *ctx, int nsteps, long *bytes);

/* Steps per recorded sub-window of awfl_step_adjoint (0, the default: the whole window). */
int awfl_set_adjoint_subwindow(awfl_ctx *ctx, int steps);

/* The dimSwitch flag of the context (1 = next step runs X,Y,Z). */
int awfl_get_dimswitch(const awfl_ctx *ctx, int *value);
int awfl_set_dimswitch(awfl_ctx *ctx, int value);

/* Host views of the tables and background the context built, for verification:
 * weno_recon (ord^3), coefs_to_gll (ord*ngll), sten_to_gll (ord*ngll), deriv (ngll^2),
 * idl (hs+2), sigma (1), gll points/weights (ord, ord, ngll, ngll); hydrostatic cells
 * (4 x (nz+2hs): dens, pressure, theta, dens*theta) and GLL (4 x nz*ngll). Any pointer
 * may be NULL. Host-only; needs no GPU work. */
int awfl_get_tables(const awfl_ctx *ctx, double *weno_recon, double *coefs_to_gll,
                    double *sten_to_gll, double *deriv, double *idl, double *sigma,
                    double *gll_pts_ord, double *gll_wts_ord, double *gll_pts_ngll,
                    double *gll_wts_ngll);
int awfl_get_background(const awfl_ctx *ctx, double *dens_c, double *pres_c, double *theta_c,
                        double *denstheta_c, double *dens_g, double *pres_g, double *theta_g,
                        double *denstheta_g);

/* Allocation-free CFL time step. No counterpart in the reference: it is an extra entry
 * point for callers that cannot call cudaMalloc -- hosts whose device memory all comes
 * from their own arena or pool and must not be allocated behind their back, or loops that
 * cannot afford the device synchronisation an allocation may cause. It needs no context
 * and allocates nothing: the caller passes the FP64 state and the device copies of the
 * hydrostatic cell averages hyDensCells and hyDensThetaCells (nz+2hs each, as returned by
 * awfl_get_background), and the reduction runs in a static device array of the library
 * (512 KiB per GPU that loads it, held until exit). Result: the same value as awfl_cfl.
 * Limits: FP64 only; nx*ny*nz <= 16,777,216 cells, larger grids are rejected with
 * AWFL_ERR_ARG (use awfl_cfl). The first call on each device looks up the array's device
 * address and keeps it for the life of the process; make that first call before any stream
 * capture, and do not call this entry point again on a device after cudaDeviceReset (the
 * reset unloads the library's device code, so the kept address no longer names the
 * array). Every call shares the one
 * array: calls that overlap on the GPU (other streams, other host threads) race.
 * Synchronises `stream`. Errors are reported by awfl_last_error(NULL). */
int awfl_cfl_noalloc(const awfl_config *cfg, const void *d_state, const void *d_hy_dens_cells,
                     const void *d_hy_denstheta_cells, double cfl, double *h_dt, void *stream);

/* Diagnostic: the FP64 path's device math on n doubles (device pointers). mode 0:
 * out = pow(x, y) by the library's correctly rounded pow (the one every FP64 kernel uses
 * in place of the reference's glibc pow); mode 1: the CUDA math library's pow, for
 * comparison; mode 2: the library's correctly rounded exp(x) (y ignored); mode 3:
 * out[i] = x[i] / x[n+i] by the FP64 kernels' division through a shared reciprocal (d_x
 * holds 2n doubles, y ignored); mode 4: the same quotients by the GPU's IEEE division. */
int awfl_selftest_pow(const void *d_x, double y, void *d_out, long n, int mode, void *stream);

/* Diagnostic: measured FMA throughput of the CUDA-core pipe the kernels run on, in TFLOP/s
 * (2 flops per FMA lane), from a ~0.1 s FMA-chain kernel on `device`: precision AWFL_FP64,
 * AWFL_FP32 (scalar FFMA) or AWFL_PEAK_FP32_PAIRED (sm_100's paired FP32 FMA, one
 * instruction for two lanes). The roofline denominator of the ADER/WENO kernels, which
 * are bound by these pipes. */
enum { AWFL_PEAK_FP32_PAIRED = 2 };
int awfl_measure_fma_peak(int precision, int device, double *tflops);

/* Device memory helpers for hosts that do not link the CUDA runtime themselves. */
int awfl_device_alloc(void **d_ptr, long bytes);
int awfl_device_free(void *d_ptr);
int awfl_copy_h2d(void *d_dst, const void *h_src, long bytes, void *stream);
int awfl_copy_d2h(void *h_dst, const void *d_src, long bytes, void *stream);
int awfl_memset_device(void *d_ptr, int value, long bytes, void *stream);
int awfl_stream_synchronize(void *stream);
int awfl_device_synchronize(void);

/* ---- Ensemble (batching) form: no counterpart in the reference ----------------------
 * An ensemble advances many independent members (each its own awfl_config: grid size,
 * domain, boundary conditions; all with the same precision and ord) together: per split
 * stage one persistent kernel covers the tiles of every member, and pairs of time steps
 * replay a CUDA graph. An FP64 member's result is bit-identical to awfl_step on its own
 * context; an FP32 member's agrees to FP32 rounding (multiply-add contraction may be
 * placed differently in the persistent kernel). The ensemble owns the member contexts (awfl_ensemble_member lends them for
 * awfl_init_state, awfl_cfl, ...); the caller owns the state buffers it binds. */
typedef struct awfl_ensemble awfl_ensemble;

int awfl_ensemble_create(const awfl_config *cfgs, int nmembers, int device, awfl_ensemble **ens);
int awfl_ensemble_destroy(awfl_ensemble *ens);
const char *awfl_ensemble_last_error(const awfl_ensemble *ens);
int awfl_ensemble_size(const awfl_ensemble *ens, int *nmembers);
int awfl_ensemble_member(awfl_ensemble *ens, int i, awfl_ctx **ctx);
/* Member i advances d_state (awfl_sizes elements of its context) with time step dt. */
int awfl_ensemble_bind(awfl_ensemble *ens, int i, void *d_state, double dt);
/* nsteps time steps of every member (dimSwitch kept by the ensemble, flipped per step). */
int awfl_ensemble_step(awfl_ensemble *ens, int nsteps, void *stream);
/* Autotuner: times `reps` launches of every candidate tile shape of each direction on
 * scratch copies of the bound states (the bound states are not advanced) and keeps the
 * fastest; synchronizes `stream`. */
int awfl_ensemble_tune(awfl_ensemble *ens, int reps, void *stream);
int awfl_ensemble_num_shapes(const awfl_ensemble *ens, int dir, int *n);
/* Candidate i of direction dir: chunk length, lines per CTA, and the tuner's ms per
 * launch (negative before tuning). */
int awfl_ensemble_tuning(const awfl_ensemble *ens, int dir, int i, int *chunk, int *lines, float *ms);
/* Shape in use for direction dir (index, chunk, lines, persistent grid size). */
int awfl_ensemble_get_shape(const awfl_ensemble *ens, int dir, int *shape, int *chunk, int *lines, int *grid);
int awfl_ensemble_set_shape(awfl_ensemble *ens, int dir, int shape);
int awfl_ensemble_get_dimswitch(const awfl_ensemble *ens, int *value);
int awfl_ensemble_set_dimswitch(awfl_ensemble *ens, int value);

#ifdef __cplusplus
}
#endif
#endif /* AWFL_H */
