// Internal declarations shared by the library's translation units (not part of the ABI).
#pragma once

#include <cuda_runtime.h>
#include <cstddef>

namespace awfl {

namespace adj {
struct SplitArgs;
}
template <class Args> struct EnsList;
struct SweepArgs32;
struct SweepArgs;

// phys_params.h:4-10
constexpr double GRAV = 9.81;
constexpr double C0 = 27.5629410929725921310572974482;
constexpr double GAMMA = 1.40027894002789400278940027894;

enum { idR = 0, idU = 1, idV = 2, idW = 3, idT = 4 };
enum { BC_PERIODIC = 0, BC_WALL = 1 };
enum { MODE_TEND = 0, MODE_APPLY = 1 };

template <int ORD> struct OrdTraits;
template <> struct OrdTraits<5> { static constexpr int NGLL = 3; };
template <> struct OrdTraits<9> { static constexpr int NGLL = 5; };

// Constant tables (Spatial:274-315), one set per order, uploaded once per device.
template <int ORD> struct Tables {
  static constexpr int HS = (ORD - 1) / 2;
  static constexpr int NG = OrdTraits<ORD>::NGLL;
  double recon[ORD * ORD * ORD];  // weno_sten_to_coefs(i, s, ii)
  double c2g[ORD * NG];            // coefs_to_gll(s, ii)
  double s2g[ORD * NG];            // sten_to_gll(s, ii)
  double deriv[NG * NG];          // derivMatrix(s, ii)
  double idl[HS + 2];
  double sigma;
  double wts[NG];                 // gllWts_ngll
  double ridl;                    // RN(1/idl[HS+1]), the bridge polynomial's divisor
};

// Per-line constants of one sweep.
struct SweepArgs {
  double *state;   // (5, nz+2hs, ny+2hs, nx+2hs)
  double *tend;    // (5, nz, ny, nx) for MODE_TEND
  long plane;      // tangent-linear sweep: offset of the tangent plane in state (else 0)
  int nx, ny, nz;
  int bc;          // BC along the sweep direction
  int weno_s, weno_w, sim2d, mode;
  double dxd;      // dx, dy or dz
  double rdxd;     // RN(1/dxd)
  double dt;
  const double *dens_c, *denstheta_c;             // hyDensCells, hyDensThetaCells (nz+2hs)
  const double *dens_g, *denstheta_g, *pres_g;    // hyDensGLL, hyDensThetaGLL, hyPressureGLL (nz*ngll)
  // x sweeps of a slab of a larger grid: the halo columns of a slab end that borders
  // another slab, [5][nz][ny][hs+1] values per side (side 0: positions -(hs+1)..-1, the
  // lower neighbour's last columns; side 1: positions nx..nx+hs, the upper neighbour's
  // first); nullptr for an end with the grid's own boundary condition
  const double *xh[2];
};


struct InitLaunch {
  void *state;
  float *state32, *comp32;  // FP32 contexts: value and Kahan planes (state unused)
  int nx, ny, nz, hs, ord;
  int xoff, nx_global;  // a slab: its first cell's global x index; the grid's nx (0: not a slab)
  double dx, dy, dz, xlen, ylen, zlen;
  int data_spec, sim2d, kind, shape;
  double x0, y0, z0, xrad, yrad, zrad, amp, pwr, noise_amp;
  unsigned long long seed;
  int noise_kind;
  const double *dens_c;
  double pts[9], wts[9];
};

// FP32 form (awfl_fp32.cu)
struct SweepArgs32;
cudaError_t launch_sweep_fp32(int ord, int dir, const SweepArgs32 &A, cudaStream_t st);
cudaError_t launch_apply_fp32(float *state, float *comp, const float *tend, float dt, int nx, int ny, int nz, int hs,
                              int nsm, cudaStream_t st);
cudaError_t launch_cfl_fp32(const float *state, const double *dens_c, const double *denstheta_c, double cfl, double dx,
                            double dy, double dz, int nx, int ny, int nz, int hs, int nsm, unsigned long long *d_out,
                            cudaStream_t st);
cudaError_t upload_tables_fp32(int ord, const double *recon, const double *c2g, const double *s2g,
                               const double *deriv, const double *idl, double sigma, const double *wts);

// Ensemble sweeps (awfl_ens32.cu, awfl_ens64.cu): launch (occ == nullptr) or query the
// occupancy of tile shape `shape` (awfl_ens.cuh).
cudaError_t ens_run_fp32(int ord, int dir, int shape, const EnsList<SweepArgs32> *E, int grid, int *occ,
                         cudaStream_t st);
cudaError_t ens_run_fp64(int ord, int dir, int shape, const EnsList<SweepArgs> *E, int grid, int *occ,
                         cudaStream_t st);
cudaError_t upload_tables_ens32(int ord, const double *recon, const double *c2g, const double *s2g,
                                const double *deriv, const double *idl, double sigma, const double *wts);
cudaError_t upload_tables_ens64(int ord, const void *tab, size_t bytes);

// Error message for entry points without a context (awfl_capi.cu).
void set_unbound_error(const char *msg);

// FP64 translation unit (awfl_fp64.cu)
cudaError_t upload_tables_fp64(int ord, const void *tab, size_t bytes);
cudaError_t launch_sweep_fp64(int ord, int dir, const SweepArgs &A, cudaStream_t st);
// Differentiation TU (awfl_adjoint.cu)
cudaError_t launch_sweep_tlm(int ord, int dir, const SweepArgs &A, cudaStream_t st);
// FP64 sweep that also records level-0 values and edges of every cell into A.tend
cudaError_t launch_sweep_rec(int ord, int dir, const SweepArgs &A, cudaStream_t st);
cudaError_t upload_tables_adj(int ord, const void *tab, size_t bytes);
// Tracer transport of the FP64 path (awfl_tracers.cu): one split of state (fused, MODE_APPLY
// arithmetic of awfl_split) and tracers; scratch holds tracer_scratch_bytes(..., 8) bytes.
// io: TRC_IN_DIVIDED, the tracers arrive divided by the current density (no division at
// the start); TRC_OUT_DIVIDED, the update leaves the interior divided by the post-split
// density (for the next split of the same step).
enum { TRC_IN_DIVIDED = 1, TRC_OUT_DIVIDED = 2 };
cudaError_t launch_split_tracers(int ord, int dir, const SweepArgs &A, double *tracers, int ntr,
                                 unsigned long long pos, double *scratch, int io, cudaStream_t st);
// Record layout of a tracer split (both precisions; planes of ncell cells, then of nfmax
// faces): R (NG*(NG-1): levels 0..NG-2 of the density series), U (NG*(NG-1): the same of
// the normal-momentum series), D (1: the pre-split rho', the stencil centre), Y (NG: 1/rho
// of the GLL points), then per face F0 (the Riemann mass flux), VN (the velocity that
// picks the upwind side), UN (the limiter's velocity), RUP (the upwind side's density),
// YUP (1/RUP). The series' last level only enters the tracer series' last momentum-flux
// level, which no edge reads, so it is not recorded. The FP32 form recomputes Y and YUP
// (its reciprocals are single fast-reciprocal instructions) and leaves their planes unused.
template <int NG> __host__ __device__ constexpr long trc_series_planes() { return (long)NG * (NG - 1); }
template <int NG> __host__ __device__ constexpr long trc_cell_planes() { return 2 * trc_series_planes<NG>() + 1 + NG; }
// scratch of one tracer split: records and fluxes of elem bytes each, and the line flags
size_t tracer_scratch_bytes(int ord, int nx, int ny, int nz, int ntr, int elem);
cudaError_t upload_tables_tracers(int ord, const void *tab, size_t bytes);
// The same in the FP32 form (awfl_tracers32.cu): the FP32 state split with FP64 tracers;
// scratch holds tracer_scratch_bytes(..., 4) bytes; dens_c: rho_h rows (FP64).
cudaError_t launch_split_tracers32(int ord, int dir, const SweepArgs32 &A, const double *dens_c, double dt,
                                   double dxd, double *tracers, int ntr, unsigned long long pos, float *scratch,
                                   int io, cudaStream_t st);
cudaError_t upload_tables_tracers32(int ord, const double *recon, const double *c2g, const double *s2g,
                                    const double *deriv, const double *idl, double sigma, const double *wts);
// Adjoint reverse sweeps (awfl_adjrev.cu)
cudaError_t launch_adjoint_split(int ord, int dir, const adj::SplitArgs &A, int need_edges, int nsm, cudaStream_t st);
cudaError_t launch_zero_halo(double *lam, int nx, int ny, int nz, int hs, int nsm, cudaStream_t st);
cudaError_t upload_tables_adjrev(int ord, const void *tab, size_t bytes);
cudaError_t launch_apply_fp64(double *state, const double *tend, double dt, int nx, int ny, int nz, int hs,
                              int nsm, cudaStream_t st);
// x += dt*0 on the interior of nplanes planes (the sim2d y split's apply of zero tendencies)
cudaError_t launch_add_zero_fp64(double *p, int nplanes, int nx, int ny, int nz, int hs, int nsm, cudaStream_t st);
cudaError_t launch_cfl_fp64(const double *state, const double *dens_c, const double *denstheta_c, double cfl,
                            double dx, double dy, double dz, int nx, int ny, int nz, int hs, int nsm,
                            unsigned long long *d_out, cudaStream_t st);
cudaError_t launch_init_state_fp64(const InitLaunch &L, cudaStream_t st);
cudaError_t launch_init_tracers_fp64(const InitLaunch &L, int ntr, cudaStream_t st);
cudaError_t launch_tracer_fields(const void *state, int fp32, long plane, const double *dens_c,
                                 const double *tracers, int ntr, int nx, int ny, int nz, int hs, int nsm, double *out,
                                 cudaStream_t st);
// interior sums x dV (partials[nblk*5] -> out[5], fixed order) and the bad-cell count
cudaError_t launch_state_sums(const void *state, int fp32, long plane, int nx, int ny, int nz, int hs, double dv,
                              double *partials, int nblk, double *out, cudaStream_t st);
cudaError_t launch_check_state(const void *state, int fp32, long plane, const double *dens_c, int nx, int ny,
                               int nz, int hs, int nsm, unsigned long long *count, cudaStream_t st);
cudaError_t run_fma_peak(int kind, int nsm, double *tflops);  // 0 FP64, 1 FP32, 2 paired FP32
cudaError_t launch_output_fields(const void *state, int fp32, long plane, const double *dens_c,
                                 const double *denstheta_c, const double *pres_c, int nx, int ny, int nz, int hs,
                                 int nsm, double *out, cudaStream_t st);
cudaError_t launch_selftest_pow(const double *x, double y, double *out, long n, int mode, cudaStream_t st);
// The hs+1 first and last interior x columns of every variable of a state (value plane)
// into send = [2][5][nz][ny][hs+1] elements of the state's type (esz 8 or 4).
cudaError_t launch_slab_pack(const void *state, int esz, int nx, int ny, int nz, int hs, void *send, cudaStream_t st);

}  // namespace awfl
