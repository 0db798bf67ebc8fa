// FP64 kernels of the AWFL Euler-3D ADER/WENO step (the parity path), sm_100a.
// Compiled with --fmad=false: no multiply-add contraction, matching the reference's CPU build.
//
// Kernel map (reference kernels it replaces, Spatial = Spatial_euler3d_cons_expl_cart_fv_Agrid.h):
//   sweep_kernel<P64,ORD,DIR>  (awfl_sweep.cuh) K1 halo fill + K2 recon/ADER + K3 edge BCs +
//                          K4 Riemann + K5 divergence (+ K6 apply when fused), one direction
//                          (Spatial:631-957 x, 994-1310 y, 1351-1696 z; Temporal_ader.h:63-65)
//   apply_kernel           K6 apply alone (Temporal_ader.h:63-65)
//   add_zero_kernel        the apply of a sim2d y split's zero tendencies
//   cfl_kernel             K0 CFL time step (Spatial:169-183)
//   init_state_kernel      K9 initial data quadrature (Spatial:428-485)
#include <cuda_runtime.h>

#include <cstring>

#include "awfl_internal.h"
#include "awfl_p64.cuh"

namespace awfl {

cudaError_t launch_sweep_fp64(int ord, int dir, const SweepArgs &A, cudaStream_t st) {
  return launch_sweep_any<P64>(ord, dir, A, st);
}



// ------------------------------------------------------------------------------------
// K6 apply (Temporal_ader.h:63-65): state(l,hs+k,hs+j,hs+i) += dt * tend(l,k,j,i).
// ------------------------------------------------------------------------------------
__global__ void apply_kernel(double *state, const double *tend, double dt, int nx, int ny, int nz, int hs) {
  const long n = 5L * nz * ny * nx;
  for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < n; idx += (long)gridDim.x * blockDim.x) {
    long r = idx;
    const int i = r % nx; r /= nx;
    const int j = r % ny; r /= ny;
    const int k = r % nz; r /= nz;
    const int l = (int)r;
    const long s = (((long)l * (nz + 2 * hs) + hs + k) * (ny + 2 * hs) + hs + j) * (nx + 2 * hs) + hs + i;
    state[s] += dt * tend[idx];
  }
}

cudaError_t launch_apply_fp64(double *state, const double *tend, double dt, int nx, int ny, int nz, int hs,
                              int nsm, cudaStream_t st) {
  const long n = 5L * nz * ny * nx;
  long blocks = (n + 255) / 256;
  const long cap = (long)nsm * 8;
  if (blocks > cap) blocks = cap;
  if (blocks < 1) blocks = 1;
  apply_kernel<<<(unsigned)blocks, 256, 0, st>>>(state, tend, dt, nx, ny, nz, hs);
  return cudaGetLastError();
}

// x += dt*0 on the interior of nplanes planes of the state layout: what the apply
// (Temporal_ader.h:63-69) does with the zero tendencies of a sim2d y split (Spatial:572-575).
// It changes no value; a -0 becomes +0, as in the reference.
__global__ void add_zero_kernel(double *p, int nplanes, int nx, int ny, int nz, int hs) {
  const long n = (long)nplanes * nz * ny * nx;
  for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < n; idx += (long)gridDim.x * blockDim.x) {
    long r = idx;
    const int i = r % nx; r /= nx;
    const int j = r % ny; r /= ny;
    const int k = r % nz; r /= nz;
    const int l = (int)r;
    const long s = (((long)l * (nz + 2 * hs) + hs + k) * (ny + 2 * hs) + hs + j) * (nx + 2 * hs) + hs + i;
    p[s] = __dadd_rn(p[s], 0.0);
  }
}

cudaError_t launch_add_zero_fp64(double *p, int nplanes, int nx, int ny, int nz, int hs, int nsm, cudaStream_t st) {
  const long n = (long)nplanes * nz * ny * nx;
  long blocks = (n + 255) / 256;
  const long cap = (long)nsm * 8;
  if (blocks > cap) blocks = cap;
  if (blocks < 1) blocks = 1;
  add_zero_kernel<<<(unsigned)blocks, 256, 0, st>>>(p, nplanes, nx, ny, nz, hs);
  return cudaGetLastError();
}

// ------------------------------------------------------------------------------------
// K0 CFL (Spatial:169-183): per-cell min(cfl*dx/max|u+-cs|, ...); block min in shared
// memory, then an atomic min on the bit pattern (valid for non-negative doubles) into
// *out, which the caller initialises to +inf.
// ------------------------------------------------------------------------------------
__global__ void cfl_kernel(const double *state, const double *dens_c, const double *denstheta_c,
                           double cfl, double dx, double dy, double dz, int nx, int ny, int nz, int hs,
                           unsigned long long *out) {
  __shared__ double red[256];
  double best = __longlong_as_double(0x7ff0000000000000LL);  // +inf
  const long n = (long)nz * ny * nx;
  const long sy = nx + 2 * hs, sz = (long)(ny + 2 * hs) * sy, sv = (long)(nz + 2 * hs) * sz;
  for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < n; idx += (long)gridDim.x * blockDim.x) {
    const int i = idx % nx;
    const int j = (idx / nx) % ny;
    const int k = idx / ((long)nx * ny);
    const long s = (hs + k) * sz + (hs + j) * sy + hs + i;
    const double r = state[s] + dens_c[hs + k];
    const double u = state[s + sv] / r;
    const double v = state[s + 2 * sv] / r;
    const double w = state[s + 3 * sv] / r;
    const double t = (state[s + 4 * sv] + denstheta_c[hs + k]) / r;
    const double p = C0 * pow_cr(r * t, GAMMA);
    const double cs = sqrt(GAMMA * p / r);
    const double au = fabs(u - cs), bu = fabs(u + cs);
    const double av = fabs(v - cs), bv = fabs(v + cs);
    const double aw = fabs(w - cs), bw = fabs(w + cs);
    const double udt = cfl * dx / (au > bu ? au : bu);
    const double vdt = cfl * dy / (av > bv ? av : bv);
    const double wdt = cfl * dz / (aw > bw ? aw : bw);
    const double m1 = udt < vdt ? udt : vdt;
    const double d = m1 < wdt ? m1 : wdt;
    best = d < best ? d : best;
  }
  red[threadIdx.x] = best;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      const double o = red[threadIdx.x + s];
      if (o < red[threadIdx.x]) red[threadIdx.x] = o;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) atomicMin(out, (unsigned long long)__double_as_longlong(red[0]));
}

cudaError_t launch_cfl_fp64(const double *state, const double *dens_c, const double *denstheta_c, double cfl,
                            double dx, double dy, double dz, int nx, int ny, int nz, int hs, int nsm,
                            unsigned long long *d_out, cudaStream_t st) {
  const long n = (long)nz * ny * nx;
  long blocks = (n + 255) / 256;
  const long cap = (long)nsm * 8;
  if (blocks > cap) blocks = cap;
  if (blocks < 1) blocks = 1;
  cfl_kernel<<<(unsigned)blocks, 256, 0, st>>>(state, dens_c, denstheta_c, cfl, dx, dy, dz, nx, ny, nz, hs, d_out);
  return cudaGetLastError();
}

// ------------------------------------------------------------------------------------
// K9 initial data (Spatial:428-485 and Profiles.h), one thread per cell.
// ------------------------------------------------------------------------------------
struct InitArgs {
  double *state;
  float *state32, *comp32;
  int nx, ny, nz, hs, ord;
  int xoff, nx_global;  // a slab of a larger grid: global x index of cell 0, the grid's nx
  double dx, dy, dz, xlen, ylen, zlen;
  int data_spec, sim2d;
  int kind, shape;
  double x0, y0, z0, xrad, yrad, zrad, amp, pwr;
  double noise_amp;
  unsigned long long seed;
  int noise_kind;
  const double *dens_c;
  double pts[9], wts[9];
};

__device__ double d_const_theta_density(double t0, double z) {  // Profiles.h:8-13
  const double exner = 1. - GRAV * z / (1004. * t0);
  const double p = pow_cr(exner, 1004. / 287.) * 1.0e5;
  const double rt = pow_cr(p / C0, 1. / GAMMA);
  return rt / t0;
}
__device__ double d_bvf_pot_temp(double t0, double bvf, double z) { return t0 * exp_cr(bvf * bvf * z / GRAV); }
__device__ double d_bvf_density(double t0, double bvf, double z) {  // Profiles.h:31-37
  const double t = d_bvf_pot_temp(t0, bvf, z);
  const double exner = 1. - GRAV * GRAV / (1004. * bvf * bvf) * (t - t0) / (t * t0);
  const double p = pow_cr(exner, 1004. / 287.) * 1.0e5;
  const double rt = pow_cr(p / C0, 1. / GAMMA);
  return rt / t;
}
__device__ double d_ellipsoid_linear(double x, double y, double z, double x0, double y0, double z0, double xrad,
                                     double yrad, double zrad, double amp) {  // Profiles.h:49-57
  const double xn = (x - x0) / xrad, yn = (y - y0) / yrad, zn = (z - z0) / zrad;
  const double dist = sqrt(xn * xn + yn * yn + zn * zn);
  const double m = 1. - dist;
  return amp * (m > 0. ? m : 0.);
}
__device__ double d_ellipsoid_cosine(double x, double y, double z, double x0, double y0, double z0, double xrad,
                                     double yrad, double zrad, double amp, double pwr) {  // Profiles.h:60-72
  double val = 0;
  const double xn = (x - x0) / xrad, yn = (y - y0) / yrad, zn = (z - z0) / zrad;
  const double dist = sqrt(xn * xn + yn * yn + zn * zn);
  if (dist <= 1.) val = amp * pow_cr((cos(3.14159265358979323846 * dist) + 1) / 2, pwr);
  return val;
}
__device__ double d_igw(double x, double y, double z, double x0, double y0, double hr, double zlen,
                        double amp) {  // Profiles.h:75-81
  const double xn = (x - x0) / hr, yn = (y - y0) / hr;
  return amp * sin(3.14159265358979323846 * z / zlen) / sqrt(1 + xn * xn + yn * yn);
}
__device__ __forceinline__ unsigned long long d_splitmix64(unsigned long long x) {
  x += 0x9E3779B97F4A7C15ULL;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
  return x ^ (x >> 31);
}

__global__ void init_state_kernel(InitArgs a) {
  const long n = (long)a.nz * a.ny * a.nx;
  const long idx = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (idx >= n) return;
  const int i = idx % a.nx, j = (idx / a.nx) % a.ny, k = idx / ((long)a.nx * a.ny);
  const int hs = a.hs;
  const long sy = a.nx + 2 * hs, sz = (long)(a.ny + 2 * hs) * sy, sv = (long)(a.nz + 2 * hs) * sz;
  const long s = (hs + k) * sz + (hs + j) * sy + hs + i;
  double acc[5] = {0, 0, 0, 0, 0};
  for (int kk = 0; kk < a.ord; kk++)
    for (int jj = 0; jj < a.ord; jj++)
      for (int ii = 0; ii < a.ord; ii++) {
        const double zloc = (k + 0.5) * a.dz + a.pts[kk] * a.dz;
        double yloc = a.sim2d ? a.ylen / 2 : (j + 0.5) * a.dy + a.pts[jj] * a.dy;
        const double xloc = (a.xoff + i + 0.5) * a.dx + a.pts[ii] * a.dx;
        const double wt = a.wts[kk] * a.wts[jj] * a.wts[ii];
        if (a.kind == 1) {
          const double th = 300, rh = d_const_theta_density(th, zloc);
          const double tp = a.shape == 0
                                ? d_ellipsoid_linear(xloc, yloc, zloc, a.x0, a.y0, a.z0, a.xrad, a.yrad, a.zrad, a.amp)
                                : d_ellipsoid_cosine(xloc, yloc, zloc, a.x0, a.y0, a.z0, a.xrad, a.yrad, a.zrad, a.amp, a.pwr);
          const double t = th + tp;
          acc[4] += (rh * t - rh * th) * wt;
        } else if (a.data_spec == 1) {
          const double th = 300, rh = d_const_theta_density(th, zloc);
          const double tp = d_ellipsoid_linear(xloc, yloc, zloc, a.xlen / 2, a.ylen / 2, 2000, 2000, 2000, 2000, 2);
          const double t = th + tp;
          acc[4] += (rh * t - rh * th) * wt;
        } else if (a.data_spec == 2) {
          const double th = 300, rh = d_const_theta_density(th, zloc);
          double tp = d_ellipsoid_linear(xloc, yloc, zloc, a.xlen / 2, a.ylen / 2, 2000, 2000, 2000, 2000, 20);
          tp += d_ellipsoid_linear(xloc, yloc, zloc, a.xlen / 2, a.ylen / 2, 8000, 2000, 2000, 2000, -20);
          const double t = th + tp;
          acc[4] += (rh * t - rh * th) * wt;
        } else if (a.data_spec == 3) {
          const double th = 300, rh = d_const_theta_density(th, zloc);
          const double tp = d_ellipsoid_cosine(xloc, yloc, zloc, a.xlen / 2, a.ylen / 2, 3000, 4000, 2000, 2000, -15, 1);
          const double t = th + tp;
          acc[4] += (rh * t - rh * th) * wt;
        } else {
          if (a.sim2d) yloc = a.ylen / 3;
          const double t0 = 300, bvf = 0.01;
          const double rh = d_bvf_density(t0, bvf, zloc);
          const double th = d_bvf_pot_temp(t0, bvf, zloc);
          const double tp = d_igw(xloc, yloc, zloc, a.xlen / 3, a.ylen / 3, 5000, a.zlen, 0.01);
          const double t = th + tp;
          acc[4] += (rh * t - rh * th) * wt;
          acc[1] += 20 * rh * wt;
          if (!a.sim2d) acc[2] += 20 * rh * wt;
        }
      }
  if (a.noise_amp > 0) {
    const unsigned long long cell = ((unsigned long long)k * a.ny + j) * a.nx_global + (a.xoff + i);
    const unsigned long long base = a.seed * 0x100000001B3ULL;
    double nz_;
    if (a.noise_kind == 1) {  // Box-Muller: u1 in (0, 1], u2 in [0, 1)
      const double u1 = (double)((d_splitmix64(base + 2 * cell) >> 11) + 1) * (1.0 / 9007199254740992.0);
      const double u2 = (double)(d_splitmix64(base + 2 * cell + 1) >> 11) * (1.0 / 9007199254740992.0);
      nz_ = a.noise_amp * sqrt(-2.0 * log(u1)) * cos(6.283185307179586476925 * u2);
    } else {
      const double u = (double)(d_splitmix64(base + cell) >> 11) * (1.0 / 9007199254740992.0);
      nz_ = (2.0 * u - 1.0) * a.noise_amp;
    }
    acc[4] += a.dens_c[hs + k] * nz_;
  }
  if (a.state32) {  // FP32 context: value plane and a zeroed Kahan plane
#pragma unroll
    for (int l = 0; l < 5; l++) {
      a.state32[s + l * sv] = (float)acc[l];
      a.comp32[s + l * sv] = 0.f;
    }
  } else {
#pragma unroll
    for (int l = 0; l < 5; l++) a.state[s + l * sv] = acc[l];
  }
}

cudaError_t launch_init_state_fp64(const InitLaunch &L, cudaStream_t st) {
  InitArgs a;
  a.state = (double *)L.state;
  a.state32 = L.state32;
  a.comp32 = L.comp32;
  a.nx = L.nx; a.ny = L.ny; a.nz = L.nz; a.hs = L.hs; a.ord = L.ord;
  a.xoff = L.xoff; a.nx_global = L.nx_global > 0 ? L.nx_global : L.nx;
  a.dx = L.dx; a.dy = L.dy; a.dz = L.dz; a.xlen = L.xlen; a.ylen = L.ylen; a.zlen = L.zlen;
  a.data_spec = L.data_spec; a.sim2d = L.sim2d; a.kind = L.kind; a.shape = L.shape;
  a.x0 = L.x0; a.y0 = L.y0; a.z0 = L.z0; a.xrad = L.xrad; a.yrad = L.yrad; a.zrad = L.zrad;
  a.amp = L.amp; a.pwr = L.pwr; a.noise_amp = L.noise_amp; a.seed = L.seed; a.dens_c = L.dens_c;
  a.noise_kind = L.noise_kind;
  for (int m = 0; m < 9; m++) { a.pts[m] = m < L.ord ? L.pts[m] : 0; a.wts[m] = m < L.ord ? L.wts[m] : 0; }
  const long n = (long)L.nz * L.ny * L.nx;
  init_state_kernel<<<(unsigned)((n + 127) / 128), 128, 0, st>>>(a);
  return cudaGetLastError();
}

// ------------------------------------------------------------------------------------
// Spatial::initTracers (Spatial:505-560): per cell and tracer, the ord^3 GLL quadrature of
// rho_h * tval with the reference's three profiles (uniform 1; the 2 K linear ellipsoid of
// radius 2 km at (xlen/2, ylen/2, 2 km); the block indicator, integer-divided bounds);
// tracers beyond the third are zero. One thread per cell; tracers (ntr, nz+2hs, ny+2hs,
// nx+2hs) FP64, interior written.
// ------------------------------------------------------------------------------------
__global__ void init_tracers_kernel(InitArgs a, int ntr) {
  const long n = (long)a.nz * a.ny * a.nx;
  const long idx = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (idx >= n) return;
  const int i = idx % a.nx, j = (idx / a.nx) % a.ny, k = idx / ((long)a.nx * a.ny);
  const int hs = a.hs;
  const long sy = a.nx + 2 * hs, sz = (long)(a.ny + 2 * hs) * sy, sv = (long)(a.nz + 2 * hs) * sz;
  const long s = (hs + k) * sz + (hs + j) * sy + hs + i;
  const int ig = a.xoff + i;
  bool inside = k >= 1 * a.nz / 10 && k < 3 * a.nz / 10 && ig >= 4 * a.nx_global / 10 && ig < 6 * a.nx_global / 10;
  if (!a.sim2d) inside = inside && j >= 4 * a.ny / 10 && j < 6 * a.ny / 10;
  for (int l = 0; l < ntr; l++) {
    double acc = 0;
    if (l < 3) {
      for (int kk = 0; kk < a.ord; kk++)
        for (int jj = 0; jj < a.ord; jj++)
          for (int ii = 0; ii < a.ord; ii++) {
            const double zloc = (k + 0.5) * a.dz + a.pts[kk] * a.dz;
            const double yloc = a.sim2d ? a.ylen / 2 : (j + 0.5) * a.dy + a.pts[jj] * a.dy;
            const double xloc = (a.xoff + i + 0.5) * a.dx + a.pts[ii] * a.dx;
            const double wt = a.wts[kk] * a.wts[jj] * a.wts[ii];
            const double rh = d_const_theta_density(300, zloc);
            double tval;
            if (l == 0) tval = 1;
            else if (l == 1) tval = d_ellipsoid_linear(xloc, yloc, zloc, a.xlen / 2, a.ylen / 2, 2000, 2000, 2000, 2000, 2);
            else tval = inside ? 1 : 0;
            acc += rh * tval * wt;
          }
    }
    a.state[s + l * sv] = acc;
  }
}

cudaError_t launch_init_tracers_fp64(const InitLaunch &L, int ntr, cudaStream_t st) {
  InitArgs a;
  memset(&a, 0, sizeof a);
  a.state = (double *)L.state;
  a.nx = L.nx; a.ny = L.ny; a.nz = L.nz; a.hs = L.hs; a.ord = L.ord;
  a.xoff = L.xoff; a.nx_global = L.nx_global > 0 ? L.nx_global : L.nx;
  a.dx = L.dx; a.dy = L.dy; a.dz = L.dz; a.xlen = L.xlen; a.ylen = L.ylen; a.zlen = L.zlen;
  a.sim2d = L.sim2d;
  for (int m = 0; m < 9; m++) { a.pts[m] = m < L.ord ? L.pts[m] : 0; a.wts[m] = m < L.ord ? L.wts[m] : 0; }
  const long n = (long)L.nz * L.ny * L.nx;
  if (n == 0 || ntr == 0) return cudaSuccess;
  init_tracers_kernel<<<(unsigned)((n + 127) / 128), 128, 0, st>>>(a, ntr);
  return cudaGetLastError();
}

// ------------------------------------------------------------------------------------
// Diagnostics: FP64 interior sums x dV with a fixed reduction order (each block sums a
// fixed stride of cells, then one block adds the block partials in order), and a count
// of cells with a non-finite value or a non-positive total density.
// ------------------------------------------------------------------------------------
constexpr int kSumThreads = 256;

__device__ __forceinline__ double state_at(const void *state, int fp32, long plane, long g) {
  if (fp32) {
    const float *s = (const float *)state;
    return (double)s[g] - (double)s[g + plane];  // value minus Kahan compensation
  }
  return ((const double *)state)[g];
}

__global__ void __launch_bounds__(kSumThreads) state_sums_kernel(const void *state, int fp32, long plane, int nx,
                                                                  int ny, int nz, int hs, double *partials) {
  __shared__ double red[5][kSumThreads];
  const long n = (long)nz * ny * nx;
  const long sy = nx + 2 * hs, sz = (long)(ny + 2 * hs) * sy, sv = (long)(nz + 2 * hs) * sz;
  double acc[5] = {0., 0., 0., 0., 0.};
  for (long c = blockIdx.x * (long)kSumThreads + threadIdx.x; c < n; c += (long)gridDim.x * kSumThreads) {
    const int i = (int)(c % nx), j = (int)((c / nx) % ny), k = (int)(c / ((long)nx * ny));
    const long g = (hs + k) * sz + (hs + j) * sy + hs + i;
#pragma unroll
    for (int v = 0; v < 5; v++) acc[v] += state_at(state, fp32, plane, g + v * sv);
  }
#pragma unroll
  for (int v = 0; v < 5; v++) red[v][threadIdx.x] = acc[v];
  __syncthreads();
  for (int s = kSumThreads / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
#pragma unroll
      for (int v = 0; v < 5; v++) red[v][threadIdx.x] += red[v][threadIdx.x + s];
    }
    __syncthreads();
  }
  if (threadIdx.x < 5) partials[blockIdx.x * 5 + threadIdx.x] = red[threadIdx.x][0];
}

__global__ void state_sums_final_kernel(const double *partials, int nblk, double dv, double *out) {
  if (threadIdx.x < 5) {
    double s = 0.;
    for (int b = 0; b < nblk; b++) s += partials[b * 5 + threadIdx.x];
    out[threadIdx.x] = s * dv;
  }
}

cudaError_t launch_state_sums(const void *state, int fp32, long plane, int nx, int ny, int nz, int hs, double dv,
                              double *partials, int nblk, double *out, cudaStream_t st) {
  state_sums_kernel<<<nblk, kSumThreads, 0, st>>>(state, fp32, plane, nx, ny, nz, hs, partials);
  state_sums_final_kernel<<<1, 32, 0, st>>>(partials, nblk, dv, out);
  return cudaGetLastError();
}

__global__ void check_state_kernel(const void *state, int fp32, long plane, const double *dens_c, int nx, int ny,
                                   int nz, int hs, unsigned long long *count) {
  const long n = (long)nz * ny * nx;
  const long sy = nx + 2 * hs, sz = (long)(ny + 2 * hs) * sy, sv = (long)(nz + 2 * hs) * sz;
  unsigned long long bad = 0;
  for (long c = blockIdx.x * (long)blockDim.x + threadIdx.x; c < n; c += (long)gridDim.x * blockDim.x) {
    const int i = (int)(c % nx), j = (int)((c / nx) % ny), k = (int)(c / ((long)nx * ny));
    const long g = (hs + k) * sz + (hs + j) * sy + hs + i;
    bool ok = true;
#pragma unroll
    for (int v = 0; v < 5; v++) ok = ok && isfinite(state_at(state, fp32, plane, g + v * sv));
    ok = ok && (dens_c[hs + k] + state_at(state, fp32, plane, g)) > 0.0;
    bad += ok ? 0 : 1;
  }
  if (bad) atomicAdd(count, bad);
}

cudaError_t launch_check_state(const void *state, int fp32, long plane, const double *dens_c, int nx, int ny,
                               int nz, int hs, int nsm, unsigned long long *count, cudaStream_t st) {
  const long n = (long)nz * ny * nx;
  long blocks = (n + 255) / 256;
  if (blocks > (long)nsm * 8) blocks = (long)nsm * 8;
  if (blocks < 1) blocks = 1;
  check_state_kernel<<<(unsigned)blocks, 256, 0, st>>>(state, fp32, plane, dens_c, nx, ny, nz, hs, count);
  return cudaGetLastError();
}

// Output diagnostics of Spatial::output (Spatial:1744-1778), FP64 from either state form:
// out[f][k][j][i], f = dens_pert, u, v, w, pot_temp_pert, pressure_pert. Same operations
// and order as the reference (IEEE division, no contraction in this translation unit,
// the correctly rounded pow for C0*(r*t)^gamma). One thread per cell: x along the block,
// y and z along the grid (no index division), a streaming kernel bound by its 88 bytes
// per cell.
constexpr int kOutX = 128;
__global__ void __launch_bounds__(kOutX) output_fields_kernel(const void *state, int fp32, long plane,
                                                             const double *dens_c, const double *denstheta_c,
                                                             const double *pres_c, int nx, int ny, int nz, int hs,
                                                             double *out) {
  const int i = blockIdx.x * kOutX + threadIdx.x, j = blockIdx.y, k = blockIdx.z;
  if (i >= nx) return;
  const long n = (long)nz * ny * nx;
  const long c = ((long)k * ny + j) * nx + i;
  const long sy = nx + 2 * hs, sz = (long)(ny + 2 * hs) * sy, sv = (long)(nz + 2 * hs) * sz;
  const long g = (hs + k) * sz + (hs + j) * sy + hs + i;
  const double dk = dens_c[hs + k], dtk = denstheta_c[hs + k], pk = pres_c[hs + k];
  const double rp = state_at(state, fp32, plane, g);
  const double mu = state_at(state, fp32, plane, g + 1 * sv);
  const double mv = state_at(state, fp32, plane, g + 2 * sv);
  const double mw = state_at(state, fp32, plane, g + 3 * sv);
  const double mt = state_at(state, fp32, plane, g + 4 * sv);
  const double r = rp + dk;
  out[c] = rp;
  out[n + c] = mu / r;
  out[2 * n + c] = mv / r;
  out[3 * n + c] = mw / r;
  const double t = (mt + dtk) / r;
  out[4 * n + c] = t - dtk / dk;
  const double p = C0 * pow_cr(r * t, GAMMA);
  out[5 * n + c] = p - pk;
}

cudaError_t launch_output_fields(const void *state, int fp32, long plane, const double *dens_c,
                                 const double *denstheta_c, const double *pres_c, int nx, int ny, int nz, int hs,
                                 int nsm, double *out, cudaStream_t st) {
  (void)nsm;
  if ((long)nz * ny * nx == 0) return cudaSuccess;
  const dim3 grid((nx + kOutX - 1) / kOutX, ny, nz);
  output_fields_kernel<<<grid, kOutX, 0, st>>>(state, fp32, plane, dens_c, denstheta_c, pres_c, nx, ny, nz, hs, out);
  return cudaGetLastError();
}

// Tracer fields of Spatial::output (Spatial:1778-1783): out[tr][k][j][i] =
// tracers(tr, hs+k, hs+j, hs+i) / (rho'(k,j,i) + hyDensCells(hs+k)). Launched like
// output_fields_kernel.
__global__ void __launch_bounds__(kOutX) tracer_fields_kernel(const void *state, int fp32, long plane,
                                                             const double *dens_c, const double *tracers, int ntr,
                                                             int nx, int ny, int nz, int hs, double *out) {
  const int i = blockIdx.x * kOutX + threadIdx.x, j = blockIdx.y, k = blockIdx.z;
  if (i >= nx) return;
  const long n = (long)nz * ny * nx;
  const long c = ((long)k * ny + j) * nx + i;
  const long sy = nx + 2 * hs, sz = (long)(ny + 2 * hs) * sy, sv = (long)(nz + 2 * hs) * sz;
  const long g = (hs + k) * sz + (hs + j) * sy + hs + i;
  const double r = state_at(state, fp32, plane, g) + dens_c[hs + k];
  for (int t = 0; t < ntr; t++) out[t * n + c] = tracers[t * sv + g] / r;
}

cudaError_t launch_tracer_fields(const void *state, int fp32, long plane, const double *dens_c,
                                 const double *tracers, int ntr, int nx, int ny, int nz, int hs, int nsm, double *out,
                                 cudaStream_t st) {
  (void)nsm;
  const long n = (long)nz * ny * nx;
  if (n == 0 || ntr == 0) return cudaSuccess;
  const dim3 grid((nx + kOutX - 1) / kOutX, ny, nz);
  tracer_fields_kernel<<<grid, kOutX, 0, st>>>(state, fp32, plane, dens_c, tracers, ntr, nx, ny, nz, hs, out);
  return cudaGetLastError();
}

// Halo columns a slab sends to its neighbours before an x split: the hs+1 first (side 0)
// and last (side 1) interior columns of each variable, [2][5][nz][ny][hs+1].
template <class T>
__global__ void slab_pack_kernel(const T *state, int nx, int ny, int nz, int hs, T *send) {
  const int w = hs + 1;
  const long n = 2L * 5 * nz * ny * w;
  const long sy = nx + 2 * hs, sz = (long)(ny + 2 * hs) * sy, sv = (long)(nz + 2 * hs) * sz;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < n; t += (long)gridDim.x * blockDim.x) {
    const int c = (int)(t % w);
    long r = t / w;
    const int j = (int)(r % ny); r /= ny;
    const int k = (int)(r % nz); r /= nz;
    const int v = (int)(r % 5);
    const int side = (int)(r / 5);
    const int i = side == 0 ? c : nx - w + c;
    send[t] = state[v * sv + (hs + k) * sz + (hs + j) * sy + hs + i];
  }
}

cudaError_t launch_slab_pack(const void *state, int esz, int nx, int ny, int nz, int hs, void *send, cudaStream_t st) {
  const long n = 2L * 5 * nz * ny * (hs + 1);
  const unsigned blocks = (unsigned)((n + 255) / 256 < 4096 ? (n + 255) / 256 : 4096);
  if (esz == 8) slab_pack_kernel<double><<<blocks, 256, 0, st>>>((const double *)state, nx, ny, nz, hs, (double *)send);
  else slab_pack_kernel<float><<<blocks, 256, 0, st>>>((const float *)state, nx, ny, nz, hs, (float *)send);
  return cudaGetLastError();
}

// Device math self-test: out[i] = pow(x[i], y) by the library's pow_cr (mode 0) or by
// the CUDA math library (mode 1); exp_cr(x[i]) (mode 2); x[i] / x[n+i] through the shared
// reciprocal (mode 3) or by IEEE division (mode 4).
__global__ void selftest_pow_kernel(const double *x, double y, double *out, long n, int mode) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (mode == 3) out[i] = divr(x[i], make_rcp<double>(x[n + i]));
  else if (mode == 4) out[i] = x[i] / x[n + i];
  else out[i] = mode == 0 ? pow_cr(x[i], y) : (mode == 1 ? pow(x[i], y) : exp_cr(x[i]));
}

cudaError_t launch_selftest_pow(const double *x, double y, double *out, long n, int mode, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  selftest_pow_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(x, y, out, n, mode);
  return cudaGetLastError();
}

// FMA throughput microbenchmark: 8 independent FMA chains per thread, `iters` rounds.
// The sink write keeps the chains live. 2 flops per FMA.
template <class T>
__global__ void __launch_bounds__(256) fma_peak_kernel(T *sink, int iters, T a, T b) {
  T x[8];
#pragma unroll
  for (int c = 0; c < 8; c++) x[c] = (T)(threadIdx.x + c) * (T)1e-3;
  for (int it = 0; it < iters; it++) {
#pragma unroll
    for (int c = 0; c < 8; c++) x[c] = fma(x[c], a, b);
  }
  T s = 0;
#pragma unroll
  for (int c = 0; c < 8; c++) s += x[c];
  if (s == (T)123.456) sink[threadIdx.x] = s;
}

// The same with sm_100's paired FP32 FMA (one instruction, two lanes): 4 flops each.
__global__ void __launch_bounds__(256) fma2_peak_kernel(float *sink, int iters, float a, float b) {
  float2 x[8];
#pragma unroll
  for (int c = 0; c < 8; c++) x[c] = make_float2((threadIdx.x + c) * 1e-3f, (threadIdx.x + c + 1) * 1e-3f);
  const float2 a2 = make_float2(a, a), b2 = make_float2(b, b);
  for (int it = 0; it < iters; it++) {
#pragma unroll
    for (int c = 0; c < 8; c++) x[c] = __ffma2_rn(x[c], a2, b2);
  }
  float s = 0;
#pragma unroll
  for (int c = 0; c < 8; c++) s += x[c].x + x[c].y;
  if (s == 123.456f) sink[threadIdx.x] = s;
}

// kind 0: FP64 FMA, 1: FP32 FMA, 2: paired FP32 FMA.
cudaError_t run_fma_peak(int kind, int nsm, double *tflops) {
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  void *sink = nullptr;
  cudaError_t e = cudaMalloc(&sink, 256 * sizeof(double));
  if (e != cudaSuccess) return e;
  const int blocks = nsm * 8, threads = 256;
  const int iters = kind == 0 ? 8192 : (kind == 1 ? 16384 : 8192);
  for (int rep = 0; rep < 2; rep++) {  // first launch warms up
    cudaEventRecord(e0);
    if (kind == 1) fma_peak_kernel<float><<<blocks, threads>>>((float *)sink, iters, 0.999999f, 1e-7f);
    else if (kind == 2) fma2_peak_kernel<<<blocks, threads>>>((float *)sink, iters, 0.999999f, 1e-7f);
    else fma_peak_kernel<double><<<blocks, threads>>>((double *)sink, iters, 0.999999999, 1e-9);
    cudaEventRecord(e1);
  }
  e = cudaEventSynchronize(e1);
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(sink);
  if (e != cudaSuccess) return e;
  e = cudaGetLastError();
  const double flops_per_inst = kind == 2 ? 4.0 : 2.0;
  *tflops = flops_per_inst * 8.0 * (double)iters * blocks * threads / (ms * 1e-3) / 1e12;
  return e;
}

cudaError_t upload_tables_fp64(int ord, const void *tab, size_t bytes) {
  if (ord == 5) return cudaMemcpyToSymbol(c_tab5, tab, bytes);
  return cudaMemcpyToSymbol(c_tab9, tab, bytes);
}

}  // namespace awfl
