// Allocation-free variant of the CFL time step (awfl_cfl_noalloc in include/awfl.h).
//
// awfl_cfl reduces the per-cell time steps into a device word that its context allocated
// with cudaMalloc. Some callers cannot call cudaMalloc at all: a host application whose
// device memory is handed out by its own arena/pool and which forbids any other
// allocation, or a time-critical loop that cannot afford the implicit device
// synchronisation cudaMalloc may cause. For them this entry point needs no context and
// allocates nothing: the caller passes the state and the two hydrostatic background
// columns it already holds on the device, and the reduction's scratch is a file-scope
// static device array of fixed size (kMaxPartials + 1 doubles = 512 KiB), which every GPU
// that loads the library holds until the process exits.
//
// The per-cell arithmetic is the same as awfl_cfl's (Spatial_euler3d_cons_expl_cart_fv_
// Agrid.h:169-183, with the library's correctly rounded pow), and the minimum is order
// independent, so both entry points return the same value.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "../../include/awfl.h"
#include "awfl_internal.h"
#include "awfl_pow.cuh"

namespace awfl {
namespace {

constexpr int kCflBlock = 256;          // cells per partial minimum
constexpr long kMaxPartials = 65536;    // => at most 16,777,216 cells per call

// Partial minima [0, kMaxPartials) and the final minimum at [kMaxPartials].
// Shared by every call on a device and left holding the last call's values; nothing in
// it needs to start at zero (pass 1 writes every partial it uses, pass 2 the final slot).
static __device__ __align__(256) double g_cfl_scratch[kMaxPartials + 1];

std::mutex g_scratch_mutex;
double *g_scratch_ptr[256];  // device address of g_cfl_scratch, per device, set on first use

__global__ void __launch_bounds__(kCflBlock) cfl_partials_kernel(
    const double *state, const double *dens_c, const double *denstheta_c, double cfl, double dx, double dy,
    double dz, int nx, int ny, int nz, int hs, double *partials) {
  __shared__ double red[kCflBlock];
  const long n = (long)nz * ny * nx;
  const long idx = blockIdx.x * (long)kCflBlock + threadIdx.x;
  double best = __longlong_as_double(0x7ff0000000000000LL);  // +inf
  if (idx < n) {
    const long sy = nx + 2 * hs, sz = (long)(ny + 2 * hs) * sy, sv = (long)(nz + 2 * hs) * sz;
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
    best = m1 < wdt ? m1 : wdt;
  }
  red[threadIdx.x] = best;
  __syncthreads();
  for (int st = kCflBlock / 2; st > 0; st >>= 1) {
    if (threadIdx.x < st && red[threadIdx.x + st] < red[threadIdx.x]) red[threadIdx.x] = red[threadIdx.x + st];
    __syncthreads();
  }
  if (threadIdx.x == 0) partials[blockIdx.x] = red[0];
}

__global__ void __launch_bounds__(1024) cfl_final_kernel(const double *partials, long np, double *out) {
  __shared__ double red[1024];
  double best = __longlong_as_double(0x7ff0000000000000LL);
  for (long b = threadIdx.x; b < np; b += 1024) best = partials[b] < best ? partials[b] : best;
  red[threadIdx.x] = best;
  __syncthreads();
  for (int st = 512; st > 0; st >>= 1) {
    if (threadIdx.x < st && red[threadIdx.x + st] < red[threadIdx.x]) red[threadIdx.x] = red[threadIdx.x + st];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = red[0];
}

}  // namespace
}  // namespace awfl

using namespace awfl;

extern "C" int awfl_cfl_noalloc(const awfl_config *cfg, const void *d_state, const void *d_hy_dens_cells,
                                const void *d_hy_denstheta_cells, double cfl, double *h_dt, void *stream) {
  char msg[256];
  if (!cfg || !d_state || !d_hy_dens_cells || !d_hy_denstheta_cells || !h_dt) {
    set_unbound_error("awfl_cfl_noalloc: NULL argument");
    return AWFL_ERR_ARG;
  }
  if (cfg->ord != 5 && cfg->ord != 9) {
    set_unbound_error("awfl_cfl_noalloc: ord must be 5 or 9");
    return AWFL_ERR_ARG;
  }
  if (cfg->precision != AWFL_FP64) {
    set_unbound_error("awfl_cfl_noalloc: only FP64 states are supported");
    return AWFL_ERR_ARG;
  }
  if (cfg->nx < 1 || cfg->ny < 1 || cfg->nz < 1 || !(cfg->xlen > 0) || !(cfg->ylen > 0) || !(cfg->zlen > 0) ||
      !(cfl > 0)) {
    set_unbound_error("awfl_cfl_noalloc: grid sizes, lengths and cfl must be positive");
    return AWFL_ERR_ARG;
  }
  const long cells = (long)cfg->nx * cfg->ny * cfg->nz;
  const long np = (cells + kCflBlock - 1) / kCflBlock;
  if (np > kMaxPartials) {
    snprintf(msg, sizeof msg,
             "awfl_cfl_noalloc: %ld cells exceed the %ld-cell limit of its static scratch (use awfl_cfl)",
             cells, kMaxPartials * kCflBlock);
    set_unbound_error(msg);
    return AWFL_ERR_ARG;
  }
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 256) {
    set_unbound_error("awfl_cfl_noalloc: no current CUDA device");
    return AWFL_ERR_CUDA;
  }
  double *scratch;
  {
    // First call on a device: look up the device address of the static array (with that
    // device current). Do this first call before any stream capture begins.
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (!g_scratch_ptr[dev]) {
      void *p = nullptr;
      cudaError_t e = cudaGetSymbolAddress(&p, g_cfl_scratch);
      if (e != cudaSuccess || !p) {
        snprintf(msg, sizeof msg, "awfl_cfl_noalloc: cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
        set_unbound_error(msg);
        return AWFL_ERR_CUDA;
      }
      g_scratch_ptr[dev] = static_cast<double *>(p);
    }
    scratch = g_scratch_ptr[dev];
  }
  const int hs = (cfg->ord - 1) / 2;
  cudaStream_t st = (cudaStream_t)stream;
  cfl_partials_kernel<<<(unsigned)np, kCflBlock, 0, st>>>(
      (const double *)d_state, (const double *)d_hy_dens_cells, (const double *)d_hy_denstheta_cells, cfl,
      cfg->xlen / cfg->nx, cfg->ylen / cfg->ny, cfg->zlen / cfg->nz, cfg->nx, cfg->ny, cfg->nz, hs, scratch);
  cfl_final_kernel<<<1, 1024, 0, st>>>(scratch, np, scratch + kMaxPartials);
  cudaError_t e = cudaGetLastError();
  double dt = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&dt, scratch + kMaxPartials, sizeof dt, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    snprintf(msg, sizeof msg, "awfl_cfl_noalloc: %s", cudaGetErrorString(e));
    set_unbound_error(msg);
    return AWFL_ERR_CUDA;
  }
  if (!(dt > 0) || !std::isfinite(dt)) {
    snprintf(msg, sizeof msg, "awfl_cfl_noalloc: non-finite or non-positive time step (%g)", dt);
    set_unbound_error(msg);
    return AWFL_ERR_STATE;
  }
  *h_dt = dt;
  return AWFL_OK;
}
