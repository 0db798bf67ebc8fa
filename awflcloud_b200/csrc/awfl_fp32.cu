// FP32 precision form of the AWFL Euler-3D ADER/WENO step, sm_100a: sweep, apply, CFL
// and conversion kernels. The scheme's FP32 arithmetic and the sweep policy P32 are in
// awfl_fp32.cuh.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "awfl_fp32.cuh"

namespace awfl {

static_assert(sizeof(TmaMap) == sizeof(CUtensorMap) && alignof(TmaMap) >= 64, "TmaMap holds a CUtensorMap");

namespace {
using EncodeTiledFn = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                   const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
// The driver's tensor-map encoder, looked up once through the runtime (no libcuda link).
EncodeTiledFn encoder() {
  static EncodeTiledFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  });
  return fn;
}
}  // namespace

void warm_tma_encoder() { (void)encoder(); }

bool prepare_sweep_map32(SweepArgs32 &A, int ord, int dir, int C, int W) {
  const int hs = (ord - 1) / 2;
  const unsigned rw = (unsigned)tma_ring_pitch_of(ord, C, W, 4);
  const unsigned box[3] = {dir == 0 ? (unsigned)C : rw, dir == 0 ? (unsigned)W : (dir == 1 ? (unsigned)C : 1u),
                           dir == 2 ? (unsigned)C : 1u};
  A.tma = encode_state_map32(&A.tmap, A.state, A.nx + 2 * hs, A.ny + 2 * hs, A.nz + 2 * hs, box) ? 1 : 0;
  return A.tma != 0;
}

bool encode_state_map32(TmaMap *m, const float *state, int xe, int ye, int ze, const unsigned (&box)[3]) {
  if (reinterpret_cast<uintptr_t>(state) % 16 != 0 || ((long)xe * 4) % 16 != 0) return false;
  for (int d = 0; d < 3; d++)
    if (box[d] < 1 || box[d] > 256) return false;
  if ((box[0] * 4u) % 16 != 0) return false;
  EncodeTiledFn fn = encoder();
  if (!fn) return false;
  const cuuint64_t dims[3] = {(cuuint64_t)xe, (cuuint64_t)ye, (cuuint64_t)5 * ze};
  const cuuint64_t strides[2] = {(cuuint64_t)xe * 4, (cuuint64_t)xe * ye * 4};
  const cuuint32_t bx[3] = {box[0], box[1], box[2]}, es[3] = {1, 1, 1};
  CUtensorMap t;
  const CUresult r = fn(&t, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float *>(state), dims, strides, bx, es,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return false;
  static_assert(sizeof t == sizeof *m, "tensor map size");
  __builtin_memcpy(m, &t, sizeof t);
  return true;
}

cudaError_t launch_sweep_fp32(int ord, int dir, const SweepArgs32 &A, cudaStream_t st) {
  return launch_sweep_any<P32>(ord, dir, A, st);
}

// Unfused Kahan apply (Temporal_ader.h:63-65) for FP32 states.
__global__ void apply32_kernel(float *state, float *comp, const float *tend, float dt, int nx, int ny, int nz, int hs) {
  const long n = 5L * nz * ny * nx;
  for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < n; idx += (long)gridDim.x * blockDim.x) {
    long r = idx;
    const int i = r % nx; r /= nx;
    const int j = r % ny; r /= ny;
    const int k = r % nz; r /= nz;
    const int l = (int)r;
    const long s = (((long)l * (nz + 2 * hs) + hs + k) * (ny + 2 * hs) + hs + j) * (nx + 2 * hs) + hs + i;
    const float y = dt * tend[idx] - comp[s];
    const float t = state[s] + y;
    comp[s] = __fsub_rn(__fsub_rn(t, state[s]), y);
    state[s] = t;
  }
}

cudaError_t launch_apply_fp32(float *state, float *comp, const float *tend, float dt, int nx, int ny, int nz, int hs,
                              int nsm, cudaStream_t st) {
  const long n = 5L * nz * ny * nx;
  long blocks = (n + 255) / 256;
  if (blocks > (long)nsm * 8) blocks = (long)nsm * 8;
  if (blocks < 1) blocks = 1;
  apply32_kernel<<<(unsigned)blocks, 256, 0, st>>>(state, comp, tend, dt, nx, ny, nz, hs);
  return cudaGetLastError();
}

// CFL time step of an FP32 state, computed in FP64 (Spatial:169-183).
__global__ void cfl32_kernel(const float *state, const double *dens_c, const double *denstheta_c, double cfl, double dx,
                             double dy, double dz, int nx, int ny, int nz, int hs, unsigned long long *out) {
  __shared__ double red[256];
  double best = __longlong_as_double(0x7ff0000000000000LL);
  const long n = (long)nz * ny * nx;
  const long sy = nx + 2 * hs, sz = (long)(ny + 2 * hs) * sy, sv = (long)(nz + 2 * hs) * sz;
  for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < n; idx += (long)gridDim.x * blockDim.x) {
    const int i = idx % nx;
    const int j = (idx / nx) % ny;
    const int k = idx / ((long)nx * ny);
    const long s = (hs + k) * sz + (hs + j) * sy + hs + i;
    const double r = (double)state[s] + dens_c[hs + k];
    const double u = (double)state[s + sv] / r;
    const double v = (double)state[s + 2 * sv] / r;
    const double w = (double)state[s + 3 * sv] / r;
    const double t = ((double)state[s + 4 * sv] + denstheta_c[hs + k]) / r;
    const double p = C0 * pow_cr(r * t, GAMMA);
    const double cs = sqrt(GAMMA * p / r);
    const double udt = cfl * dx / fmax(fabs(u - cs), fabs(u + cs));
    const double vdt = cfl * dy / fmax(fabs(v - cs), fabs(v + cs));
    const double wdt = cfl * dz / fmax(fabs(w - cs), fabs(w + cs));
    best = fmin(best, fmin(fmin(udt, vdt), wdt));
  }
  red[threadIdx.x] = best;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s && red[threadIdx.x + s] < red[threadIdx.x]) red[threadIdx.x] = red[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) atomicMin(out, (unsigned long long)__double_as_longlong(red[0]));
}

cudaError_t launch_cfl_fp32(const float *state, const double *dens_c, const double *denstheta_c, double cfl, double dx,
                            double dy, double dz, int nx, int ny, int nz, int hs, int nsm, unsigned long long *d_out,
                            cudaStream_t st) {
  const long n = (long)nz * ny * nx;
  long blocks = (n + 255) / 256;
  if (blocks > (long)nsm * 8) blocks = (long)nsm * 8;
  if (blocks < 1) blocks = 1;
  cfl32_kernel<<<(unsigned)blocks, 256, 0, st>>>(state, dens_c, denstheta_c, cfl, dx, dy, dz, nx, ny, nz, hs, d_out);
  return cudaGetLastError();
}

// FP64 state -> FP32 state (value plane) and zeroed compensation plane.
__global__ void to_fp32_kernel(const double *src, float *dst, float *comp, long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    dst[i] = (float)src[i];
    comp[i] = 0.f;
  }
}

cudaError_t launch_to_fp32(const double *src, float *dst, float *comp, long n, int nsm, cudaStream_t st) {
  long blocks = (n + 255) / 256;
  if (blocks > (long)nsm * 16) blocks = (long)nsm * 16;
  if (blocks < 1) blocks = 1;
  to_fp32_kernel<<<(unsigned)blocks, 256, 0, st>>>(src, dst, comp, n);
  return cudaGetLastError();
}

cudaError_t upload_tables_fp32(int ord, const double *recon, const double *c2g, const double *s2g,
                               const double *deriv, const double *idl, double sigma, const double *wts) {
  return upload_tables32_here(ord, recon, c2g, s2g, deriv, idl, sigma, wts);
}

}  // namespace awfl
