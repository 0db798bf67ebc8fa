// Ensemble (batched) sweeps of the FP32 form: the persistent kernels of awfl_ens.cuh
// instantiated for the P32 policy, sm_100a. Same flags as awfl_fp32.cu.
#include <cuda_runtime.h>

// 512 threads' registers per SM at ord 5 (at most 128 a thread): the persistent sweeps then
// hold 4 CTAs of 128 threads per SM like the single-grid FP32 sweep, instead of 3 at the
// compiler's 142-150 registers
#ifndef AWFL_ENS_THREADS_PER_SM_ORD5
#define AWFL_ENS_THREADS_PER_SM_ORD5 512
#endif
#include "awfl_ens.cuh"
#include "awfl_fp32.cuh"

namespace awfl {

cudaError_t ens_run_fp32(int ord, int dir, int shape, const EnsList<SweepArgs32> *E, int grid, int *occ,
                         cudaStream_t st) {
  return ens_run<P32>(ord, dir, shape, E, grid, occ, st);
}

cudaError_t upload_tables_ens32(int ord, const double *recon, const double *c2g, const double *s2g,
                                const double *deriv, const double *idl, double sigma, const double *wts) {
  return upload_tables32_here(ord, recon, c2g, s2g, deriv, idl, sigma, wts);
}

}  // namespace awfl
