// Ensemble (batched) sweeps of the FP64 parity path: the persistent kernels of
// awfl_ens.cuh instantiated for the P64 policy, sm_100a. Same flags as awfl_fp64.cu
// (--fmad=false), so every member stays bit-identical to the reference arithmetic.
#include <cuda_runtime.h>

#include "awfl_ens.cuh"
#include "awfl_p64.cuh"

namespace awfl {

cudaError_t ens_run_fp64(int ord, int dir, int shape, const EnsList<SweepArgs> *E, int grid, int *occ,
                         cudaStream_t st) {
  return ens_run<P64>(ord, dir, shape, E, grid, occ, st);
}

cudaError_t upload_tables_ens64(int ord, const void *tab, size_t bytes) {
  if (ord == 5) return cudaMemcpyToSymbol(c_tab5, tab, bytes);
  return cudaMemcpyToSymbol(c_tab9, tab, bytes);
}

}  // namespace awfl
