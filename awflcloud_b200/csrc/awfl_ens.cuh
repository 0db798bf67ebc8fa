// Batched (ensemble) form of the line sweep: one persistent kernel per split stage runs
// the sweep tiles of every member of an ensemble whose members have different grid sizes.
//
// The work of one direction is a list of tiles (a tile = W lines of one member, the unit
// one CTA of the single-grid sweep handles): members sorted by line length, longest first,
// each contributing nbx * nby tiles. A grid of (occupancy x SM count) CTAs strides over
// the tile list; each tile runs exactly the single-grid sweep body (sweep_tile), so an FP64
// member's result is bit-identical to stepping it alone, whatever the tile shape (FP32:
// equal up to where the compiler contracts multiply-adds).
//
// Tile shapes (C cells per chunk, W lines per CTA) are candidates for the autotuner
// (awfl_ensemble_tune): per order and direction, EnsShapes lists them; entry 0 is used
// until the ensemble is tuned.
#pragma once

#include <cuda_runtime.h>

#include "awfl_sweep.cuh"

namespace awfl {

template <class Args> struct EnsList {
  const Args *args;    // per listed member, in work order
  const long *prefix;  // n + 1 entries: first tile of each listed member, then the total
  const int *nbx;      // tiles across lines; tile t of a member is (t % nbx, t / nbx)
  int n;               // listed members
  long total;          // tiles
};

// CTAs per SM the register budget must allow: the policy's own figure, or, where the
// including unit defines AWFL_ENS_THREADS_PER_SM_ORD5, that many threads per SM at ord 5
#ifndef AWFL_ENS_THREADS_PER_SM_ORD5
#define AWFL_ENS_THREADS_PER_SM_ORD5 0
#endif
template <class P, int ORD, int C, int W> constexpr int ens_min_blocks() {
  return (ORD == 5 && AWFL_ENS_THREADS_PER_SM_ORD5 > 0) ? AWFL_ENS_THREADS_PER_SM_ORD5 / (C * W) : P::min_blocks(ORD);
}

template <class P, int ORD, int DIR, int C, int W>
__global__ void __launch_bounds__(C *W, (ens_min_blocks<P, ORD, C, W>())) ens_sweep_kernel(EnsList<typename P::Args> E) {
  __shared__ typename P::Args sA;
  for (long t = blockIdx.x; t < E.total; t += gridDim.x) {
    int lo = 0, hi = E.n - 1;
    while (lo < hi) {  // last member whose first tile is <= t
      const int mid = (lo + hi + 1) >> 1;
      if (E.prefix[mid] <= t) lo = mid;
      else hi = mid - 1;
    }
    const long local = t - E.prefix[lo];
    const int nbx = E.nbx[lo];
    if (threadIdx.x == 0 && threadIdx.y == 0) sA = E.args[lo];
    __syncthreads();
    if constexpr (P::kTmaRing) {
      // the member's tensor map, in the list in global memory (nullptr: cp.async only)
      const void *tm = P::tma_map_global(sA, E.args + lo);
      if (tm && threadIdx.x == 0 && threadIdx.y == 0)  // the issuing thread sees the host-written map
        asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;\n" ::"l"(tm) : "memory");
      sweep_tile<P, ORD, DIR, C, W, true>(sA, (int)(local % nbx), (int)(local / nbx), tm);
    } else {
      sweep_tile<P, ORD, DIR, C, W>(sA, (int)(local % nbx), (int)(local / nbx));
    }
    __syncthreads();  // the next tile reuses sA and the shared-memory ring
  }
}

template <int ORD, int DIR> struct EnsShapes;
template <> struct EnsShapes<5, 0> {
  static constexpr int n = 4;
  static constexpr int C[4] = {32, 32, 8, 16}, W[4] = {4, 2, 16, 8};
};
template <> struct EnsShapes<5, 1> {
  static constexpr int n = 4;
  static constexpr int C[4] = {4, 8, 4, 8}, W[4] = {32, 16, 16, 8};
};
template <> struct EnsShapes<5, 2> {
  static constexpr int n = 4;
  static constexpr int C[4] = {4, 8, 4, 8}, W[4] = {32, 16, 16, 8};
};
template <> struct EnsShapes<9, 0> {
  static constexpr int n = 2;
  static constexpr int C[2] = {32, 32}, W[2] = {2, 4};
};
template <> struct EnsShapes<9, 1> {
  static constexpr int n = 2;
  static constexpr int C[2] = {8, 8}, W[2] = {16, 8};
};
template <> struct EnsShapes<9, 2> {
  static constexpr int n = 2;
  static constexpr int C[2] = {8, 8}, W[2] = {16, 8};
};

// Launch, occupancy and shape queries for one policy, order, direction and shape index.
template <class P, int ORD, int DIR, int I> struct EnsOne {
  static constexpr int C = EnsShapes<ORD, DIR>::C[I], W = EnsShapes<ORD, DIR>::W[I];
  static cudaError_t launch(const EnsList<typename P::Args> &E, int grid, cudaStream_t st) {
    dim3 block(DIR == 0 ? C : W, DIR == 0 ? W : C);
    ens_sweep_kernel<P, ORD, DIR, C, W><<<grid, block, 0, st>>>(E);
    return cudaGetLastError();
  }
  static cudaError_t occupancy(int *blocks_per_sm) {
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, ens_sweep_kernel<P, ORD, DIR, C, W>, C * W, 0);
  }
};

template <class P, int ORD, int DIR>
cudaError_t ens_dispatch(int shape, const EnsList<typename P::Args> *E, int grid, int *occ, cudaStream_t st) {
  static_assert(EnsShapes<ORD, DIR>::n == 2 || EnsShapes<ORD, DIR>::n == 4, "shape table");
  if (shape < 0 || shape >= EnsShapes<ORD, DIR>::n) return cudaErrorInvalidValue;
#define AWFL_ENS_CASE(I)                                                       \
  case I:                                                                      \
    if constexpr (I < EnsShapes<ORD, DIR>::n) {                                \
      if (occ) return EnsOne<P, ORD, DIR, I>::occupancy(occ);                  \
      return EnsOne<P, ORD, DIR, I>::launch(*E, grid, st);                     \
    }                                                                          \
    break;
  switch (shape) {
    AWFL_ENS_CASE(0)
    AWFL_ENS_CASE(1)
    AWFL_ENS_CASE(2)
    AWFL_ENS_CASE(3)
  }
#undef AWFL_ENS_CASE
  return cudaErrorInvalidValue;
}

// One entry point per policy: launch (occ == nullptr) or occupancy query (occ != nullptr).
template <class P>
cudaError_t ens_run(int ord, int dir, int shape, const EnsList<typename P::Args> *E, int grid, int *occ,
                    cudaStream_t st) {
  if (ord == 5) {
    if (dir == 0) return ens_dispatch<P, 5, 0>(shape, E, grid, occ, st);
    if (dir == 1) return ens_dispatch<P, 5, 1>(shape, E, grid, occ, st);
    return ens_dispatch<P, 5, 2>(shape, E, grid, occ, st);
  }
  if (dir == 0) return ens_dispatch<P, 9, 0>(shape, E, grid, occ, st);
  if (dir == 1) return ens_dispatch<P, 9, 1>(shape, E, grid, occ, st);
  return ens_dispatch<P, 9, 2>(shape, E, grid, occ, st);
}

inline int ens_num_shapes(int ord, int dir) {
  if (ord == 5) return dir == 0 ? EnsShapes<5, 0>::n : EnsShapes<5, 1>::n;
  return dir == 0 ? EnsShapes<9, 0>::n : EnsShapes<9, 1>::n;
}
inline void ens_shape(int ord, int dir, int i, int *C, int *W) {
  if (ord == 5) {
    if (dir == 0) { *C = EnsShapes<5, 0>::C[i]; *W = EnsShapes<5, 0>::W[i]; }
    else if (dir == 1) { *C = EnsShapes<5, 1>::C[i]; *W = EnsShapes<5, 1>::W[i]; }
    else { *C = EnsShapes<5, 2>::C[i]; *W = EnsShapes<5, 2>::W[i]; }
  } else {
    if (dir == 0) { *C = EnsShapes<9, 0>::C[i]; *W = EnsShapes<9, 0>::W[i]; }
    else if (dir == 1) { *C = EnsShapes<9, 1>::C[i]; *W = EnsShapes<9, 1>::W[i]; }
    else { *C = EnsShapes<9, 2>::C[i]; *W = EnsShapes<9, 2>::W[i]; }
  }
}

}  // namespace awfl
