// Reverse sweeps of the discrete adjoint (FP64), sm_100a.
//
// One directional split's adjoint runs as five grid-stride kernels over the per-thread
// functions of awfl_adj_split.h:
//   adj_edges_kernel   cell        recompute level-0 values and edges (linearisation point)
//   adj_face_kernel    face        flux adjoint -> Riemann reverse -> (lqL, lqR)
//   adj_cell_kernel    cell        edge adjoints -> ADER reverse -> level-0 adjoints
//   adj_weno_kernel    var x cell  level-0 adjoints -> WENO reverse -> stencil adjoints
//   adj_gather_kernel  cell        lam += the stencil adjoints that read the cell
//                                  (deterministic)
// The arithmetic is plain FP64 with contracted multiply-adds; it is a derivative, not a
// replay of the reference's rounding.
#include <cuda_runtime.h>

#include "awfl_adj_split.h"
#include "awfl_internal.h"

namespace awfl {

static __constant__ Tables<5> a_tab5;
static __constant__ Tables<9> a_tab9;

template <int ORD> __device__ __forceinline__ const Tables<ORD> &atab();
template <> __device__ __forceinline__ const Tables<5> &atab<5>() { return a_tab5; }
template <> __device__ __forceinline__ const Tables<9> &atab<9>() { return a_tab9; }

constexpr int kAdjThreads = 128;
// CTAs per SM requested of the two largest reverse kernels at ord 5 (register bound; the
// compiler's 243-254 registers give 2; measured at 128x128x64: 3 CTAs at 168 registers with
// spills no faster, 4 at 128 registers 12% slower)
#ifndef AWFL_ADJ_MINB
#define AWFL_ADJ_MINB 1
#endif

template <int ORD, int DIR> __global__ void __launch_bounds__(kAdjThreads) adj_edges_kernel(adj::SplitArgs A) {
  const long n = adj::ncell_of(A);
  for (long c = blockIdx.x * (long)blockDim.x + threadIdx.x; c < n; c += (long)gridDim.x * blockDim.x)
    adj::split_edges<ORD, DIR>(atab<ORD>(), A, c);
}

template <int DIR> __global__ void __launch_bounds__(kAdjThreads) adj_face_kernel(adj::SplitArgs A) {
  const long n = adj::nface_of<DIR>(A);
  for (long f = blockIdx.x * (long)blockDim.x + threadIdx.x; f < n; f += (long)gridDim.x * blockDim.x)
    adj::split_face<DIR>(A, f);
}

template <int ORD, int DIR>
__global__ void __launch_bounds__(kAdjThreads, ORD == 5 ? AWFL_ADJ_MINB : 1) adj_cell_kernel(adj::SplitArgs A) {
  const long n = adj::ncell_of(A);
  for (long c = blockIdx.x * (long)blockDim.x + threadIdx.x; c < n; c += (long)gridDim.x * blockDim.x)
    adj::split_cell_dt<ORD, DIR>(atab<ORD>(), A, c);
}

template <int ORD, int DIR>
__global__ void __launch_bounds__(kAdjThreads, ORD == 5 ? AWFL_ADJ_MINB : 1) adj_weno_kernel(adj::SplitArgs A) {
  const long n = 5 * adj::ncell_of(A);
  for (long x = blockIdx.x * (long)blockDim.x + threadIdx.x; x < n; x += (long)gridDim.x * blockDim.x)
    adj::split_weno<ORD, DIR>(atab<ORD>(), A, x);
}

template <int ORD, int DIR> __global__ void __launch_bounds__(kAdjThreads) adj_gather_kernel(adj::SplitArgs A) {
  const long n = adj::ncell_of(A);
  for (long c = blockIdx.x * (long)blockDim.x + threadIdx.x; c < n; c += (long)gridDim.x * blockDim.x)
    adj::split_gather<ORD, DIR>(A, c);
}

// Halo entries of an adjoint state are zero: halos are rebuilt from the interior before
// every use, so the result does not depend on them.
__global__ void zero_halo_kernel(double *lam, int nx, int ny, int nz, int hs) {
  const long sx = nx + 2 * hs, sy = ny + 2 * hs, sz = nz + 2 * hs;
  const long n = 5 * sz * sy * sx;
  for (long g = blockIdx.x * (long)blockDim.x + threadIdx.x; g < n; g += (long)gridDim.x * blockDim.x) {
    const int i = (int)(g % sx), j = (int)((g / sx) % sy), k = (int)((g / (sx * sy)) % sz);
    if (i < hs || i >= nx + hs || j < hs || j >= ny + hs || k < hs || k >= nz + hs) lam[g] = 0.;
  }
}

static unsigned grid_for(long n, int nsm) {
  long b = (n + kAdjThreads - 1) / kAdjThreads;
  const long cap = (long)nsm * 16;
  if (b > cap) b = cap;
  return (unsigned)(b < 1 ? 1 : b);
}

template <int ORD, int DIR>
static cudaError_t split_t(const adj::SplitArgs &A, int need_edges, int nsm, cudaStream_t st) {
  const long n = adj::ncell_of(A), nf = adj::nface_of<DIR>(A);
  if (need_edges) adj_edges_kernel<ORD, DIR><<<grid_for(n, nsm), kAdjThreads, 0, st>>>(A);
  adj_face_kernel<DIR><<<grid_for(nf, nsm), kAdjThreads, 0, st>>>(A);
  adj_cell_kernel<ORD, DIR><<<grid_for(n, nsm), kAdjThreads, 0, st>>>(A);
  adj_weno_kernel<ORD, DIR><<<grid_for(5 * n, nsm), kAdjThreads, 0, st>>>(A);
  adj_gather_kernel<ORD, DIR><<<grid_for(n, nsm), kAdjThreads, 0, st>>>(A);
  return cudaGetLastError();
}

cudaError_t launch_adjoint_split(int ord, int dir, const adj::SplitArgs &A, int need_edges, int nsm, cudaStream_t st) {
  if (ord == 5) {
    if (dir == 0) return split_t<5, 0>(A, need_edges, nsm, st);
    if (dir == 1) return split_t<5, 1>(A, need_edges, nsm, st);
    return split_t<5, 2>(A, need_edges, nsm, st);
  }
  if (dir == 0) return split_t<9, 0>(A, need_edges, nsm, st);
  if (dir == 1) return split_t<9, 1>(A, need_edges, nsm, st);
  return split_t<9, 2>(A, need_edges, nsm, st);
}

cudaError_t launch_zero_halo(double *lam, int nx, int ny, int nz, int hs, int nsm, cudaStream_t st) {
  const long n = 5L * (nx + 2 * hs) * (ny + 2 * hs) * (nz + 2 * hs);
  zero_halo_kernel<<<grid_for(n, nsm), kAdjThreads, 0, st>>>(lam, nx, ny, nz, hs);
  return cudaGetLastError();
}

cudaError_t upload_tables_adjrev(int ord, const void *tab, size_t bytes) {
  if (ord == 5) return cudaMemcpyToSymbol(a_tab5, tab, bytes);
  return cudaMemcpyToSymbol(a_tab9, tab, bytes);
}

}  // namespace awfl
