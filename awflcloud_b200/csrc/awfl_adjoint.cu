// Differentiation form of the FP64 step: the tangent-linear sweep (forward mode, Dual
// scalars through the same templated FP64 code) and the recording forward sweep of the
// discrete adjoint (its reverse sweeps are in awfl_adjrev.cu). Compiled with --fmad=false
// like the FP64 path.
#include <cuda_runtime.h>

#include "awfl_dual.cuh"
#include "awfl_internal.h"
#include "awfl_p64.cuh"

namespace awfl {

// ------------------------------------------------------------------------------------
// Tangent-linear policy: the FP64 arithmetic on Dual numbers. The state buffer holds the
// value plane and, A.plane elements further, the tangent plane; both advance together.
// The time step dt is a fixed parameter (not differentiated).
// ------------------------------------------------------------------------------------
struct PTLM {
  using Real = Dual;
  static constexpr int kWdiv = 2;
  static constexpr bool kAsyncRing = false;
  static constexpr bool kTmaRing = false;
  static constexpr bool kSlab = false;
  static constexpr int min_blocks(int) { return 1; }
  using Args = SweepArgs;
  struct Aux {};
  static __device__ __forceinline__ void load_aux(const Args &, long, long, Aux &) {}

  template <int ORD, int DIR, class S>
  static __device__ __forceinline__ void recon(const S &sten, int kb, const Args &A, Dual (&eL)[5], Dual (&eR)[5],
                                               Dual &src, long) {
    cell_recon<ORD, DIR>(sten, kb, A, eL, eR, src);
  }
  template <int DIR, int NG>
  static __device__ __forceinline__ void flux(const Dual (&qL)[5], const Dual (&qR)[5], int kf, const Args &A,
                                              Dual (&F)[5]) {
    riemann<DIR, NG>(qL, qR, kf, A, F);
  }
  template <int DIR>
  static __device__ __forceinline__ Dual tendency(int v, Dual Fl, Dual Fr, Dual sa, const Args &A) {
    const Dual d = -(Fr - Fl) / A.dxd;
    if (DIR == 0) return (A.sim2d && v == idV) ? Dual(0.0) : d;
    if (DIR == 1) return d;
    return (A.sim2d && v == idV) ? Dual(0.0) : (v == idW ? sa : Dual(0.0)) + d;
  }
  static __device__ __forceinline__ void apply(const Args &A, long g, Dual orig, Dual tnd, const Aux &, int) {
    A.state[g] = orig.v + A.dt * tnd.v;
    A.state[g + A.plane] = orig.d + A.dt * tnd.d;
  }
  static __device__ __forceinline__ Dual load(const Args &A, long g) { return Dual(A.state[g], A.state[g + A.plane]); }
  static __device__ __forceinline__ void store(const Args &A, long g, Dual x) {
    A.state[g] = x.v;
    A.state[g + A.plane] = x.d;
  }
  static __device__ __forceinline__ void store_tend(const Args &A, long g, Dual x) { A.tend[g] = x.d; }
};

cudaError_t launch_sweep_tlm(int ord, int dir, const SweepArgs &A, cudaStream_t st) {
  return launch_sweep_any<PTLM>(ord, dir, A, st);
}

// ------------------------------------------------------------------------------------
// Recording FP64 policy for the adjoint's forward recomputation: the P64 arithmetic (so
// the recomputed trajectory is bit-identical to awfl_step's) that also keeps, per cell,
// the level-0 GLL values and the time-averaged edge states the reverse sweep starts from.
// A.tend points at the split's record: q0 (5*NGLL planes of ncell), then eL, eR (10).
// ------------------------------------------------------------------------------------
struct P64Rec : P64 {
  static constexpr bool kSlab = false;
  template <int ORD> struct Rec {
    double *q0;
    long n, cell;
    __device__ __forceinline__ void level0(int v, int ii, const double &x) const {
      q0[(v * OrdTraits<ORD>::NGLL + ii) * n + cell] = x;
    }
    template <class Q> __device__ __forceinline__ void series(const Q &) const {}
  };
  template <int ORD, int DIR, class S>
  static __device__ __forceinline__ void recon(const S &sten, int kb, const Args &A, double (&eL)[5],
                                               double (&eR)[5], double &src, long cell) {
    if (cell < 0) {  // the periodic prologue's repeat of cell L-1: recorded in its chunk
      cell_recon<ORD, DIR>(sten, kb, A, eL, eR, src);
      return;
    }
    constexpr int NG = OrdTraits<ORD>::NGLL;
    const long n = (long)A.nx * A.ny * A.nz;
    cell_recon<ORD, DIR>(sten, kb, A, eL, eR, src, Rec<ORD>{A.tend, n, cell});
    double *e = A.tend + 5L * NG * n;
#pragma unroll
    for (int v = 0; v < 5; v++) {
      e[v * n + cell] = eL[v];
      e[(5 + v) * n + cell] = eR[v];
    }
  }
};
template <int ORD, int DIR> struct PolicyShape<P64Rec, ORD, DIR> : PolicyShape<P64, ORD, DIR> {};

cudaError_t launch_sweep_rec(int ord, int dir, const SweepArgs &A, cudaStream_t st) {
  return launch_sweep_any<P64Rec>(ord, dir, A, st);
}

cudaError_t upload_tables_adj(int ord, const void *tab, size_t bytes) {
  if (ord == 5) return cudaMemcpyToSymbol(c_tab5, tab, bytes);
  return cudaMemcpyToSymbol(c_tab9, tab, bytes);
}

}  // namespace awfl
