// FP64 sweep policy P64 (the reference's arithmetic) over the line-sweep skeleton.
// Included by the translation units that instantiate FP64 sweeps (awfl_fp64.cu,
// awfl_ens64.cu); each has its own copy of the constant tables (awfl_device.cuh).
#pragma once

#include "awfl_device.cuh"
#include "awfl_internal.h"
#include "awfl_sweep.cuh"

namespace awfl {

// ------------------------------------------------------------------------------------
// FP64 physics policy of the line sweep (awfl_sweep.cuh): the reference's arithmetic.
// ------------------------------------------------------------------------------------
#ifdef AWFL_FP64_OUTLINE_RIEMANN
struct Q5 {
  double v[5];
};
template <int DIR, int NG> static __device__ __noinline__ Q5 riemann_call(Q5 qL, Q5 qR, int kf, const SweepArgs *A) {
  Q5 F;
  riemann<DIR, NG>(qL.v, qR.v, kf, *A, F.v);
  return F;
}
#endif

struct P64 {
  using Real = double;
  static constexpr int kWdiv = 1;
  static constexpr bool kAsyncRing = true;
  static constexpr bool kTmaRing = false;
  static constexpr bool kSlab = true;  // awfl_split_slab
  // ord 5: 4 CTAs per SM (<= 128 registers), more warps to hide the FP64 latency
  // (measured +17%); ord 9 would spill heavily at that budget
#ifndef AWFL_P64_MIN_BLOCKS_ORD5
#define AWFL_P64_MIN_BLOCKS_ORD5 4
#endif
  static constexpr int min_blocks(int ord) { return ord == 5 ? AWFL_P64_MIN_BLOCKS_ORD5 : 1; }
  using Args = SweepArgs;
  struct Aux {};
  static __device__ __forceinline__ void load_aux(const Args &, long, long, Aux &) {}

  template <int ORD, int DIR, class S>
  static __device__ __forceinline__ void recon(const S &sten, int kb, const Args &A, double (&eL)[5],
                                               double (&eR)[5], double &src, long) {
    cell_recon<ORD, DIR>(sten, kb, A, eL, eR, src);
  }

  template <int DIR, int NG>
  static __device__ __forceinline__ void flux(const double (&qL)[5], const double (&qR)[5], int kf, const Args &A,
                                              double (&F)[5]) {
#ifdef AWFL_FP64_OUTLINE_RIEMANN
    Q5 a, b;
#pragma unroll
    for (int v = 0; v < 5; v++) {
      a.v[v] = qL[v];
      b.v[v] = qR[v];
    }
    const Q5 f = riemann_call<DIR, NG>(a, b, kf, &A);
#pragma unroll
    for (int v = 0; v < 5; v++) F[v] = f.v[v];
#else
    riemann<DIR, NG>(qL, qR, kf, A, F);
#endif
  }

  // K5 divergence (Spatial:940-956, 1298-1310, 1680-1696): z adds onto the gravity source.
  template <int DIR>
  static __device__ __forceinline__ double tendency(int v, double Fl, double Fr, double sa, const Args &A) {
    const double d = divd(-(Fr - Fl), rcp_known(A.dxd, A.rdxd));
    if (DIR == 0) return (A.sim2d && v == idV) ? 0.0 : d;
    if (DIR == 1) return d;
    return (A.sim2d && v == idV) ? 0.0 : (v == idW ? sa : 0.0) + d;
  }

  // K6 apply (Temporal_ader.h:63-65)
  static __device__ __forceinline__ void apply(const Args &A, long g, double orig, double tnd, const Aux &, int) {
    A.state[g] = orig + A.dt * tnd;
  }
  static __device__ __forceinline__ double load(const Args &A, long g) { return A.state[g]; }
  static __device__ __forceinline__ void store(const Args &A, long g, double x) { A.state[g] = x; }
  static __device__ __forceinline__ void store_tend(const Args &A, long g, double x) { A.tend[g] = x; }
};

// Single-grid sweep shapes of the FP64 path, ord 5 (chunk x lines; measured at
// 256x256x128 with the current kernel against x 32 x 4 / 8 x 16 and y, z 4 x 32 / 16 x 8,
// which took 1-2% longer): x 16 x 8, y and z 8 x 16. The macros let a build try others.
#ifndef AWFL_P64_XC
#define AWFL_P64_XC 16
#define AWFL_P64_XW 8
#endif
#ifndef AWFL_P64_YC
#define AWFL_P64_YC 8
#define AWFL_P64_YW 16
#endif
#ifndef AWFL_P64_ZC
#define AWFL_P64_ZC 8
#define AWFL_P64_ZW 16
#endif
template <> struct PolicyShape<P64, 5, 0> { static constexpr int C = AWFL_P64_XC, W = AWFL_P64_XW; };
template <> struct PolicyShape<P64, 5, 1> { static constexpr int C = AWFL_P64_YC, W = AWFL_P64_YW; };
template <> struct PolicyShape<P64, 5, 2> { static constexpr int C = AWFL_P64_ZC, W = AWFL_P64_ZW; };

}  // namespace awfl
