// GENERATED by awflcloud_b200/gen_tables.py -- do not edit by hand.
// coefs_to_tv(n) evaluators: r = c0*(a_q*a_q); r = r + (c*a_m)*a_q ... in the
// reference's term order (TransformMatrices.h coefs_to_tv).
#pragma once

#if defined(__CUDACC__)
#define AWFL_TV_HD __host__ __device__ __forceinline__
#else
#define AWFL_TV_HD inline
#endif

template <class T> AWFL_TV_HD T awfl_tv_n3(const T *a) {
  T r = T(0x1.0000000000000p+0) * (a[1] * a[1]);
  r = r + T(0x1.1555555555555p+2) * (a[2] * a[2]);
  return r;
}

template <class T> AWFL_TV_HD T awfl_tv_n5(const T *a) {
  T r = T(0x1.0000000000000p+0) * (a[1] * a[1]);
  r = r + T(0x1.1555555555555p+2) * (a[2] * a[2]);
  r = r + T(0x1.0000000000000p-1) * a[1] * a[3];
  r = r + T(0x1.38e6666666666p+5) * (a[3] * a[3]);
  r = r + T(0x1.0cccccccccccdp+2) * a[2] * a[4];
  r = r + T(0x1.38e6666666666p+9) * (a[4] * a[4]);
  return r;
}

template <class T> AWFL_TV_HD T awfl_tv_n9(const T *a) {
  T r = T(0x1.0000000000000p+0) * (a[1] * a[1]);
  r = r + T(0x1.1555555555555p+2) * (a[2] * a[2]);
  r = r + T(0x1.0000000000000p-1) * a[1] * a[3];
  r = r + T(0x1.38e6666666666p+5) * (a[3] * a[3]);
  r = r + T(0x1.0cccccccccccdp+2) * a[2] * a[4];
  r = r + T(0x1.38eaf8af8af8bp+9) * (a[4] * a[4]);
  r = r + T(0x1.0000000000000p-3) * a[1] * a[5];
  r = r + T(0x1.f889249249249p+5) * a[3] * a[5];
  r = r + T(0x1.e8ef3acb2cb2dp+13) * (a[5] * a[5]);
  r = r + T(0x1.8db6db6db6db7p+0) * a[2] * a[6];
  r = r + T(0x1.7a6830c30c30cp+10) * a[4] * a[6];
  r = r + T(0x1.1306911249249p+19) * (a[6] * a[6]);
  r = r + T(0x1.0000000000000p-5) * a[1] * a[7];
  r = r + T(0x1.0525555555555p+5) * a[3] * a[7];
  r = r + T(0x1.9de1f55555555p+15) * a[5] * a[7];
  r = r + T(0x1.a5220e2400000p+24) * (a[7] * a[7]);
  r = r + T(0x1.071c71c71c71cp-1) * a[2] * a[8];
  r = r + T(0x1.0525555555555p+10) * a[4] * a[8];
  r = r + T(0x1.3669780000000p+21) * a[6] * a[8];
  r = r + T(0x1.a5220e2400000p+30) * (a[8] * a[8]);
  return r;
}

// Gradients of the quadratic forms above: g[m] += lam * d tv / d a[m].
template <class T> AWFL_TV_HD void awfl_tv_grad_n3(const T *a, T lam, T *g) {
  g[1] += lam * (T(0x1.0000000000000p+1) * a[1]);
  g[2] += lam * (T(0x1.1555555555555p+3) * a[2]);
}

template <class T> AWFL_TV_HD void awfl_tv_grad_n5(const T *a, T lam, T *g) {
  g[1] += lam * (T(0x1.0000000000000p+1) * a[1]);
  g[2] += lam * (T(0x1.1555555555555p+3) * a[2]);
  g[1] += lam * (T(0x1.0000000000000p-1) * a[3]);
  g[3] += lam * (T(0x1.0000000000000p-1) * a[1]);
  g[3] += lam * (T(0x1.38e6666666666p+6) * a[3]);
  g[2] += lam * (T(0x1.0cccccccccccdp+2) * a[4]);
  g[4] += lam * (T(0x1.0cccccccccccdp+2) * a[2]);
  g[4] += lam * (T(0x1.38e6666666666p+10) * a[4]);
}

template <class T> AWFL_TV_HD void awfl_tv_grad_n9(const T *a, T lam, T *g) {
  g[1] += lam * (T(0x1.0000000000000p+1) * a[1]);
  g[2] += lam * (T(0x1.1555555555555p+3) * a[2]);
  g[1] += lam * (T(0x1.0000000000000p-1) * a[3]);
  g[3] += lam * (T(0x1.0000000000000p-1) * a[1]);
  g[3] += lam * (T(0x1.38e6666666666p+6) * a[3]);
  g[2] += lam * (T(0x1.0cccccccccccdp+2) * a[4]);
  g[4] += lam * (T(0x1.0cccccccccccdp+2) * a[2]);
  g[4] += lam * (T(0x1.38eaf8af8af8bp+10) * a[4]);
  g[1] += lam * (T(0x1.0000000000000p-3) * a[5]);
  g[5] += lam * (T(0x1.0000000000000p-3) * a[1]);
  g[3] += lam * (T(0x1.f889249249249p+5) * a[5]);
  g[5] += lam * (T(0x1.f889249249249p+5) * a[3]);
  g[5] += lam * (T(0x1.e8ef3acb2cb2dp+14) * a[5]);
  g[2] += lam * (T(0x1.8db6db6db6db7p+0) * a[6]);
  g[6] += lam * (T(0x1.8db6db6db6db7p+0) * a[2]);
  g[4] += lam * (T(0x1.7a6830c30c30cp+10) * a[6]);
  g[6] += lam * (T(0x1.7a6830c30c30cp+10) * a[4]);
  g[6] += lam * (T(0x1.1306911249249p+20) * a[6]);
  g[1] += lam * (T(0x1.0000000000000p-5) * a[7]);
  g[7] += lam * (T(0x1.0000000000000p-5) * a[1]);
  g[3] += lam * (T(0x1.0525555555555p+5) * a[7]);
  g[7] += lam * (T(0x1.0525555555555p+5) * a[3]);
  g[5] += lam * (T(0x1.9de1f55555555p+15) * a[7]);
  g[7] += lam * (T(0x1.9de1f55555555p+15) * a[5]);
  g[7] += lam * (T(0x1.a5220e2400000p+25) * a[7]);
  g[2] += lam * (T(0x1.071c71c71c71cp-1) * a[8]);
  g[8] += lam * (T(0x1.071c71c71c71cp-1) * a[2]);
  g[4] += lam * (T(0x1.0525555555555p+10) * a[8]);
  g[8] += lam * (T(0x1.0525555555555p+10) * a[4]);
  g[6] += lam * (T(0x1.3669780000000p+21) * a[8]);
  g[8] += lam * (T(0x1.3669780000000p+21) * a[6]);
  g[8] += lam * (T(0x1.a5220e2400000p+31) * a[8]);
}

