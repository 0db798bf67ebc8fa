// Project-written stand-in for the YAKL portability library, used ONLY to build the
// reference's own headers (driver.cpp, Spatial_euler3d_cons_expl_cart_fv_Agrid.h,
// Temporal_ader.h, WenoLimiter.h, TransformMatrices.h) on the CPU as a test oracle.
//
// This is test infrastructure: nothing in the shipped library includes it.
//
// YAKL itself is an absent git submodule of the reference (.gitmodules:1-3; its pinned
// commit is not recoverable). The reference uses it for containers and loop launch only
// (const.h:4-19). This file supplies exactly the semantics those headers rely on:
//   * Array<T,N,mem,styleC>: C-order (last index fastest), shallow/ref-counted copies,
//     const operator() returning T& (lambdas capture arrays by value and write through them).
//   * SArray<T,N,D...>: fixed-size C-order value array; assigning a scalar FILLS every
//     entry (the z-split gravity source relies on it, Spatial...h:1439).
//   * c::parallel_for over SimpleBounds<N>: OpenMP collapse over the N indices.
//   * ParallelMin: exact minimum (order independent).
//   * intrinsics::matmul_cr: (col,row)-indexed product,
//     C(c,r) = sum_k A(k,r) * B(c,k), k ascending from 0.
//   * memset, fence, init, finalize.
#pragma once

#include <cmath>
#include <math.h>
#include <cstdlib>
#include <cstring>
#include <cstddef>
#include <string>
#include <memory>
#include <vector>
#include <iostream>
#include <algorithm>
#include <stdexcept>

#define YAKL_INLINE inline
#define YAKL_LAMBDA [=]

namespace yakl {

  int constexpr memDevice = 1;
  int constexpr memHost   = 2;
  int constexpr styleC    = 1;

  inline void init() {}
  inline void finalize() {}
  inline void fence() {}

  template <class T> inline T min(T a, T b) { return a < b ? a : b; }
  template <class T> inline T max(T a, T b) { return a > b ? a : b; }

  // Dynamically sized, reference-counted, C-ordered array.
  template <class T, int N, int MEM, int STYLE> class Array {
  public:
    std::shared_ptr<T> store;  // array storage (shared_ptr<T> with array deleter)
    T *ptr = nullptr;
    size_t dims[N > 0 ? N : 1] = {0};
    std::string label;

    Array() {}

    template <class... I> Array(char const *lab, I... d) {
      static_assert(sizeof...(I) == N, "Array: wrong number of dimensions");
      label = lab;
      size_t dd[] = {static_cast<size_t>(d)...};
      size_t tot = 1;
      for (int i = 0; i < N; i++) { dims[i] = dd[i]; tot *= dd[i]; }
      store = std::shared_ptr<T>(new T[tot](), std::default_delete<T[]>());
      ptr = store.get();
    }

    size_t totElems() const {
      size_t tot = 1;
      for (int i = 0; i < N; i++) tot *= dims[i];
      return tot;
    }
    size_t get_elem_count() const { return totElems(); }

    T *data() const { return ptr; }
    bool initialized() const { return ptr != nullptr; }
    int extent(int i) const { return (int)dims[i]; }

    template <class... I> inline T &operator()(I... ind) const {
      static_assert(sizeof...(I) == N, "Array: wrong number of indices");
      size_t ii[] = {static_cast<size_t>(ind)...};
      size_t off = 0;
      for (int i = 0; i < N; i++) {
#ifdef AWFL_SHIM_BOUNDS_CHECK
        if (ii[i] >= dims[i]) throw std::out_of_range(label + ": index out of range");
#endif
        off = off * dims[i] + ii[i];
      }
      return ptr[off];
    }

    Array<T, N, memHost, STYLE> createHostCopy() const {
      Array<T, N, memHost, STYLE> ret;
      ret.label = label;
      for (int i = 0; i < N; i++) ret.dims[i] = dims[i];
      size_t tot = totElems();
      ret.store = std::shared_ptr<T>(new T[tot], std::default_delete<T[]>());
      ret.ptr = ret.store.get();
      for (size_t i = 0; i < tot; i++) ret.ptr[i] = ptr[i];
      return ret;
    }

    template <int MEM2> void deep_copy_to(Array<T, N, MEM2, STYLE> const &dst) const {
      std::memcpy(dst.ptr, ptr, sizeof(T) * totElems());
    }
  };

  // Statically sized C-ordered array. Default construction leaves storage uninitialised,
  // as the reference's code never reads an entry before writing it.
  template <class T, int N, unsigned... D> class SArray {
  public:
    static constexpr unsigned dimsArr[sizeof...(D)] = {D...};
    static constexpr size_t total() {
      size_t t = 1;
      for (unsigned d : {D...}) t *= d;
      return t;
    }
    T myData[total()];

    SArray() {}
    SArray(T val) { for (size_t i = 0; i < total(); i++) myData[i] = val; }
    SArray &operator=(T val) {
      for (size_t i = 0; i < total(); i++) myData[i] = val;
      return *this;
    }

    template <class... I> inline T &operator()(I... ind) {
      static_assert(sizeof...(I) == N, "SArray: wrong number of indices");
      size_t ii[] = {static_cast<size_t>(ind)...};
      size_t off = 0;
      for (int i = 0; i < N; i++) off = off * dimsArr[i] + ii[i];
      return myData[off];
    }
    template <class... I> inline T const &operator()(I... ind) const {
      static_assert(sizeof...(I) == N, "SArray: wrong number of indices");
      size_t ii[] = {static_cast<size_t>(ind)...};
      size_t off = 0;
      for (int i = 0; i < N; i++) off = off * dimsArr[i] + ii[i];
      return myData[off];
    }
    T *data() { return myData; }
    T const *data() const { return myData; }
  };

  template <class T, int N, int MEM, int STYLE>
  inline void memset(Array<T, N, MEM, STYLE> const &arr, T val) {
    size_t tot = arr.totElems();
    for (size_t i = 0; i < tot; i++) arr.ptr[i] = val;
  }

  template <class T, int MEM> class ParallelMin {
    size_t n;
  public:
    ParallelMin(size_t n_) : n(n_) {}
    T operator()(T const *p) const {
      T m = p[0];
      for (size_t i = 1; i < n; i++) if (p[i] < m) m = p[i];
      return m;
    }
  };

  namespace intrinsics {
    // C(c,r) = sum_k A(k,r) * B(c,k); A is (colsA x rowsA) = (K x R), B is (C x K).
    template <class T, unsigned K, unsigned R, unsigned C>
    inline SArray<T, 2, C, R> matmul_cr(SArray<T, 2, K, R> const &A, SArray<T, 2, C, K> const &B) {
      SArray<T, 2, C, R> ret;
      for (unsigned c = 0; c < C; c++) {
        for (unsigned r = 0; r < R; r++) {
          T tmp = 0;
          for (unsigned k = 0; k < K; k++) tmp += A(k, r) * B(c, k);
          ret(c, r) = tmp;
        }
      }
      return ret;
    }
  }

  namespace c {
    template <int N> struct SimpleBounds {
      int d[N];
      template <class... I> SimpleBounds(I... dd) : d{static_cast<int>(dd)...} {
        static_assert(sizeof...(I) == N, "SimpleBounds: wrong number of dimensions");
      }
    };
    template <int N> using Bounds = SimpleBounds<N>;

    template <class F> inline void parallel_for(SimpleBounds<1> const &b, F const &f) {
      #pragma omp parallel for
      for (int i = 0; i < b.d[0]; i++) f(i);
    }
    template <class F> inline void parallel_for(int n, F const &f) {
      #pragma omp parallel for
      for (int i = 0; i < n; i++) f(i);
    }
    template <class F> inline void parallel_for(SimpleBounds<2> const &b, F const &f) {
      #pragma omp parallel for collapse(2)
      for (int i = 0; i < b.d[0]; i++)
        for (int j = 0; j < b.d[1]; j++) f(i, j);
    }
    template <class F> inline void parallel_for(SimpleBounds<3> const &b, F const &f) {
      #pragma omp parallel for collapse(3)
      for (int i = 0; i < b.d[0]; i++)
        for (int j = 0; j < b.d[1]; j++)
          for (int k = 0; k < b.d[2]; k++) f(i, j, k);
    }
    template <class F> inline void parallel_for(SimpleBounds<4> const &b, F const &f) {
      #pragma omp parallel for collapse(4)
      for (int i = 0; i < b.d[0]; i++)
        for (int j = 0; j < b.d[1]; j++)
          for (int k = 0; k < b.d[2]; k++)
            for (int l = 0; l < b.d[3]; l++) f(i, j, k, l);
    }
  }
}
