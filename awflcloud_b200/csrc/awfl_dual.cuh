// Forward-mode dual number (value, tangent) for the tangent-linear sweep.
//
// The FP64 device code (awfl_device.cuh) is templated on its scalar type; instantiated
// with Dual it evaluates the reference arithmetic on the value part -- the same operations
// in the same order as the FP64 path, so the base trajectory is bit-identical -- and the
// exact derivative along one direction on the tangent part.
#pragma once

#include "awfl_pow.cuh"

namespace awfl {

struct Dual {
  double v, d;
  __host__ __device__ Dual() : v(0), d(0) {}
  __host__ __device__ Dual(double x) : v(x), d(0) {}
  __host__ __device__ Dual(double x, double t) : v(x), d(t) {}
  __device__ Dual &operator+=(const Dual &o) { v += o.v; d += o.d; return *this; }
  __device__ Dual &operator-=(const Dual &o) { v -= o.v; d -= o.d; return *this; }
  __device__ Dual &operator*=(const Dual &o) { d = d * o.v + v * o.d; v *= o.v; return *this; }
  __device__ Dual &operator/=(const Dual &o) { const double q = v / o.v; d = (d - q * o.d) / o.v; v = q; return *this; }
};

__device__ __forceinline__ Dual operator-(const Dual &a) { return Dual(-a.v, -a.d); }
__device__ __forceinline__ Dual operator+(const Dual &a, const Dual &b) { return Dual(a.v + b.v, a.d + b.d); }
__device__ __forceinline__ Dual operator-(const Dual &a, const Dual &b) { return Dual(a.v - b.v, a.d - b.d); }
__device__ __forceinline__ Dual operator*(const Dual &a, const Dual &b) { return Dual(a.v * b.v, a.d * b.v + a.v * b.d); }
__device__ __forceinline__ Dual operator/(const Dual &a, const Dual &b) {
  const double q = a.v / b.v;
  return Dual(q, (a.d - q * b.d) / b.v);
}
__device__ __forceinline__ Dual operator+(const Dual &a, double b) { return Dual(a.v + b, a.d); }
__device__ __forceinline__ Dual operator+(double a, const Dual &b) { return Dual(a + b.v, b.d); }
__device__ __forceinline__ Dual operator-(const Dual &a, double b) { return Dual(a.v - b, a.d); }
__device__ __forceinline__ Dual operator-(double a, const Dual &b) { return Dual(a - b.v, -b.d); }
__device__ __forceinline__ Dual operator*(const Dual &a, double b) { return Dual(a.v * b, a.d * b); }
__device__ __forceinline__ Dual operator*(double a, const Dual &b) { return Dual(a * b.v, a * b.d); }
__device__ __forceinline__ Dual operator/(const Dual &a, double b) { return Dual(a.v / b, a.d / b); }
__device__ __forceinline__ Dual operator/(double a, const Dual &b) {
  const double q = a / b.v;
  return Dual(q, -q * b.d / b.v);
}
__device__ __forceinline__ bool operator>(const Dual &a, double b) { return a.v > b; }
__device__ __forceinline__ bool operator<(const Dual &a, double b) { return a.v < b; }

// d(x^y) = y x^(y-1) dx = y (x^y / x) dx, with the value part as the FP64 path computes it.
__device__ __forceinline__ Dual pow_cr(const Dual &x, double y) {
  const double p = pow_cr(x.v, y);
  return Dual(p, y * (p / x.v) * x.d);
}
// (the double overload keeps unqualified sqrt(double) calls inside namespace awfl working)
__device__ __forceinline__ double sqrt(double x) { return ::sqrt(x); }
__device__ __forceinline__ Dual sqrt(const Dual &x) {
  const double s = ::sqrt(x.v);
  return Dual(s, 0.5 * x.d / s);
}

}  // namespace awfl
