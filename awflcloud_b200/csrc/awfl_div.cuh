// IEEE division by a divisor shared by several quotients, for the FP64 parity path.
//
// The reference divides with the CPU's correctly rounded division everywhere. Several of
// its quotients share a divisor: the four velocity-like ratios and the eight Cauchy-
// product quotients of a GLL point all divide by its density, the WENO normalisations
// divide all weights by one sum, and every tendency divides by dx. Each IEEE division on
// the GPU is a reciprocal-approximation sequence of ~10 FP64 instructions; here the
// correctly rounded reciprocal y = RN(1/b) is formed once, and each quotient a/b costs one
// multiply and four FMAs:
//
//   q0 = RN(a*y);  q1 = RN(q0 + RN(a - b*q0)*y);  q2 = RN(q1 + (a - b*q1)*y)
//
// q1 is within one ulp of a/b (q0 is within 1.5 ulp, and the first correction leaves
// half an ulp plus ~2^-52 ulp), so b*q1 differs from a by an exactly representable
// remainder, and by Markstein's theorem (P. Markstein, "Computation of elementary
// functions on the IBM RISC System/6000 processor", IBM J. Res. Dev. 34(1), 1990: with y
// within half an ulp of 1/b and q within one ulp of a/b, RN(q + (a - bq)y) = RN(a/b)) q2
// is the correctly rounded quotient -- the IEEE result bit for bit, for operands whose
// quotient, remainder and reciprocal stay in the normal range (the path's values are
// physical quantities of order 1e-20 .. 1e20). A zero dividend returns RN(a*y), which
// carries IEEE's sign of zero. Tested against the GPU's IEEE division on random and
// edge-case operands (tests/test_pow_gpu.py) and through the bit-exact parity tests.
//
// The scalar type may also be the tangent-linear Dual; its quotients keep the plain
// division (their value parts are bit-identical either way).
#pragma once

namespace awfl {

template <class Sc> struct Rcp {
  Sc b;
};
template <> struct Rcp<double> {
  double b, y;  // divisor and RN(1/b)
};

template <class Sc> __device__ __forceinline__ Rcp<Sc> make_rcp(const Sc &b) { return Rcp<Sc>{b}; }
template <> __device__ __forceinline__ Rcp<double> make_rcp(const double &b) { return Rcp<double>{b, 1.0 / b}; }
// a divisor whose reciprocal RN(1/b) is already known (host-computed, or a folded constant)
__host__ __device__ __forceinline__ Rcp<double> rcp_known(double b, double y) { return Rcp<double>{b, y}; }

__device__ __forceinline__ double div_markstein(double a, double b, double y) {
  const double q0 = __dmul_rn(a, y);
  const double q1 = __fma_rn(__fma_rn(-q0, b, a), y, q0);
  const double q2 = __fma_rn(__fma_rn(-q1, b, a), y, q1);
  return a == 0.0 ? q0 : q2;
}

// a / r.b, correctly rounded
template <class Sc> __device__ __forceinline__ Sc divr(const Sc &a, const Rcp<Sc> &r) { return a / r.b; }
__device__ __forceinline__ double divr(const double &a, const Rcp<double> &r) { return div_markstein(a, r.b, r.y); }
// a / r.b, correctly rounded for every dividend: nonzero ones below 2^-900 in magnitude
// (where the quotient or the remainder could leave the normal range, as transported
// tracer values that decay towards zero can) take the IEEE division itself; a zero
// dividend stays on the short path, whose RN(a*y) is IEEE's signed zero
__device__ __forceinline__ double divr_any(double a, const Rcp<double> &r) {
  return (fabs(a) < 0x1p-900 && a != 0.0) ? a / r.b : div_markstein(a, r.b, r.y);
}
// any scalar divided by a double divisor with a known reciprocal
template <class Sc> __device__ __forceinline__ Sc divd(const Sc &a, const Rcp<double> &r) { return a / r.b; }
__device__ __forceinline__ double divd(const double &a, const Rcp<double> &r) { return div_markstein(a, r.b, r.y); }

// a / k for a small positive integer k that is a constant once loops are unrolled: 1 and
// powers of two are exact multiplications; others use the constant-folded reciprocal.
template <class Sc> __device__ __forceinline__ Sc divk(const Sc &a, int k) {
  if (k == 1) return a;
  if ((k & (k - 1)) == 0) return a * (1.0 / k);
  return divd(a, rcp_known((double)k, 1.0 / k));
}

// divk for dividends of any magnitude (divr_any's range)
__device__ __forceinline__ double divk_any(double a, int k) {
  if (k == 1) return a;
  if ((k & (k - 1)) == 0) return a * (1.0 / k);
  return divr_any(a, rcp_known((double)k, 1.0 / k));
}

// the reciprocal of 2b from that of b (exact: a power-of-two scaling)
template <class Sc> __device__ __forceinline__ Rcp<Sc> rcp_twice(const Rcp<Sc> &r) { return Rcp<Sc>{2. * r.b}; }
__device__ __forceinline__ Rcp<double> rcp_twice(const Rcp<double> &r) { return Rcp<double>{2. * r.b, 0.5 * r.y}; }

}  // namespace awfl
