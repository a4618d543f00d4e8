// dual.cuh -- forward-mode dual numbers (value + one directional derivative) for the adjoint of the
// node-local pieces of the right-hand side (mixture transport properties, finite-rate chemistry).
// Templated device code instantiated with Dual computes, next to each value, its derivative along
// one seeded input; a vector-Jacobian product over k node inputs is then k such evaluations.
#pragma once

#include <cuda_runtime.h>

namespace ostc {
// The type and its functions sit in their own namespace: unqualified exp / log / sqrt / pow on
// doubles elsewhere in ostc keep resolving to the CUDA math functions, and calls on Dual find these
// by argument-dependent lookup.
namespace ad {

struct Dual {
  double v, d;
  __host__ __device__ Dual() : v(0), d(0) {}
  __host__ __device__ Dual(double x) : v(x), d(0) {}  // constants carry no derivative
  __host__ __device__ Dual(double x, double dx) : v(x), d(dx) {}
  __host__ __device__ explicit operator double() const { return v; }
  __host__ __device__ Dual &operator+=(const Dual &o) { v += o.v; d += o.d; return *this; }
  __host__ __device__ Dual &operator-=(const Dual &o) { v -= o.v; d -= o.d; return *this; }
  __host__ __device__ Dual &operator*=(const Dual &o) { d = d * o.v + v * o.d; v *= o.v; return *this; }
  __host__ __device__ Dual &operator/=(const Dual &o) {
    const double q = v / o.v;
    d = (d - q * o.d) / o.v;
    v = q;
    return *this;
  }
};

__host__ __device__ inline Dual operator-(const Dual &a) { return Dual(-a.v, -a.d); }
__host__ __device__ inline Dual operator+(Dual a, const Dual &b) { return a += b; }
__host__ __device__ inline Dual operator-(Dual a, const Dual &b) { return a -= b; }
__host__ __device__ inline Dual operator*(Dual a, const Dual &b) { return a *= b; }
__host__ __device__ inline Dual operator/(Dual a, const Dual &b) { return a /= b; }
__host__ __device__ inline Dual operator+(Dual a, double b) { a.v += b; return a; }
__host__ __device__ inline Dual operator+(double b, Dual a) { a.v += b; return a; }
__host__ __device__ inline Dual operator-(Dual a, double b) { a.v -= b; return a; }
__host__ __device__ inline Dual operator-(double b, const Dual &a) { return Dual(b - a.v, -a.d); }
__host__ __device__ inline Dual operator*(Dual a, double b) { return Dual(a.v * b, a.d * b); }
__host__ __device__ inline Dual operator*(double b, Dual a) { return Dual(a.v * b, a.d * b); }
__host__ __device__ inline Dual operator/(Dual a, double b) { return Dual(a.v / b, a.d / b); }
__host__ __device__ inline Dual operator/(double b, const Dual &a) {
  const double q = b / a.v;
  return Dual(q, -q * a.d / a.v);
}
__host__ __device__ inline bool operator<(const Dual &a, const Dual &b) { return a.v < b.v; }
__host__ __device__ inline bool operator>(const Dual &a, const Dual &b) { return a.v > b.v; }
__host__ __device__ inline bool operator<=(const Dual &a, const Dual &b) { return a.v <= b.v; }
__host__ __device__ inline bool operator>=(const Dual &a, const Dual &b) { return a.v >= b.v; }

__device__ inline Dual exp(const Dual &a) {
  const double e = ::exp(a.v);
  return Dual(e, e * a.d);
}
__device__ inline Dual log(const Dual &a) { return Dual(::log(a.v), a.d / a.v); }
__device__ inline Dual fabs(const Dual &a) { return a.v < 0 ? -a : a; }
__device__ inline Dual log10(const Dual &a) { return Dual(::log10(a.v), a.d / (a.v * 2.302585092994045684)); }
__device__ inline Dual sqrt(const Dual &a) {
  const double s = ::sqrt(a.v);
  return Dual(s, 0.5 * a.d / s);
}
// x^y with a constant exponent
__device__ inline Dual pow(const Dual &x, double y) {
  const double p = ::pow(x.v, y);
  return Dual(p, y == 0.0 ? 0.0 : y * ::pow(x.v, y - 1.0) * x.d);
}
// b^y with a constant base
__device__ inline Dual pow(double b, const Dual &y) {
  const double p = ::pow(b, y.v);
  return Dual(p, p * ::log(b) * y.d);
}
// x^y, both carrying derivatives (the exponent's term only where it has one)
__device__ inline Dual pow(const Dual &x, const Dual &y) {
  Dual r = pow(x, y.v);
  if (y.d != 0.0) r.d += r.v * ::log(x.v) * y.d;
  return r;
}

__device__ inline Dual arrhenius(const Dual &lt, const Dual &ti, double A, double b, double Ea) {
  return A * exp(b * lt - Ea * ti);
}

}  // namespace ad

using ad::Dual;
template <> __device__ __forceinline__ Dual tsqrt<Dual>(Dual x) { return ad::sqrt(x); }
template <> __device__ __forceinline__ Dual tpow<Dual>(Dual x, Dual y) { return ad::pow(x, y); }

}  // namespace ostc
