// mhd_dual.cuh -- forward-mode dual numbers for the derivative form.
//
// Dual<N> carries a value and its derivatives with respect to N parameters;
// every arithmetic operation applies the chain rule.  Comparisons look at
// the value only, so branches follow the primal computation.  At a point
// where a function is not differentiable (sqrt and fabs at 0) the derivative
// is taken as 0: the pairs where this happens in the SPMHD equations (equal
// pressures in the conduction signal speed, equal transverse velocities in
// the resistive signal speed) multiply the non-differentiable factor by a
// difference that vanishes with it, so 0 is the limit of the product's
// derivative.
#pragma once

#include <cuda_runtime.h>
#include <math.h>

namespace mhd {

template <int N>
struct Dual {
  double v;
  double d[N];
  __host__ __device__ constexpr Dual() : v(0.0), d{} {}
  __host__ __device__ constexpr Dual(double x) : v(x), d{} {}
};

template <int N>
__host__ __device__ inline Dual<N> operator+(const Dual<N>& a, const Dual<N>& b) {
  Dual<N> r(a.v + b.v);
  for (int k = 0; k < N; k++) r.d[k] = a.d[k] + b.d[k];
  return r;
}
template <int N>
__host__ __device__ inline Dual<N> operator-(const Dual<N>& a, const Dual<N>& b) {
  Dual<N> r(a.v - b.v);
  for (int k = 0; k < N; k++) r.d[k] = a.d[k] - b.d[k];
  return r;
}
template <int N>
__host__ __device__ inline Dual<N> operator-(const Dual<N>& a) {
  Dual<N> r(-a.v);
  for (int k = 0; k < N; k++) r.d[k] = -a.d[k];
  return r;
}
template <int N>
__host__ __device__ inline Dual<N> operator*(const Dual<N>& a, const Dual<N>& b) {
  Dual<N> r(a.v * b.v);
  for (int k = 0; k < N; k++) r.d[k] = a.d[k] * b.v + a.v * b.d[k];
  return r;
}
// The value is the IEEE quotient; the derivative parts are scaled by one
// reciprocal (an FP64 division costs many instructions, N of them dominated
// the dual arithmetic).
template <int N>
__host__ __device__ inline Dual<N> operator/(const Dual<N>& a, const Dual<N>& b) {
  Dual<N> r(a.v / b.v);
  const double inv = 1.0 / b.v;
  for (int k = 0; k < N; k++) r.d[k] = (a.d[k] - r.v * b.d[k]) * inv;
  return r;
}
template <int N>
__host__ __device__ inline Dual<N> operator+(const Dual<N>& a, double b) { return a + Dual<N>(b); }
template <int N>
__host__ __device__ inline Dual<N> operator+(double a, const Dual<N>& b) { return Dual<N>(a) + b; }
template <int N>
__host__ __device__ inline Dual<N> operator-(const Dual<N>& a, double b) { return a - Dual<N>(b); }
template <int N>
__host__ __device__ inline Dual<N> operator-(double a, const Dual<N>& b) { return Dual<N>(a) - b; }
template <int N>
__host__ __device__ inline Dual<N> operator*(const Dual<N>& a, double b) {
  Dual<N> r(a.v * b);
  for (int k = 0; k < N; k++) r.d[k] = a.d[k] * b;
  return r;
}
template <int N>
__host__ __device__ inline Dual<N> operator*(double a, const Dual<N>& b) { return b * a; }
template <int N>
__host__ __device__ inline Dual<N> operator/(const Dual<N>& a, double b) {
  Dual<N> r(a.v / b);
  const double inv = 1.0 / b;
  for (int k = 0; k < N; k++) r.d[k] = a.d[k] * inv;
  return r;
}
template <int N>
__host__ __device__ inline Dual<N> operator/(double a, const Dual<N>& b) { return Dual<N>(a) / b; }
template <int N, class T>
__host__ __device__ inline Dual<N>& operator+=(Dual<N>& a, const T& b) { return a = a + b; }
template <int N, class T>
__host__ __device__ inline Dual<N>& operator-=(Dual<N>& a, const T& b) { return a = a - b; }
template <int N, class T>
__host__ __device__ inline Dual<N>& operator*=(Dual<N>& a, const T& b) { return a = a * b; }
template <int N, class T>
__host__ __device__ inline Dual<N>& operator/=(Dual<N>& a, const T& b) { return a = a / b; }

__host__ __device__ inline double val(double a) { return a; }
template <int N>
__host__ __device__ inline double val(const Dual<N>& a) { return a.v; }

#define MHD_DUAL_CMP_(op)                                                                    \
  template <int N>                                                                           \
  __host__ __device__ inline bool operator op(const Dual<N>& a, const Dual<N>& b) {          \
    return a.v op b.v;                                                                       \
  }                                                                                          \
  template <int N>                                                                           \
  __host__ __device__ inline bool operator op(const Dual<N>& a, double b) { return a.v op b; } \
  template <int N>                                                                           \
  __host__ __device__ inline bool operator op(double a, const Dual<N>& b) { return a op b.v; }
MHD_DUAL_CMP_(<)
MHD_DUAL_CMP_(>)
MHD_DUAL_CMP_(<=)
MHD_DUAL_CMP_(>=)
#undef MHD_DUAL_CMP_

template <int N>
__host__ __device__ inline Dual<N> sqrt(const Dual<N>& a) {
  Dual<N> r(::sqrt(a.v));
  const double s = a.v > 0.0 ? 0.5 / r.v : 0.0;
  for (int k = 0; k < N; k++) r.d[k] = a.d[k] * s;
  return r;
}
template <int N>
__host__ __device__ inline Dual<N> fabs(const Dual<N>& a) {
  const double s = a.v > 0.0 ? 1.0 : (a.v < 0.0 ? -1.0 : 0.0);
  Dual<N> r(::fabs(a.v));
  for (int k = 0; k < N; k++) r.d[k] = a.d[k] * s;
  return r;
}
template <int N>
__host__ __device__ inline Dual<N> exp(const Dual<N>& a) {
  Dual<N> r(::exp(a.v));
  for (int k = 0; k < N; k++) r.d[k] = a.d[k] * r.v;
  return r;
}
template <int N>
__host__ __device__ inline Dual<N> pow(const Dual<N>& a, double e) {
  Dual<N> r(::pow(a.v, e));
  const double s = a.v != 0.0 ? e * r.v / a.v : 0.0;
  for (int k = 0; k < N; k++) r.d[k] = a.d[k] * s;
  return r;
}

// Scalar-generic spellings: one name for double and for Dual<N>, for code
// written over either (the global math functions cannot be overloaded in
// this namespace without ambiguity).
__host__ __device__ inline double gsqrt(double a) { return ::sqrt(a); }
__host__ __device__ inline double gfabs(double a) { return ::fabs(a); }
__host__ __device__ inline double gpow(double a, double e) { return ::pow(a, e); }
template <int N>
__host__ __device__ inline Dual<N> gsqrt(const Dual<N>& a) { return sqrt(a); }
template <int N>
__host__ __device__ inline Dual<N> gfabs(const Dual<N>& a) { return fabs(a); }
template <int N>
__host__ __device__ inline Dual<N> gpow(const Dual<N>& a, double e) { return pow(a, e); }

}  // namespace mhd
