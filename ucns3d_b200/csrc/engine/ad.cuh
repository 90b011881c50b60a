// Forward-mode dual numbers for the discrete adjoint and tangent kernels.
//
// Dual<N> carries a value and N directional derivatives.  The templated gas,
// rotation, HLLC, limiter and boundary functions of device.cuh evaluated on
// Dual<N> give their exact derivatives (up to rounding) along N seeded
// directions: N = 1 for the tangent, N = 10 for the 5x10 Jacobian of a face
// flux with respect to its two states (or state and free-stream state), which
// the adjoint then applies transposed.  Branches (wave-speed selection, the
// sign of the contact speed, limiter cases, supersonic switches) follow the
// values, so each derivative is that of the branch the primal takes.
//
// The type and its overloads live in their own namespace so that they are
// found only by argument-dependent lookup and never shadow the double
// versions of sqrt/fmin/... .
#pragma once

#include "device.cuh"

namespace ucg {
namespace ad {

template <int N>
struct Dual {
  double v;
  double d[N];
  __host__ __device__ __forceinline__ Dual() {}
  __host__ __device__ __forceinline__ Dual(double x) : v(x) {
#pragma unroll
    for (int i = 0; i < N; ++i) d[i] = 0.0;
  }
};

template <int N>
__host__ __device__ __forceinline__ double value(const Dual<N>& a) {
  return a.v;
}

template <int N>
__host__ __device__ __forceinline__ Dual<N> operator-(const Dual<N>& a) {
  Dual<N> r;
  r.v = -a.v;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = -a.d[i];
  return r;
}
template <int N>
__host__ __device__ __forceinline__ Dual<N> operator+(const Dual<N>& a, const Dual<N>& b) {
  Dual<N> r;
  r.v = a.v + b.v;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = a.d[i] + b.d[i];
  return r;
}
template <int N>
__host__ __device__ __forceinline__ Dual<N> operator-(const Dual<N>& a, const Dual<N>& b) {
  Dual<N> r;
  r.v = a.v - b.v;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = a.d[i] - b.d[i];
  return r;
}
template <int N>
__host__ __device__ __forceinline__ Dual<N> operator*(const Dual<N>& a, const Dual<N>& b) {
  Dual<N> r;
  r.v = a.v * b.v;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * b.v + a.v * b.d[i];
  return r;
}
template <int N>
__host__ __device__ __forceinline__ Dual<N> operator/(const Dual<N>& a, const Dual<N>& b) {
  Dual<N> r;
  r.v = a.v / b.v;
  const double ib = 1.0 / b.v;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = (a.d[i] - r.v * b.d[i]) * ib;
  return r;
}
template <int N>
__host__ __device__ __forceinline__ Dual<N> operator+(const Dual<N>& a, double b) {
  Dual<N> r = a;
  r.v = a.v + b;
  return r;
}
template <int N>
__host__ __device__ __forceinline__ Dual<N> operator+(double a, const Dual<N>& b) {
  Dual<N> r = b;
  r.v = a + b.v;
  return r;
}
template <int N>
__host__ __device__ __forceinline__ Dual<N> operator-(const Dual<N>& a, double b) {
  Dual<N> r = a;
  r.v = a.v - b;
  return r;
}
template <int N>
__host__ __device__ __forceinline__ Dual<N> operator-(double a, const Dual<N>& b) {
  Dual<N> r;
  r.v = a - b.v;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = -b.d[i];
  return r;
}
template <int N>
__host__ __device__ __forceinline__ Dual<N> operator*(const Dual<N>& a, double b) {
  Dual<N> r;
  r.v = a.v * b;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * b;
  return r;
}
template <int N>
__host__ __device__ __forceinline__ Dual<N> operator*(double a, const Dual<N>& b) {
  Dual<N> r;
  r.v = a * b.v;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = a * b.d[i];
  return r;
}
template <int N>
__host__ __device__ __forceinline__ Dual<N> operator/(const Dual<N>& a, double b) {
  Dual<N> r;
  r.v = a.v / b;
  const double ib = 1.0 / b;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * ib;
  return r;
}
template <int N>
__host__ __device__ __forceinline__ Dual<N> operator/(double a, const Dual<N>& b) {
  Dual<N> r;
  r.v = a / b.v;
  const double s = -r.v / b.v;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = s * b.d[i];
  return r;
}
template <int N>
__host__ __device__ __forceinline__ Dual<N> sqrt(const Dual<N>& a) {
  Dual<N> r;
  r.v = ::sqrt(a.v);
  const double s = 0.5 / r.v;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = s * a.d[i];
  return r;
}
template <int N>
__host__ __device__ __forceinline__ Dual<N> fabs(const Dual<N>& a) {
  return a.v < 0.0 ? -a : a;
}
template <int N>
__host__ __device__ __forceinline__ Dual<N> fmin(const Dual<N>& a, const Dual<N>& b) {
  return b.v < a.v ? b : a;
}
template <int N>
__host__ __device__ __forceinline__ Dual<N> fmax(const Dual<N>& a, const Dual<N>& b) {
  return b.v > a.v ? b : a;
}
template <int N>
__host__ __device__ __forceinline__ Dual<N> fmin(const Dual<N>& a, double b) {
  return b < a.v ? Dual<N>(b) : a;
}
template <int N>
__host__ __device__ __forceinline__ Dual<N> fmax(const Dual<N>& a, double b) {
  return b > a.v ? Dual<N>(b) : a;
}

}  // namespace ad
}  // namespace ucg
