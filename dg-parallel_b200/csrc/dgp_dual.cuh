// Forward-mode dual numbers: a value and its derivatives along N directions.
// The point physics in dgp_laws.cuh is templated on its arithmetic type, so
// evaluating it on Dual<T, N> yields the exact Jacobians of the volume,
// numerical and boundary fluxes that the discrete adjoint needs (the adjoint
// Riemann-flux Jacobians are the Jacobians of the very code the forward step
// runs, branches included).
#pragma once

#include <cuda_runtime.h>

namespace dgp {

// the plain overloads stay visible next to the Dual ones inside the namespace
using ::exp;
using ::fabs;
using ::pow;
using ::sqrt;

template <typename T, int N>
struct Dual {
  T v;
  T d[N];
  __device__ __forceinline__ Dual() : v(0) {
#pragma unroll
    for (int i = 0; i < N; ++i) d[i] = 0;
  }
  // constants (literals, law parameters, far-field values)
  __device__ __forceinline__ Dual(double c) : v((T)c) {
#pragma unroll
    for (int i = 0; i < N; ++i) d[i] = 0;
  }
  __device__ __forceinline__ Dual(float c) : v((T)c) {
#pragma unroll
    for (int i = 0; i < N; ++i) d[i] = 0;
  }
  __device__ __forceinline__ Dual(int c) : v((T)c) {
#pragma unroll
    for (int i = 0; i < N; ++i) d[i] = 0;
  }
  // the k-th input variable with value x (k outside [0, N): a constant)
  __device__ static __forceinline__ Dual var(T x, int k) {
    Dual r(0);
    r.v = x;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = (i == k) ? (T)1 : (T)0;
    return r;
  }
  __device__ __forceinline__ Dual& operator+=(const Dual& b) { return *this = *this + b; }
  __device__ __forceinline__ Dual& operator-=(const Dual& b) { return *this = *this - b; }
  __device__ __forceinline__ Dual& operator*=(const Dual& b) { return *this = *this * b; }
  __device__ __forceinline__ Dual& operator/=(const Dual& b) { return *this = *this / b; }
  __device__ friend __forceinline__ Dual operator+(const Dual& a, const Dual& b) {
    Dual r;
    r.v = a.v + b.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] + b.d[i];
    return r;
  }
  __device__ friend __forceinline__ Dual operator-(const Dual& a, const Dual& b) {
    Dual r;
    r.v = a.v - b.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] - b.d[i];
    return r;
  }
  __device__ friend __forceinline__ Dual operator-(const Dual& a) {
    Dual r;
    r.v = -a.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = -a.d[i];
    return r;
  }
  __device__ friend __forceinline__ Dual operator*(const Dual& a, const Dual& b) {
    Dual r;
    r.v = a.v * b.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * b.v + a.v * b.d[i];
    return r;
  }
  __device__ friend __forceinline__ Dual operator/(const Dual& a, const Dual& b) {
    Dual r;
    const T ib = (T)1 / b.v;
    r.v = a.v * ib;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = (a.d[i] - r.v * b.d[i]) * ib;
    return r;
  }
  // comparisons act on values (the branch the primal code takes)
  __device__ friend __forceinline__ bool operator<(const Dual& a, const Dual& b) { return a.v < b.v; }
  __device__ friend __forceinline__ bool operator>(const Dual& a, const Dual& b) { return a.v > b.v; }
  __device__ friend __forceinline__ bool operator<=(const Dual& a, const Dual& b) { return a.v <= b.v; }
  __device__ friend __forceinline__ bool operator>=(const Dual& a, const Dual& b) { return a.v >= b.v; }
};

template <typename T, int N>
__device__ __forceinline__ Dual<T, N> sqrt(const Dual<T, N>& a) {
  Dual<T, N> r;
  r.v = ::sqrt(a.v);
  const T h = (T)0.5 / r.v;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * h;
  return r;
}

template <typename T, int N>
__device__ __forceinline__ Dual<T, N> rsqrt(const Dual<T, N>& a) {
  Dual<T, N> r;
  r.v = ::rsqrt(a.v);
  const T dr = (T)-0.5 * r.v * r.v * r.v;  // d/dx x^(-1/2)
#pragma unroll
  for (int k = 0; k < N; ++k) r.d[k] = dr * a.d[k];
  return r;
}

template <typename T, int N>
__device__ __forceinline__ Dual<T, N> fabs(const Dual<T, N>& a) {
  return a.v < (T)0 ? -a : a;
}

template <typename T, int N>
__device__ __forceinline__ Dual<T, N> exp(const Dual<T, N>& a) {
  Dual<T, N> r;
  r.v = ::exp(a.v);
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * r.v;
  return r;
}

// a^c for a constant exponent
template <typename T, int N>
__device__ __forceinline__ Dual<T, N> pow(const Dual<T, N>& a, const Dual<T, N>& c) {
  Dual<T, N> r;
  r.v = ::pow(a.v, c.v);
  const T g = c.v * ::pow(a.v, c.v - (T)1);
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * g;
  return r;
}

}  // namespace dgp
