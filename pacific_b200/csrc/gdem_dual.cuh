// gdem_dual.cuh -- forward-mode dual numbers for the contact-law Jacobians
// of the adjoint step.
//
// Dual<N> carries a value and N directional derivatives.  The contact law of
// the adjoint (gdem_adjoint.cu) is written once for a generic scalar and
// evaluated with Dual<1> seeded on one input at a time, which yields one
// column of the contact's Jacobian per evaluation; with Dual<3> seeded on
// (kn, en, muc) it gives the forward-mode check of the parameter gradient.
// Branches follow the value part, so a derivative is the derivative of the
// branch taken (the law is piecewise smooth).
#pragma once
#include <cuda_runtime.h>

namespace gdem {

template <int N>
struct Dual {
  static constexpr int kN = N;
  double v;
  double d[N];
};

template <int N>
__host__ __device__ __forceinline__ Dual<N> dconst(double a) {
  Dual<N> r;
  r.v = a;
#pragma unroll
  for (int k = 0; k < N; ++k) r.d[k] = 0.;
  return r;
}
template <int N>
__host__ __device__ __forceinline__ Dual<N> operator+(Dual<N> a, Dual<N> b) {
  Dual<N> r;
  r.v = a.v + b.v;
#pragma unroll
  for (int k = 0; k < N; ++k) r.d[k] = a.d[k] + b.d[k];
  return r;
}
template <int N>
__host__ __device__ __forceinline__ Dual<N> operator-(Dual<N> a, Dual<N> b) {
  Dual<N> r;
  r.v = a.v - b.v;
#pragma unroll
  for (int k = 0; k < N; ++k) r.d[k] = a.d[k] - b.d[k];
  return r;
}
template <int N>
__host__ __device__ __forceinline__ Dual<N> operator-(Dual<N> a) {
  Dual<N> r;
  r.v = -a.v;
#pragma unroll
  for (int k = 0; k < N; ++k) r.d[k] = -a.d[k];
  return r;
}
template <int N>
__host__ __device__ __forceinline__ Dual<N> operator*(Dual<N> a, Dual<N> b) {
  Dual<N> r;
  r.v = a.v * b.v;
#pragma unroll
  for (int k = 0; k < N; ++k) r.d[k] = a.d[k] * b.v + a.v * b.d[k];
  return r;
}
template <int N>
__host__ __device__ __forceinline__ Dual<N> operator/(Dual<N> a, Dual<N> b) {
  Dual<N> r;
  r.v = a.v / b.v;
  const double ib = 1. / b.v;
#pragma unroll
  for (int k = 0; k < N; ++k) r.d[k] = (a.d[k] - r.v * b.d[k]) * ib;
  return r;
}
template <int N>
__host__ __device__ __forceinline__ Dual<N> operator*(double s, Dual<N> a) {
  Dual<N> r;
  r.v = s * a.v;
#pragma unroll
  for (int k = 0; k < N; ++k) r.d[k] = s * a.d[k];
  return r;
}
template <int N>
__host__ __device__ __forceinline__ Dual<N> operator*(Dual<N> a, double s) { return s * a; }
template <int N>
__host__ __device__ __forceinline__ Dual<N> operator+(Dual<N> a, double s) {
  a.v += s;
  return a;
}
template <int N>
__host__ __device__ __forceinline__ Dual<N> operator+(double s, Dual<N> a) { return a + s; }
template <int N>
__host__ __device__ __forceinline__ Dual<N> operator-(Dual<N> a, double s) {
  a.v -= s;
  return a;
}
template <int N>
__host__ __device__ __forceinline__ Dual<N> operator-(double s, Dual<N> a) { return (-a) + s; }
template <int N>
__host__ __device__ __forceinline__ Dual<N> operator/(Dual<N> a, double s) {
  return a * (1. / s);
}
template <int N>
__host__ __device__ __forceinline__ Dual<N> operator/(double s, Dual<N> b) {
  return dconst<N>(s) / b;
}
template <int N>
__host__ __device__ __forceinline__ Dual<N> dsqrt(Dual<N> a) {
  Dual<N> r;
  r.v = sqrt(a.v);
  const double h = r.v > 0. ? 0.5 / r.v : 0.;
#pragma unroll
  for (int k = 0; k < N; ++k) r.d[k] = a.d[k] * h;
  return r;
}
__host__ __device__ __forceinline__ double dsqrt(double a) { return sqrt(a); }
template <int N>
__host__ __device__ __forceinline__ Dual<N> dlog(Dual<N> a) {
  Dual<N> r;
  r.v = log(a.v);
  const double ia = 1. / a.v;
#pragma unroll
  for (int k = 0; k < N; ++k) r.d[k] = a.d[k] * ia;
  return r;
}
__host__ __device__ __forceinline__ double dlog(double a) { return log(a); }
template <int N>
__host__ __device__ __forceinline__ Dual<N> dfabs(Dual<N> a) { return a.v < 0. ? -a : a; }
__host__ __device__ __forceinline__ double dfabs(double a) { return fabs(a); }
__host__ __device__ __forceinline__ double val(double a) { return a; }
template <int N>
__host__ __device__ __forceinline__ double val(Dual<N> a) { return a.v; }
// A constant of scalar type T.
template <typename T>
struct Scal {
  __host__ __device__ static T make(double a) { return dconst<T::kN>(a); }
};
template <>
struct Scal<double> {
  __host__ __device__ static double make(double a) { return a; }
};

// Generic 3-vector.
template <typename T>
struct V3 {
  T x, y, z;
};
template <typename T>
__host__ __device__ __forceinline__ V3<T> v3(T a, T b, T c) {
  V3<T> r;
  r.x = a; r.y = b; r.z = c;
  return r;
}
template <typename T>
__host__ __device__ __forceinline__ V3<T> operator+(V3<T> a, V3<T> b) {
  return v3(a.x + b.x, a.y + b.y, a.z + b.z);
}
template <typename T>
__host__ __device__ __forceinline__ V3<T> operator-(V3<T> a, V3<T> b) {
  return v3(a.x - b.x, a.y - b.y, a.z - b.z);
}
template <typename T>
__host__ __device__ __forceinline__ V3<T> operator-(V3<T> a) { return v3(-a.x, -a.y, -a.z); }
template <typename T>
__host__ __device__ __forceinline__ V3<T> operator*(T s, V3<T> a) {
  return v3(s * a.x, s * a.y, s * a.z);
}
template <typename T>
__host__ __device__ __forceinline__ V3<T> operator/(V3<T> a, T s) {
  return v3(a.x / s, a.y / s, a.z / s);
}
template <typename T>
__host__ __device__ __forceinline__ T vdot(V3<T> a, V3<T> b) {
  return a.x * b.x + a.y * b.y + a.z * b.z;
}
template <typename T>
__host__ __device__ __forceinline__ V3<T> vcross(V3<T> a, V3<T> b) {
  return v3(a.y * b.z - a.z * b.y, -a.x * b.z + a.z * b.x, a.x * b.y - a.y * b.x);
}
template <typename T>
__host__ __device__ __forceinline__ T vnorm(V3<T> a) { return dsqrt(vdot(a, a)); }

}  // namespace gdem
