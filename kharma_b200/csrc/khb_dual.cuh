// khb_dual.cuh -- forward-mode dual numbers (value and one tangent) for the adjoint kernels.
//
// The adjoint of each local operator (a face flux, a zone's source, a zone's P -> U) needs that
// operator's Jacobian.  Evaluating the same templated device functions the forward kernels use
// (calc_4vecs, prim_to_flux, vchar, mc_lim ...) on Dual<T> seeded with a unit tangent on one input
// gives one column of the Jacobian; branches (max, min, the MC limiter) follow the value, as the
// forward evaluation does.
#pragma once

#include <cuda_runtime.h>

namespace khb {

template <typename T>
struct Dual {
    T v, d;
    __host__ __device__ __forceinline__ Dual() {}
    __host__ __device__ __forceinline__ Dual(T x) : v(x), d(T(0)) {}
    __host__ __device__ __forceinline__ Dual(T x, T dx) : v(x), d(dx) {}
    __host__ __device__ __forceinline__ Dual& operator+=(const Dual& o) { v += o.v; d += o.d; return *this; }
    __host__ __device__ __forceinline__ Dual& operator-=(const Dual& o) { v -= o.v; d -= o.d; return *this; }
    __host__ __device__ __forceinline__ Dual& operator*=(const Dual& o) { d = d * o.v + v * o.d; v *= o.v; return *this; }
};

template <typename T> __host__ __device__ __forceinline__ Dual<T> operator+(Dual<T> a, Dual<T> b) { return Dual<T>(a.v + b.v, a.d + b.d); }
template <typename T> __host__ __device__ __forceinline__ Dual<T> operator-(Dual<T> a, Dual<T> b) { return Dual<T>(a.v - b.v, a.d - b.d); }
template <typename T> __host__ __device__ __forceinline__ Dual<T> operator-(Dual<T> a) { return Dual<T>(-a.v, -a.d); }
template <typename T> __host__ __device__ __forceinline__ Dual<T> operator*(Dual<T> a, Dual<T> b) { return Dual<T>(a.v * b.v, a.d * b.v + a.v * b.d); }
template <typename T> __host__ __device__ __forceinline__ Dual<T> operator/(Dual<T> a, Dual<T> b)
{
    const T q = a.v / b.v;
    return Dual<T>(q, (a.d - q * b.d) / b.v);
}
template <typename T> __host__ __device__ __forceinline__ bool operator<(Dual<T> a, Dual<T> b) { return a.v < b.v; }
template <typename T> __host__ __device__ __forceinline__ bool operator>(Dual<T> a, Dual<T> b) { return a.v > b.v; }
template <typename T> __host__ __device__ __forceinline__ bool operator<=(Dual<T> a, Dual<T> b) { return a.v <= b.v; }
template <typename T> __host__ __device__ __forceinline__ bool operator>=(Dual<T> a, Dual<T> b) { return a.v >= b.v; }

__device__ __forceinline__ Dual<double> dsqrt(Dual<double> a)
{
    const double s = sqrt(a.v);
    return Dual<double>(s, (s > 0.) ? a.d / (2. * s) : 0.);
}
__device__ __forceinline__ Dual<float> dsqrt(Dual<float> a)
{
    const float s = sqrtf(a.v);
    return Dual<float>(s, (s > 0.f) ? a.d / (2.f * s) : 0.f);
}
__device__ __forceinline__ Dual<double> dabs(Dual<double> a) { return (a.v < 0.) ? -a : a; }
__device__ __forceinline__ Dual<float> dabs(Dual<float> a) { return (a.v < 0.f) ? -a : a; }

} // namespace khb
