// dual.cuh -- forward-mode dual numbers with N partials, for the Jacobians of the
// advection schemes.  Evaluating the scheme templates of schemes.cuh on D<N> gives the
// face flux and its exact derivatives along the branch the FP64 form takes (the
// switches and limiters are decided on the values), so tangent-linear and adjoint
// kernels use the very arithmetic of the forward kernels.
#pragma once
#include <cuda_runtime.h>

#include "schemes.cuh"

template <int N> struct D {
    double v;
    double d[N];
    __host__ __device__ __forceinline__ D() : v(0.) {
#pragma unroll
        for (int q = 0; q < N; q++) d[q] = 0.;
    }
    __host__ __device__ __forceinline__ D(double x) : v(x) {
#pragma unroll
        for (int q = 0; q < N; q++) d[q] = 0.;
    }
    // the q-th independent variable with value x
    __host__ __device__ __forceinline__ static D var(double x, int q) {
        D r(x);
        r.d[q] = 1.;
        return r;
    }
};

template <int N> __host__ __device__ __forceinline__ D<N> operator+(const D<N> &a, const D<N> &b)
{
    D<N> r(a.v + b.v);
#pragma unroll
    for (int q = 0; q < N; q++) r.d[q] = a.d[q] + b.d[q];
    return r;
}
template <int N> __host__ __device__ __forceinline__ D<N> operator-(const D<N> &a, const D<N> &b)
{
    D<N> r(a.v - b.v);
#pragma unroll
    for (int q = 0; q < N; q++) r.d[q] = a.d[q] - b.d[q];
    return r;
}
template <int N> __host__ __device__ __forceinline__ D<N> operator-(const D<N> &a)
{
    D<N> r(-a.v);
#pragma unroll
    for (int q = 0; q < N; q++) r.d[q] = -a.d[q];
    return r;
}
template <int N> __host__ __device__ __forceinline__ D<N> operator*(const D<N> &a, const D<N> &b)
{
    D<N> r(a.v * b.v);
#pragma unroll
    for (int q = 0; q < N; q++) r.d[q] = a.d[q] * b.v + a.v * b.d[q];
    return r;
}
// the value is the correctly rounded quotient (the forward's); the partials use one
// reciprocal of the divisor
template <int N> __host__ __device__ __forceinline__ D<N> operator/(const D<N> &a, const D<N> &b)
{
    const double qv = a.v / b.v;
    const double rb = 1. / b.v;
    D<N> r(qv);
#pragma unroll
    for (int q = 0; q < N; q++) r.d[q] = (a.d[q] - qv * b.d[q]) * rb;
    return r;
}
template <int N> __host__ __device__ __forceinline__ bool operator<(const D<N> &a, const D<N> &b) { return a.v < b.v; }
template <int N> __host__ __device__ __forceinline__ bool operator>(const D<N> &a, const D<N> &b) { return a.v > b.v; }
template <int N> __host__ __device__ __forceinline__ D<N> dabs(const D<N> &a) { return a.v < 0. ? -a : a; }

template <> __host__ __device__ __forceinline__ bool ratio_gt<D<5>>(D<5> a, D<5> b, D<5> thr) { return ratio_gt<double>(a.v, b.v, thr.v); }
template <> __host__ __device__ __forceinline__ bool ratio_gt<D<4>>(D<4> a, D<4> b, D<4> thr) { return ratio_gt<double>(a.v, b.v, thr.v); }
// min(|num/den|, 1), branch decided on the values exactly as the FP64 form decides it
template <int N> __host__ __device__ __forceinline__ D<N> min_abs_ratio_1_dual(const D<N> &num, const D<N> &den)
{
    if (fabs(num.v) >= fabs(den.v)) return D<N>(1.);
    const D<N> q = dabs(num / den);
    return q.v < 1. ? q : D<N>(1.);
}
template <> __host__ __device__ __forceinline__ D<5> min_abs_ratio_1<D<5>>(D<5> num, D<5> den) { return min_abs_ratio_1_dual(num, den); }
template <> __host__ __device__ __forceinline__ D<4> min_abs_ratio_1<D<4>>(D<4> num, D<4> den) { return min_abs_ratio_1_dual(num, den); }
