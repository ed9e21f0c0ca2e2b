// First-order dual numbers (value, derivative along one direction) for the
// tangent (forward-mode) derivatives of the metric and residual expressions:
// every operation applies the chain rule of the operation it replaces, in the
// same operand order, so the value part equals the plain FP64 evaluation.
#pragma once

#include <cuda_runtime.h>

namespace v2d {

struct Dual {
    double v, d;
};

__host__ __device__ __forceinline__ Dual dual_const(double v) { return {v, 0.0}; }

__host__ __device__ __forceinline__ Dual operator-(Dual a) { return {-a.v, -a.d}; }
__host__ __device__ __forceinline__ Dual operator+(Dual a, Dual b) { return {a.v + b.v, a.d + b.d}; }
__host__ __device__ __forceinline__ Dual operator+(Dual a, double b) { return {a.v + b, a.d}; }
__host__ __device__ __forceinline__ Dual operator+(double a, Dual b) { return {a + b.v, b.d}; }
__host__ __device__ __forceinline__ Dual operator-(Dual a, Dual b) { return {a.v - b.v, a.d - b.d}; }
__host__ __device__ __forceinline__ Dual operator-(Dual a, double b) { return {a.v - b, a.d}; }
__host__ __device__ __forceinline__ Dual operator-(double a, Dual b) { return {a - b.v, -b.d}; }
__host__ __device__ __forceinline__ Dual operator*(Dual a, Dual b)
{
    return {a.v * b.v, a.d * b.v + a.v * b.d};
}
__host__ __device__ __forceinline__ Dual operator*(Dual a, double b) { return {a.v * b, a.d * b}; }
__host__ __device__ __forceinline__ Dual operator*(double a, Dual b) { return {a * b.v, a * b.d}; }
// (a/b)' = (a' - (a/b) b') / b
__host__ __device__ __forceinline__ Dual operator/(Dual a, Dual b)
{
    const double q = a.v / b.v;
    return {q, (a.d - q * b.d) / b.v};
}
__host__ __device__ __forceinline__ Dual operator/(Dual a, double b) { return {a.v / b, a.d / b}; }
__host__ __device__ __forceinline__ Dual operator/(double a, Dual b)
{
    const double q = a / b.v;
    return {q, -q * b.d / b.v};
}
__host__ __device__ __forceinline__ Dual& operator+=(Dual &a, Dual b)
{
    a.v += b.v;
    a.d += b.d;
    return a;
}
// square root for templated code: tsqrt(double) is the plain sqrt
__host__ __device__ __forceinline__ double tsqrt(double a) { return ::sqrt(a); }
__host__ __device__ __forceinline__ Dual tsqrt(Dual a)
{
    const double r = ::sqrt(a.v);
    return {r, a.d / (2.0 * r)};
}

// a constant of either type
template <class T> __host__ __device__ __forceinline__ T tconst(double v);
template <> __host__ __device__ __forceinline__ double tconst<double>(double v) { return v; }
template <> __host__ __device__ __forceinline__ Dual tconst<Dual>(double v) { return {v, 0.0}; }

// value of a scalar of either type (branch conditions compare values)
__host__ __device__ __forceinline__ double value_of(double a) { return a; }
__host__ __device__ __forceinline__ double value_of(Dual a) { return a.v; }

}  // namespace v2d
