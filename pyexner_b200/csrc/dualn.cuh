// Dual numbers with N tangent directions, for the local Jacobians of the reverse-mode
// (adjoint) kernels: one evaluation of a face or cell formula on DualN<N> inputs seeded
// with the N inputs of one cell gives the derivatives of its outputs with respect to
// those inputs.  Value arithmetic is the plain float64 arithmetic (the translation unit
// is compiled with --fmad=false); branch and tie conventions are those of Dual.
#pragma once
#include <cmath>

#include "dual.cuh"

namespace pxb {

template <int N>
struct DualN {
    double v;
    double d[N];
    __host__ __device__ DualN() : v(0.0) {
        for (int k = 0; k < N; ++k) d[k] = 0.0;
    }
    __host__ __device__ DualN(double x) : v(x) {
        for (int k = 0; k < N; ++k) d[k] = 0.0;
    }
    // input k of the seeded set
    __host__ __device__ static DualN seed(double x, int k) {
        DualN r(x);
        r.d[k] = 1.0;
        return r;
    }

    friend __host__ __device__ DualN operator+(const DualN& a, const DualN& b) {
        DualN r(a.v + b.v);
        for (int k = 0; k < N; ++k) r.d[k] = a.d[k] + b.d[k];
        return r;
    }
    friend __host__ __device__ DualN operator-(const DualN& a, const DualN& b) {
        DualN r(a.v - b.v);
        for (int k = 0; k < N; ++k) r.d[k] = a.d[k] - b.d[k];
        return r;
    }
    friend __host__ __device__ DualN operator-(const DualN& a) {
        DualN r(-a.v);
        for (int k = 0; k < N; ++k) r.d[k] = -a.d[k];
        return r;
    }
    friend __host__ __device__ DualN operator*(const DualN& a, const DualN& b) {
        DualN r(a.v * b.v);
        for (int k = 0; k < N; ++k) r.d[k] = a.d[k] * b.v + a.v * b.d[k];
        return r;
    }
    friend __host__ __device__ DualN operator/(const DualN& a, const DualN& b) {
        const double q = a.v / b.v;
        DualN r(q);
        for (int k = 0; k < N; ++k) r.d[k] = (a.d[k] - q * b.d[k]) / b.v;
        return r;
    }
    friend __host__ __device__ bool operator<(const DualN& a, const DualN& b) { return a.v < b.v; }
    friend __host__ __device__ bool operator>(const DualN& a, const DualN& b) { return a.v > b.v; }
    friend __host__ __device__ bool operator<=(const DualN& a, const DualN& b) { return a.v <= b.v; }
    friend __host__ __device__ bool operator>=(const DualN& a, const DualN& b) { return a.v >= b.v; }
    friend __host__ __device__ bool operator==(const DualN& a, const DualN& b) { return a.v == b.v; }
    friend __host__ __device__ bool operator!=(const DualN& a, const DualN& b) { return a.v != b.v; }

    // f(x) with f'(x) = fp, tangents that are exactly 0 stay 0 (no 0 * inf)
    __host__ __device__ DualN apply(double fx, double fp) const {
        DualN r(fx);
        for (int k = 0; k < N; ++k) r.d[k] = chain(d[k], fp);
        return r;
    }

    friend __device__ DualN d_sqrt(const DualN& x) {
        const double s = sqrt(x.v);
        return x.apply(s, 0.5 / s);
    }
    friend __device__ DualN d_cbrt(const DualN& x) {
        const double c = cbrt(x.v);
        return x.apply(c, 1.0 / (3.0 * c * c));
    }
    friend __device__ DualN d_pow(const DualN& x, const DualN& y) {  // constant exponents only
        const double p = pow(x.v, y.v);
        return x.apply(p, y.v * pow(x.v, y.v - 1.0));
    }
    friend __device__ DualN d_acos(const DualN& x) { return x.apply(acos(x.v), -1.0 / sqrt(1.0 - x.v * x.v)); }
    friend __device__ DualN d_cos(const DualN& x) { return x.apply(cos(x.v), -sin(x.v)); }
    friend __device__ DualN fabs(const DualN& x) {
        DualN r(::fabs(x.v));
        for (int k = 0; k < N; ++k) r.d[k] = x.v > 0.0 ? x.d[k] : (x.v < 0.0 ? -x.d[k] : 0.0);
        return r;
    }
    friend __device__ bool d_isfinite(const DualN& x) { return isfinite(x.v); }
    friend __device__ DualN mul_rn(const DualN& a, const DualN& b) { return a * b; }
};

}  // namespace pxb
