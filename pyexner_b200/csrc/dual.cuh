// Forward-mode dual numbers for the tangent-linear (JVP) model of the float64 step.
//
// A Dual carries a value and a directional derivative.  Its value part performs exactly
// the float64 operations of the plain build (the translation unit that instantiates the
// kernels on Dual is compiled with --fmad=false, like the float64 one), so the value of a
// dual run is the float64 run bit for bit; the derivative part follows the chain rule.
// Branches and selects (wet/dry, upwinding, clamps) take the value's branch, as JAX's
// forward mode does through jnp.where; at a clamp tie (x == lo exactly) the tangent of x
// is kept where JAX would average the two.  Where the chain rule gives 0 * inf (a square
// or cube root, or acos, at a point where the argument's tangent is zero, e.g. the
// (theta - theta_c)^0.5 factor of MPM below the Shields threshold), the tangent is 0.
#pragma once
#include <cmath>
#include <cstdint>

namespace pxb {

struct Dual {
    double v, d;
    __host__ __device__ Dual() : v(0.0), d(0.0) {}
    __host__ __device__ Dual(double x) : v(x), d(0.0) {}
    __host__ __device__ Dual(double x, double t) : v(x), d(t) {}
};

__host__ __device__ inline Dual operator+(Dual a, Dual b) { return Dual(a.v + b.v, a.d + b.d); }
__host__ __device__ inline Dual operator-(Dual a, Dual b) { return Dual(a.v - b.v, a.d - b.d); }
__host__ __device__ inline Dual operator-(Dual a) { return Dual(-a.v, -a.d); }
__host__ __device__ inline Dual operator*(Dual a, Dual b) { return Dual(a.v * b.v, a.d * b.v + a.v * b.d); }
__host__ __device__ inline Dual operator/(Dual a, Dual b) {
    const double q = a.v / b.v;
    return Dual(q, (a.d - q * b.d) / b.v);
}
__host__ __device__ inline Dual& operator+=(Dual& a, Dual b) { return a = a + b; }
__host__ __device__ inline Dual& operator*=(Dual& a, Dual b) { return a = a * b; }
__host__ __device__ inline bool operator<(Dual a, Dual b) { return a.v < b.v; }
__host__ __device__ inline bool operator>(Dual a, Dual b) { return a.v > b.v; }
__host__ __device__ inline bool operator<=(Dual a, Dual b) { return a.v <= b.v; }
__host__ __device__ inline bool operator>=(Dual a, Dual b) { return a.v >= b.v; }
__host__ __device__ inline bool operator==(Dual a, Dual b) { return a.v == b.v; }
__host__ __device__ inline bool operator!=(Dual a, Dual b) { return a.v != b.v; }

// tangent t * f'(x) with 0 where t == 0 (no 0 * inf)
__host__ __device__ inline double chain(double t, double fprime) { return t == 0.0 ? 0.0 : t * fprime; }

__device__ inline Dual d_sqrt(Dual x) {
    const double s = sqrt(x.v);
    return Dual(s, chain(x.d, 0.5 / s));
}
__device__ inline Dual d_cbrt(Dual x) {
    const double c = cbrt(x.v);
    return Dual(c, chain(x.d, 1.0 / (3.0 * c * c)));
}
__device__ inline Dual d_pow(Dual x, Dual y) {
    const double p = pow(x.v, y.v);
    double t = chain(x.d, y.v * pow(x.v, y.v - 1.0));
    if (y.d != 0.0) t += log(x.v) * p * y.d;
    return Dual(p, t);
}
__device__ inline Dual d_acos(Dual x) { return Dual(acos(x.v), chain(x.d, -1.0 / sqrt(1.0 - x.v * x.v))); }
__device__ inline Dual d_cos(Dual x) { return Dual(cos(x.v), chain(x.d, -sin(x.v))); }
__device__ inline Dual fabs(Dual x) { return Dual(::fabs(x.v), x.v > 0.0 ? x.d : (x.v < 0.0 ? -x.d : 0.0)); }
__device__ inline bool d_isfinite(Dual x) { return isfinite(x.v); }
__device__ inline Dual mul_rn(Dual a, Dual b) { return a * b; }

// host side: x^y for a constant exponent (set-up tables)
__host__ inline Dual hpow(Dual x, double y) {
    const double p = std::pow(x.v, y);
    return Dual(p, chain(x.d, y * std::pow(x.v, y - 1.0)));
}

// Scratch and arguments of the dual CFL reduction (tangent.cuh).
struct DualScratch {
    unsigned long long maxbits;  // running max of the speed values' bits
    double dsum;                 // sum of the tangents of the faces at the maximum
    double t_step, t_next;       // simulation time of the step (as CflScratch)
    unsigned int step;
    unsigned int nties;          // number of faces at the maximum
};

struct DualCflArgs {
    int ny, nx;
    long long pitch;
    const Dual *h, *hu, *hv, *G;
    const uint8_t* nodata;
    double dx, cfl, floor_dt;
    DualScratch* scr;
    Dual* dt_out;
    double* dt_log;      // optional values of dt per step
    double* dt_dot_log;  // optional tangents of dt per step
    int* err;            // the plan's error word (bit 2: non-finite dt)
};

}  // namespace pxb
