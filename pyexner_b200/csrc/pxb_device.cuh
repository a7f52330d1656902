// Device-side building blocks of the PyExner B200 step: constants, NaN-faithful
// helpers, per-cell precomputes and the per-face Riemann / bedload / wave-speed math.
//
// The arithmetic follows the reference expression by expression (operation order,
// clamps, masks) so that the float64 build, compiled with --fmad=false, reproduces the
// reference to rounding of the transcendental functions.  Citations are to PyExner's
// src/PyExner/solvers/kernels/roe_exner.py unless stated otherwise.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "pxb_types.h"

namespace pxb {

constexpr double G_ACC = 9.81;     // src/utils/constants.py:33
constexpr double DRY_TOL = 1e-4;   // constants.py:29
constexpr double SED_TOL = 1e-5;   // constants.py:30
constexpr double VEL_TOL = 1e-6;   // constants.py:31
constexpr double DT_FLOOR = 1e-6;  // roe_exner_solver.py:121
constexpr double TWO_PI = 6.283185307179586;  // 2*jnp.pi as a Python float
constexpr unsigned FULL = 0xffffffffu;

// jnp.maximum(x, lo) for a constant lo: NaN in x propagates.
template <class T>
__device__ __forceinline__ T clamp_lo(T x, T lo) { return x < lo ? lo : x; }
// jnp.maximum(a, b) with NaN from either side.
template <class T>
__device__ __forceinline__ T nan_max(T a, T b) { return (a < b || b != b) ? b : a; }
// jnp.clip(x, -1, 1) keeping NaN.
template <class T>
__device__ __forceinline__ T clip1(T x) { return x < T(-1) ? T(-1) : (x > T(1) ? T(1) : x); }

__device__ __forceinline__ float d_sqrt(float x) { return sqrtf(x); }
__device__ __forceinline__ double d_sqrt(double x) { return sqrt(x); }
__device__ __forceinline__ float d_cbrt(float x) { return cbrtf(x); }
__device__ __forceinline__ double d_cbrt(double x) { return cbrt(x); }
__device__ __forceinline__ float d_pow(float x, float y) { return powf(x, y); }
__device__ __forceinline__ double d_pow(double x, double y) { return pow(x, y); }
__device__ __forceinline__ float d_acos(float x) { return acosf(x); }
__device__ __forceinline__ double d_acos(double x) { return acos(x); }
__device__ __forceinline__ float d_cos(float x) { return cosf(x); }
__device__ __forceinline__ double d_cos(double x) { return cos(x); }
__device__ __forceinline__ bool d_isfinite(float x) { return isfinite(x); }
__device__ __forceinline__ bool d_isfinite(double x) { return isfinite(x); }

// Float32 building blocks.  The float build trades the last ulp for throughput: the
// hardware approximations below are accurate to about 2^-22 relative, far inside the
// float32 accuracy budget of the step.  The float64 build uses none of them.
__device__ __forceinline__ float f_rcp(float x) { float y; asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x)); return y; }
__device__ __forceinline__ float f_rsqrt(float x) { float y; asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x)); return y; }
__device__ __forceinline__ float f_sqrt(float x) { float y; asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x)); return y; }
__device__ __forceinline__ float f_lg2(float x) { float y; asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x)); return y; }
__device__ __forceinline__ float f_ex2(float x) { float y; asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x)); return y; }
// Products that must not be fused into an FMA: sign decisions of the Exner upwinding
// depend on exact cancellations (mirror states at reflective walls give exactly 0).
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
template <class T>
__host__ __device__ constexpr bool is_f32() { return sizeof(T) == 4; }

// Sums of several products.  The float build contracts a * b + c into one FMA, but a
// sum of two products can be contracted either way and the compiler's choice depends on
// the code around the inlined expression, so two kernels sharing a formula could differ
// in the last bit.  Such sums are spelled out here:
//   sum2 / dif2: both products rounded on their own, then added (mirror states at
//                reflective walls cancel exactly, as in the reference's arithmetic);
//   fsum2:       a * b fused onto the rounded c * d (sums of squares, no cancellation).
// In the float64 build (--fmad=false) all three are the plain expression.
template <class T>
__device__ __forceinline__ T sum2(T a, T b, T c, T d) { return mul_rn(a, b) + mul_rn(c, d); }
template <class T>
__device__ __forceinline__ T dif2(T a, T b, T c, T d) { return mul_rn(a, b) - mul_rn(c, d); }
__device__ __forceinline__ float fsum2(float a, float b, float c, float d) { return __fmaf_rn(a, b, __fmul_rn(c, d)); }

// ---------------------------------------------------------------- hydrodynamic faces
// Per-cell values used by the Roe-Exner face flux (roe_exner.py:317-335, 421-425, 455).
template <class T>
struct HCell {
    T h;   // max(h, DRY_TOL)
    T u;   // hu / h if wet else 0
    T v;
    T sq;  // sqrt(h)
    T c;   // sqrt(g h)
    T zt;  // z + z_b with z_b floored at SED_TOL*0.01 below SED_TOL
    T nb;  // n_b
};

template <class T>
__device__ __forceinline__ HCell<T> make_hcell(T h, T hu, T hv, T zb, T z, T nb) {
    HCell<T> p;
    const T hc = clamp_lo(h, T(DRY_TOL));
    const bool wet = hc > T(DRY_TOL);
    p.h = hc;
    if constexpr (is_f32<T>()) {
        // per-cell values are rounded products (mul_rn): no later sum can fuse them
        const float rs = f_rsqrt(hc);
        const float r = rs * rs;
        p.u = wet ? mul_rn(hu, r) : 0.f;
        p.v = wet ? mul_rn(hv, r) : 0.f;
        p.sq = mul_rn(hc, rs);
        p.c = mul_rn(3.1320919526731650f, p.sq);  // sqrt(g) sqrt(h)
    } else {
        p.u = wet ? hu / hc : T(0);
        p.v = wet ? hv / hc : T(0);
        p.sq = d_sqrt(hc);
        p.c = d_sqrt(T(G_ACC) * hc);
    }
    const T zbc = zb > T(SED_TOL) ? zb : T(SED_TOL * 0.01);
    p.zt = z + zbc;
    p.nb = nb;
    return p;
}

// Roe-Exner fluctuations of one face (roe_exner.py:312-533).  YF selects the y-face
// orientation (normal (0,-1): normal velocity -v, tangential u); otherwise (1,0).
// Outputs upwP (to cell j) and upwM (to cell i) in (h, hu, hv).
template <class T, bool YF>
__device__ __forceinline__ void roe_exner_face(const HCell<T>& I, const HCell<T>& J, T dx, T P[3], T M[3]) {
    const T uhi = YF ? -I.v : I.u, vhi = YF ? I.u : I.v;
    const T uhj = YF ? -J.v : J.u, vhj = YF ? J.u : J.v;
    const T den = I.sq + J.sq;
    const T ht = T(0.5) * (I.h + J.h);
    T ct, ut, vt, rct = T(0);
    if constexpr (is_f32<T>()) {
        const float rden = f_rcp(den);
        const float gh = 9.81f * ht;
        rct = f_rsqrt(gh);
        ct = mul_rn(gh, rct);
        ut = sum2(uhi, I.sq, uhj, J.sq) * rden;
        vt = sum2(vhi, I.sq, vhj, J.sq) * rden;
    } else {
        ct = d_sqrt(T(G_ACC) * ht);
        ut = (uhi * I.sq + uhj * J.sq) / den;
        vt = (vhi * I.sq + vhj * J.sq) / den;
    }
    const T l1r = ut - ct;
    const T l3r = ut + ct;
    // Harten-Hyman (roe_exner.py:357-371); the VEL_TOL guard only in the lambda_3 speed
    T l1 = l1r, lE1 = T(0);
    const T ei = uhi - I.c, ej = uhj - J.c;
    const bool m1 = (ei < T(0)) && (ej > T(0));
    T l3 = l3r, lE3 = T(0);
    const T fi = uhi + I.c, fj = uhj + J.c;
    const bool m3 = (fi < T(0)) && (fj > T(0));
    // transonic faces are rare: the float build skips the block for the whole warp
    // when no lane needs it (all lanes evaluate every face, so the vote is safe)
    bool need = true;
    if constexpr (is_f32<T>()) need = __any_sync(FULL, m1 || m3);
    if (need) {
        if (m1) {
            const T t = ei * (ej - l1r) / (ej - ei);
            lE1 = l1r - t;
            l1 = t;
        }
        if (m3) {
            const T num = fj * (l3r - fi);
            lE3 = l3r - num / (fj - fi);
            l3 = num / ((fj - fi) + T(VEL_TOL));
        }
    }
    const T dh = J.h - I.h;
    const T dhu = dif2(J.h, uhj, I.h, uhi);
    const T dhv = dif2(J.h, vhj, I.h, vhi);
    const T dz = J.zt - I.zt;
    const T thrust = mul_rn(-T(G_ACC) * ht, dz);
    const T nt = T(0.5) * (I.nb + J.nb);
    T a1, a2, a3, b1;
    if constexpr (is_f32<T>()) {
        const float r2 = -0.5f * rct;  // 1 / (-2 c)
        a1 = (-l3r * dh + dhu) * r2;
        a2 = (-vt * dh + dhv) * rct;
        a3 = (l1r * dh - dhu) * r2;
        // h^(-4/3) with the DRY_TOL floor of h^(4/3) (h^(4/3) < DRY_TOL  <=>  h < DRY_TOL^(3/4))
        const float rp = ht < 1e-3f ? 1e4f : f_ex2(-1.3333333333f * f_lg2(ht));
        const float sf = nt * nt * f_sqrt(fsum2(ut, ut, vt, vt)) * ut * rp;
        const float tau = mul_rn(9.81f * ht * sf, dx);
        b1 = mul_rn(thrust - tau, r2);
    } else {
        const T den2 = T(-2.0) * ct;
        a1 = (-l3r * dh + dhu) / den2;
        a2 = (-vt * dh + dhv) / ct;
        a3 = (l1r * dh - dhu) / den2;
        const T sf = (nt * nt * d_sqrt(ut * ut + vt * vt) * ut) / clamp_lo(d_pow(ht, T(4.0 / 3.0)), T(DRY_TOL));
        const T tau = T(G_ACC) * ht * sf * dx;
        b1 = (thrust - tau) / den2;
    }
    const T b3 = -b1;
    // Upwinded waves (roe_exner.py:484-507); P columns (1,l1,vt), (0,0,ct), (1,l3,vt).
    T p0 = T(0), p1 = T(0), p2 = T(0), n0 = T(0), n1 = T(0), n2 = T(0);
    if constexpr (is_f32<T>()) {
        // Branch-free split.  With A_k = [lambda_k > 0] w_k + [lambda_E,k > 0] e_k and
        // T_k = w_k + e_k (k = 1, 3; e_k = lambda_E,k alpha_k, zero without the fix):
        //   upwP = (A1 + A3, A1 l1 + A3 l3, (A1 + A3) vt + [ut > 0] w2 ct)
        //   upwM = the same with T_k - A_k and [ut <= 0].
        // (b1, w2c, e1, e3 are rounded products, so each sum below has one product to fuse)
        // When no face of the warp needs the entropy fix (the vote above; lambda_E = 0) the
        // e_k terms are dropped for the whole warp; they add only zeros then (the sign of a
        // zero flux component may differ, which no update can see).
        const float w1 = __fmaf_rn(l1, a1, -b1), w2c = mul_rn(ut * a2, ct), w3 = __fmaf_rn(l3, a3, -b3);
        float A1, A3, B1, B3;
        if (need) {
            const float e1 = mul_rn(lE1, a1), e3 = mul_rn(lE3, a3);
            A1 = (l1 > 0.f ? w1 : 0.f) + (lE1 > 0.f ? e1 : 0.f);
            A3 = (l3 > 0.f ? w3 : 0.f) + (lE3 > 0.f ? e3 : 0.f);
            B1 = (w1 + e1) - A1;
            B3 = (w3 + e3) - A3;
        } else {
            A1 = l1 > 0.f ? w1 : 0.f;
            A3 = l3 > 0.f ? w3 : 0.f;
            B1 = w1 - A1;  // as (w1 + e1) - A1, NaN included
            B3 = w3 - A3;
        }
        const bool s2 = ut > 0.f;
        p0 = A1 + A3;
        p1 = sum2(A1, l1, A3, l3);
        p2 = __fmaf_rn(p0, vt, s2 ? w2c : 0.f);
        n0 = B1 + B3;
        n1 = sum2(B1, l1, B3, l3);
        n2 = __fmaf_rn(n0, vt, s2 ? 0.f : w2c);
    } else {
    {
        const T w = l1 * a1 - b1;
        if (l1 > T(0)) { p0 = p0 + w; p1 = p1 + w * l1; p2 = p2 + w * vt; }
        else if (l1 <= T(0)) { n0 = n0 + w; n1 = n1 + w * l1; n2 = n2 + w * vt; }
    }
    {
        const T w = ut * a2;  // beta_2 = 0
        if (ut > T(0)) p2 = p2 + w * ct;
        else if (ut <= T(0)) n2 = n2 + w * ct;
    }
    {
        const T w = l3 * a3 - b3;
        if (l3 > T(0)) { p0 = p0 + w; p1 = p1 + w * l3; p2 = p2 + w * vt; }
        else if (l3 <= T(0)) { n0 = n0 + w; n1 = n1 + w * l3; n2 = n2 + w * vt; }
    }
    // Entropy-fix waves (roe_exner.py:510-524); lambda_E2 = 0 adds nothing.
    if (m1) {
        const T e = lE1 * a1;
        if (lE1 > T(0)) { p0 = p0 + e; p1 = p1 + e * l1; p2 = p2 + e * vt; }
        else if (lE1 <= T(0)) { n0 = n0 + e; n1 = n1 + e * l1; n2 = n2 + e * vt; }
    }
    if (m3) {
        const T e = lE3 * a3;
        if (lE3 > T(0)) { p0 = p0 + e; p1 = p1 + e * l3; p2 = p2 + e * vt; }
        else if (lE3 <= T(0)) { n0 = n0 + e; n1 = n1 + e * l3; n2 = n2 + e * vt; }
    }
    }
    // back to (x, y) (roe_exner.py:526-531)
    if (YF) {
        P[0] = p0; P[1] = p2; P[2] = -p1;
        M[0] = n0; M[1] = n2; M[2] = -n1;
    } else {
        P[0] = p0; P[1] = p1; P[2] = p2;
        M[0] = n0; M[1] = n1; M[2] = n2;
    }
}

// ----------------------------------------------------------------------- bedload
// Per-cell values of the Exner face (roe_exner.py:620-646).
template <class T>
struct ECell {
    T h;   // depth as stored (activity test)
    T zb;  // z_b as stored (activity test, update base)
    T zbe; // floored z_b
    T sq;  // sqrt(floored h)
    T u, v, um;  // velocity, |u|^2
    T G;
};

template <class T>
__device__ __forceinline__ ECell<T> make_ecell(T h, T hu, T hv, T zb, T G) {
    ECell<T> e;
    const T he = h > T(DRY_TOL) ? h : T(DRY_TOL * 0.01);
    const bool wet = he > T(DRY_TOL);
    e.h = h;
    e.zb = zb;
    e.zbe = zb > T(SED_TOL) ? zb : T(SED_TOL * 0.01);
    if constexpr (is_f32<T>()) {
        const float rs = f_rsqrt(he);
        const float r = rs * rs;
        e.sq = mul_rn(he, rs);
        e.u = wet ? mul_rn(hu, r) : 0.f;
        e.v = wet ? mul_rn(hv, r) : 0.f;
    } else {
        e.sq = d_sqrt(he);
        e.u = wet ? hu / he : T(0);
        e.v = wet ? hv / he : T(0);
    }
    if constexpr (is_f32<T>()) e.um = fsum2(e.u, e.u, e.v, e.v);
    else e.um = e.u * e.u + e.v * e.v;
    e.G = G;
    return e;
}

template <class T, bool YF>
__device__ __forceinline__ T exner_face(const ECell<T>& I, const ECell<T>& J) {
    const T uhi = YF ? -I.v : I.u;
    const T uhj = YF ? -J.v : J.u;
    const T gt = T(0.5) * (I.G + J.G);
    const T dz = J.zbe - I.zbe;
    // lambda_4 = dq/dz, or the Roe-averaged normal velocity when |dz| <= SED_TOL; only
    // its sign is used.  Products are rounded separately (no FMA) so that exact
    // cancellations stay exact, as in the reference's arithmetic.
    const bool big = fabs(dz) > T(SED_TOL);
    if constexpr (is_f32<T>()) {
        // q_b + corrector = G q + (G~ - G) |u|^2 u = G~ |u|^2 u: the float build takes the
        // two products of dq as the upwind fluxes (the float64 build keeps the reference's
        // two-term form)
        const float pi = mul_rn(mul_rn(gt, I.um), uhi), pj = mul_rn(mul_rn(gt, J.um), uhj);
        const float dq = pj - pi;
        const bool up_big = (dq == 0.f) || (dq == dq && ((dq > 0.f) == (dz > 0.f)));
        const float num = mul_rn(uhi, I.sq) + mul_rn(uhj, J.sq);  // sign of ut (denominator > 0)
        const bool up = big ? up_big : (num >= 0.f);
        return up ? pi : pj;
    }
    const T qi = mul_rn(I.G * I.um, uhi);
    const T qj = mul_rn(J.G * J.um, uhj);
    const T qbi = qi + (gt - I.G) * I.um * uhi;
    const T qbj = qj + (gt - J.G) * J.um * uhj;
    bool up;
    {
        const T ut = (uhi * I.sq + uhj * J.sq) / (I.sq + J.sq);
        const T dq = gt * J.um * uhj - gt * I.um * uhi;
        const T lam4 = big ? dq / dz : ut;
        up = lam4 >= T(0);
    }
    return up ? qbi : qbj;
}

// Exner face activity (roe_exner.py:687-701): wet on either side, neither side nodata,
// and not both sediment layers below SED_TOL.
template <class T>
__device__ __forceinline__ bool exner_active(const ECell<T>& I, const ECell<T>& J, bool mi, bool mj) {
    return ((I.h > T(DRY_TOL)) || (J.h > T(DRY_TOL))) && !(mi || mj) &&
           !((I.zb < T(SED_TOL)) && (J.zb < T(SED_TOL)));
}

// ----------------------------------------------------------------- grass factor
template <class T>
struct SedT {
    T np2;    // n_p^2
    T sm1d;   // (s - 1) d50
    T thc;    // theta_c
    T np3sg;  // n_p^3 sqrt(g)
    T sm1;    // s - 1
    T frac;
};

template <class T>
struct SedTable {
    SedT<T> s[PXB_MAX_SED];
    int n;
    T one_minus_por;  // 1 - mean(porosity)
    T n_p_mix;        // (mean(d50*frac))^(1/6) / 21.1   (compute_n)
    // float path only: folded constants
    T k_theta[PXB_MAX_SED];  // n_p^2 / ((s-1) d50)
    T k_g1[PXB_MAX_SED];     // frac * n_p^3 sqrt(g) / (s-1) * 8
    T inv_one_minus_por;
};

// Meyer-Peter & Mueller grass factor of one cell (roe_exner.py:85-130).
template <class T>
__device__ __forceinline__ T mpm_grass(T h, T hu, T hv, bool nodata, const SedTable<T>& S) {
    if constexpr (is_f32<T>()) {
        // G = sum_k frac n_p^3 sqrt(g)/((s-1) sqrt h) * 8 sqrt(dth)/(th^1.5 + 1e-5) * dth
        const float hc = clamp_lo(h, float(DRY_TOL));
        float rs = f_rsqrt(hc);
        float rcb = f_ex2(-0.33333333333f * f_lg2(hc));  // h^(-1/3)
        {
            // Below the Shields threshold in every lane and class G is 0.  The unrefined
            // theta (relative error under 1e-5) decides it with a 1e-4 margin, so such warps
            // return before the refinement; the full evaluation gives the same 0 there (and
            // 0 for a NaN depth or velocity too).
            const float r0 = rs * rs;
            const float u0 = hu * r0, v0 = hv * r0;
            const float q0 = fsum2(u0, u0, v0, v0) * rcb;
            bool above = false;
#pragma unroll 1
            for (int k = 0; k < S.n; ++k) above = above || (S.k_theta[k] * q0 > 0.9999f * S.s[k].thc);
            if (!__any_sync(FULL, above)) return 0.f;
        }
        // one Newton step each: the threshold (theta - theta_c)^1.5 amplifies errors in theta
        rs = rs * (1.5f - 0.5f * hc * rs * rs);
        const float r = rs * rs;
        const float u = hu * r, v = hv * r;
        const float vel2 = fsum2(u, u, v, v);
        rcb = rcb * (4.f - hc * rcb * rcb * rcb) * (1.f / 3.f);
        float G = 0.f;
#pragma unroll 1
        for (int k = 0; k < S.n; ++k) {
            {
                const float th = fmaxf(S.k_theta[k] * vel2 * rcb, 0.f);
                const float dth = th - S.s[k].thc;
                // below the Shields threshold G is 0: skip the block when no lane is above it
                if (__any_sync(FULL, dth > 0.f)) {
                    const float pos = dth > 0.f ? dth : 0.f;
                    const float th15 = th * f_sqrt(th);
                    G += S.k_g1[k] * rs * f_sqrt(pos) * pos * f_rcp(th15 + 1e-5f);
                }
            }
        }
        G *= S.inv_one_minus_por;
        if (nodata) G = 0.f;
        return hc > float(DRY_TOL) ? G : 0.f;
    }
    const T hc = clamp_lo(h, T(DRY_TOL));
    const T u = hu / hc, v = hv / hc;
    const T vel2 = u * u + v * v;
    const T cb = d_cbrt(hc);
    const T sqh = d_sqrt(hc);
    T G = T(0);
    for (int k = 0; k < S.n; ++k) {
        const SedT<T>& s = S.s[k];
        T theta = (s.np2 * vel2) / (s.sm1d * cb);
        theta = clamp_lo(theta, T(0));
        const T dth = clamp_lo(theta - s.thc, T(0));
        const T g1 = s.np3sg / (s.sm1 * sqh);
        const T g2 = T(8.0) * d_sqrt(dth) / (d_pow(theta, T(1.5)) + T(1e-5));
        const T contrib = s.frac * g1 * g2 * dth;
        G = (k == 0) ? contrib : G + contrib;
    }
    G = G / S.one_minus_por;
    if (nodata) G = T(0);
    return hc > T(DRY_TOL) ? G : T(0);
}

// Constant grass factor pass-through (roe_exner.py:136-140).
template <class T>
__device__ __forceinline__ T const_grass(T h, T G, bool nodata) {
    if (nodata) G = T(0);
    return h > T(DRY_TOL) ? G : T(0);
}

// ------------------------------------------------------------------ wave speeds
template <class T>
struct CCell {
    T h;  // max(h, DRY_TOL)
    T sq, u, v, G;
    T rs;  // 1/sqrt(h) (float path)
};

template <class T>
__device__ __forceinline__ CCell<T> make_ccell(T h, T hu, T hv, T G) {
    CCell<T> p;
    p.h = clamp_lo(h, T(DRY_TOL));
    if constexpr (is_f32<T>()) {
        p.rs = f_rsqrt(p.h);
        const float r = p.rs * p.rs;
        p.sq = mul_rn(p.h, p.rs);
        p.u = mul_rn(hu, r);
        p.v = mul_rn(hv, r);
    } else {
        p.rs = T(0);
        p.sq = d_sqrt(p.h);
        p.u = hu / p.h;
        p.v = hv / p.h;
    }
    p.G = G;
    return p;
}

// Extreme roots of the coupled cubic (roe_exner.py:163-209), trigonometric Cardano,
// with the linear speeds when a < 1e-5.
template <class T>
__device__ __forceinline__ void cubic_extremes(T ut, T at, T ct, T& lmin, T& lmax) {
    if (at < T(1e-5)) {
        lmin = ut - ct;
        lmax = ut + ct;
        return;
    }
    if constexpr (is_f32<T>()) {
        // float Cardano; where |cos(theta)| is within 1e-3 of 1 (two roots close
        // together) the trigonometric form loses digits, so those faces redo the
        // solve in float64.
        const float b = -2.f * ut;
        const float c = dif2(1.f + at, ct * ct, ut, ut);
        const float d = -(ct * ct) * at * ut;
        const float p = dif2(-3.f, c, b, b) * (1.f / 3.f);
        const float q = (mul_rn(2.f * b * b, b) + mul_rn(9.f * b, c) + mul_rn(27.f, d)) * (-1.f / 27.f);
        // (3q / 2p) sqrt(-3/p); p < 0 for three real roots, otherwise this is NaN and the
        // float64 solve below takes over
        const float rp = f_rcp(p);
        const float xr = 1.5f * q * rp * f_sqrt(-3.f * rp);
        if (fabsf(xr) > 0.999f || xr != xr) {
            double dl, du;
            cubic_extremes<double>(double(ut), double(at), double(ct), dl, du);
            lmin = float(dl);
            lmax = float(du);
            return;
        }
        const float th = acosf(xr);
        const float sq = 2.f * f_sqrt(-p * (1.f / 3.f));
        const float shift = mul_rn(b, 1.f / 3.f);
        // th / 3 is in [0, pi/3]: the hardware sine / cosine are within 2^-21 absolute there
        float sn, cs;
        __sincosf(th * (1.f / 3.f), &sn, &cs);
        lmax = __fmaf_rn(sq, cs, shift);
        // cos((th + 2 pi)/3) = -cos(th/3)/2 - sqrt(3)/2 sin(th/3)
        lmin = __fmaf_rn(sq, __fmaf_rn(-0.5f, cs, -mul_rn(0.86602540378f, sn)), shift);
        return;
    }
    const T b = T(-2) * ut;
    const T c = (T(1) + at) * (ct * ct) - ut * ut;
    const T d = -(ct * ct) * at * ut;
    const T p = (T(-3) * c - b * b) / T(3);
    const T q = (T(2) * (b * (b * b)) - T(-9) * b * c + T(27) * d) / T(-27);
    const T x = clip1((T(3) * q) / (T(2) * p) * d_sqrt(T(-3) / p));
    const T th = d_acos(x);
    const T sq = T(2) * d_sqrt(-p / T(3));
    const T shift = -b / T(-3);
    lmax = sq * d_cos(th / T(3)) + shift;
    lmin = sq * d_cos((th + T(TWO_PI)) / T(3)) + shift;
}

// Largest characteristic speed of one face (roe_exner.py:211-255); the face step is
// dx / speed, so the global minimum step is dx / (maximum speed).
template <class T, bool YF>
__device__ __forceinline__ T face_speed(const CCell<T>& I, const CCell<T>& J) {
    const T uhi = YF ? -I.v : I.u, vhi = YF ? I.u : I.v;
    const T uhj = YF ? -J.v : J.u, vhj = YF ? J.u : J.v;
    const T den = I.sq + J.sq;
    const T ht = T(0.5) * (I.h + J.h);
    const T gt = T(0.5) * (I.G + J.G);
    T ut, ct, at;
    if constexpr (is_f32<T>()) {
        ut = mul_rn(sum2(uhi, I.sq, uhj, J.sq), f_rcp(den));  // rounded: u~ -+ c~ as in face_speed_nog
        ct = f_sqrt(9.81f * ht);
        const float s4 = __fmaf_rn(vhi, vhj, __fmaf_rn(uhj, uhj, fsum2(uhi, uhi, uhi, uhj)));
        at = gt * s4 * (I.rs * J.rs);
    } else {
        ut = (uhi * I.sq + uhj * J.sq) / den;
        ct = d_sqrt(T(G_ACC) * ht);
        at = gt * (uhi * uhi + uhi * uhj + uhj * uhj + vhi * vhj) / (I.sq * J.sq);
    }
    const T l1 = ut - ct, l3 = ut + ct;
    T lmin, lmax;
    cubic_extremes(ut, at, ct, lmin, lmax);
    const T roe = nan_max(fabs(lmin), fabs(lmax));
    const T swe = nan_max(fabs(l1), fabs(l3));
    return roe < T(VEL_TOL) ? swe : roe;
}

// face_speed of a face whose two cells carry no G (G = 0, so a~ = 0 and the cubic's
// extreme roots are u~ -+ c~): the same value, without a~ and the cubic branch.
template <class T, bool YF>
__device__ __forceinline__ T face_speed_nog(const CCell<T>& I, const CCell<T>& J) {
    const T uhi = YF ? -I.v : I.u;
    const T uhj = YF ? -J.v : J.u;
    const T den = I.sq + J.sq;
    const T ht = T(0.5) * (I.h + J.h);
    T ut, ct;
    if constexpr (is_f32<T>()) {
        ut = mul_rn(sum2(uhi, I.sq, uhj, J.sq), f_rcp(den));
        ct = f_sqrt(9.81f * ht);
    } else {
        ut = (uhi * I.sq + uhj * J.sq) / den;
        ct = d_sqrt(T(G_ACC) * ht);
    }
    return nan_max(fabs(ut - ct), fabs(ut + ct));
}

// Order-preserving map of a non-negative (or NaN) float to unsigned bits for atomicMax.
__device__ __forceinline__ unsigned long long speed_bits(double s) { return (unsigned long long)__double_as_longlong(s); }
__device__ __forceinline__ unsigned long long speed_bits(float s) { return (unsigned long long)(unsigned)__float_as_uint(s); }
__device__ __forceinline__ double bits_speed(unsigned long long b, double) { return __longlong_as_double((long long)b); }
__device__ __forceinline__ float bits_speed(unsigned long long b, float) { return __uint_as_float((unsigned)b); }

// ----------------------------------------------------------------- ring recipes
__device__ __forceinline__ int ring_slot(int r, int c, int ny, int nx) {
    if (r == 0) return c;
    if (r == ny - 1) return nx + c;
    if (c == 0) return 2 * nx + r;
    if (c == nx - 1) return 2 * nx + ny + r;
    return -1;
}

}  // namespace pxb
