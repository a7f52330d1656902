// Set-up kernels: the pointwise part of init_fn_roeexner (n_b and G,
// PyExner src/PyExner/solvers/roe_exner_solver.py:58-78) and the exact, handler-by-handler
// boundary application of BoundaryManager.apply (src/PyExner/domain/boundary_registry.py:183-187).
//
// The generic application runs each handler as a gather of all donor values into a
// scratch buffer followed by a scatter into the boundary cells, which is the jax
// semantics of `state.h.at[by, bx].set(state.h[iy, ix])` (reads before writes within a
// handler, later handlers overwrite earlier ones).  It serves the set-up and the general
// stage path; the fused stage kernel uses the ring recipes resolved from the same handlers.
#pragma once
#include "pxb_device.cuh"

namespace pxb {

template <class T>
struct InitArgs {
    int ny, nx;
    long long pitch;
    const T *h, *hu, *hv, *zb, *n;
    T *nb, *G;
    const uint8_t* nodata;
    int mpm;
    SedTable<T> sed;
};

template <class T>
__global__ void __launch_bounds__(256) re_init_kernel(const InitArgs<T> a) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const int r = blockIdx.y * blockDim.y + threadIdx.y;
    if (r >= a.ny || c >= a.nx) return;
    const long long i = (long long)r * a.pitch + c;
    const bool m0 = a.nodata ? (a.nodata[i] != 0) : false;
    if (a.mpm) {
        // compute_n (roe_exner.py:64-73)
        a.nb[i] = a.zb[i] > T(SED_TOL) ? a.sed.n_p_mix : a.n[i];
        a.G[i] = mpm_grass(a.h[i], a.hu[i], a.hv[i], m0, a.sed);
    } else {
        a.nb[i] = a.n[i];
        a.G[i] = const_grass(a.h[i], a.G[i], m0);
    }
}

// Field slots of the generic handler kernels (a null slot is skipped).
//   Roe-Exner: 0 h, 1 hu, 2 hv, 3 z_b, 4 n, 5 G
//   Roe:       0 h, 1 hu, 2 hv, 3 z,   4 n, 5 (unused)
template <class T>
struct BcArgs {
    T* f[6];
    const long long* cells;
    const long long* donors;
    int count;
    int kind;
    T nx, ny;
    T c0, c1;             // constant momenta (ConstantInflux, ConstantOutflux, ZeroMomentum; NaN = keep)
    T q, vx, vy;          // ConstantOutflux: discharge and direction (float32 values)
    float neg_alpha, zb0;  // Berthon / NormalFlowDepth: z_b = fl32(fl32(neg_alpha * fl32(t)) + zb0)
    T hb;                 // NormalFlowDepth: depth q/u
    const double* tptr;   // simulation time on the device, or null: use tval
    double tval;
    T* tmp;  // 6 * count values
};

// Depth of a ConstantOutflux cell: five Newton steps on the outgoing Riemann invariant
// of the donor, q/h + 2 sqrt(g h) = un + 2 sqrt(g h_i) (roeexner_constantoutflux.py:29-58).
template <class T>
__device__ __forceinline__ T outflux_depth(T h, T hu, T hv, T q, T vx, T vy) {
    const T G = T(9.81), TINY = T(1e-8);
    const T h_i = nan_max(h, TINY);
    const T u_i = hu / h_i, v_i = hv / h_i;
    const T un_i = u_i * vx + v_i * vy;
    const T rp = un_i + T(2) * d_sqrt(G * h_i);
    T hb = h_i;
    for (int it = 0; it < 5; ++it) {
        hb = nan_max(hb, TINY);
        const T c = d_sqrt(G * hb);
        const T f = q / hb + T(2) * c - rp;
        const T df = -q / (hb * hb) + G / nan_max(c, TINY);
        hb = nan_max(hb - f / df, TINY);
    }
    return hb;
}

// z_b of the Berthon analytic solution at time t, in float32 like the reference's
// float32 values (roeexner_berthon.py:49-52): -alpha * t + zb0.
__device__ __forceinline__ float berthon_zb(float neg_alpha, float zb0, double t) {
    return __fadd_rn(__fmul_rn(neg_alpha, __double2float_rn(t)), zb0);
}

template <class T>
__global__ void bc_gather_kernel(const BcArgs<T> a) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= a.count) return;
    const long long d = a.donors[k];
    auto ld = [&](int slot) { return a.f[slot] ? a.f[slot][d] : T(0); };  // null slots read as 0
    T* t = a.tmp;
    const int n = a.count;
    switch (a.kind) {
        case PXB_BC_RE_REFLECTIVE: {  // roeexner_reflective.py:17-63
            const T hu = ld(1), hv = ld(2);
            const T mom_n = hu * a.nx + hv * a.ny;
            const T mom_t = -hu * a.ny + hv * a.nx;
            const T mom_r = -mom_n;
            t[0 * n + k] = ld(0);
            t[1 * n + k] = mom_r * a.nx - mom_t * a.ny;
            t[2 * n + k] = mom_r * a.ny + mom_t * a.nx;
            t[3 * n + k] = ld(3);
            t[4 * n + k] = ld(4);
            t[5 * n + k] = ld(5);
            break;
        }
        case PXB_BC_RE_TRANSMISSIVE:  // roeexner_transmissive.py:17-31
            t[0 * n + k] = ld(0);
            t[1 * n + k] = ld(1);
            t[2 * n + k] = ld(2);
            break;
        case PXB_BC_RE_TRANSMISSIVEBED:  // roeexner_transmissivebed.py:17-27
            t[3 * n + k] = ld(3);
            break;
        case PXB_BC_RE_CONSTANTINFLUX:  // roeexner_constantinflux.py:18-48
            t[1 * n + k] = a.c0;
            t[2 * n + k] = a.c1;
            break;
        case PXB_BC_ROE_REFLECTIVE:  // roe_reflective.py:18-44
            t[0 * n + k] = ld(0);
            t[3 * n + k] = ld(3);
            t[4 * n + k] = ld(4);
            t[1 * n + k] = ld(1) * (T(1) - T(2) * a.nx * a.nx);
            t[2 * n + k] = ld(2) * (T(1) - T(2) * a.ny * a.ny);
            break;
        case PXB_BC_ROE_TRANSMISSIVE:  // roe_transmissive.py:17-43
            t[0 * n + k] = ld(0);
            t[1 * n + k] = ld(1);
            t[2 * n + k] = ld(2);
            t[3 * n + k] = ld(3);
            t[4 * n + k] = ld(4);
            break;
        case PXB_BC_RE_CONSTANTOUTFLUX:  // roeexner_constantoutflux.py:18-73
            t[0 * n + k] = outflux_depth(ld(0), ld(1), ld(2), a.q, a.vx, a.vy);
            t[1 * n + k] = a.c0;
            t[2 * n + k] = a.c1;
            break;
        case PXB_BC_RE_BERTHON:  // roeexner_berthon.py:19-56
            t[3 * n + k] = T(berthon_zb(a.neg_alpha, a.zb0, a.tptr ? *a.tptr : a.tval));
            break;
        case PXB_BC_RE_NORMALFLOWDEPTH:  // roeexner_normalflowdepth.py:19-51
            t[0 * n + k] = a.hb;
            t[1 * n + k] = ld(1);
            t[2 * n + k] = ld(2);
            t[3 * n + k] = T(berthon_zb(a.neg_alpha, a.zb0, a.tptr ? *a.tptr : a.tval));
            break;
        case PXB_BC_RE_STEEPFALL:  // roeexner_steepfall.py:17-26
            t[3 * n + k] = ld(3) - T(1);
            break;
        case PXB_BC_RE_ZEROMOMENTUM:  // roeexner_zeromomentum.py:16-31; the donor is the cell
            t[1 * n + k] = (a.c0 != a.c0) ? ld(1) : a.c0;
            t[2 * n + k] = (a.c1 != a.c1) ? ld(2) : a.c1;
            break;
        default:
            break;
    }
}

__host__ __device__ inline unsigned bc_field_mask(int kind) {
    switch (kind) {
        case PXB_BC_RE_REFLECTIVE: return 0x3f;
        case PXB_BC_RE_TRANSMISSIVE: return 0x07;
        case PXB_BC_RE_TRANSMISSIVEBED: return 0x08;
        case PXB_BC_RE_CONSTANTINFLUX: return 0x06;
        case PXB_BC_ROE_REFLECTIVE: return 0x1f;
        case PXB_BC_ROE_TRANSMISSIVE: return 0x1f;
        case PXB_BC_RE_CONSTANTOUTFLUX: return 0x07;
        case PXB_BC_RE_BERTHON: return 0x08;
        case PXB_BC_RE_NORMALFLOWDEPTH: return 0x0f;
        case PXB_BC_RE_STEEPFALL: return 0x08;
        case PXB_BC_RE_ZEROMOMENTUM: return 0x06;
        default: return 0;
    }
}

template <class T>
__global__ void bc_scatter_kernel(const BcArgs<T> a) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= a.count) return;
    const long long b = a.cells[k];
    const unsigned fm = bc_field_mask(a.kind);
    for (int s = 0; s < 6; ++s)
        if (((fm >> s) & 1u) && a.f[s]) a.f[s][b] = a.tmp[s * a.count + k];
}

}  // namespace pxb
