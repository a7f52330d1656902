// Set-up kernels: the pointwise part of init_fn_roeexner (n_b and G,
// PyExner src/PyExner/solvers/roe_exner_solver.py:58-78) and the exact, handler-by-handler
// boundary application of BoundaryManager.apply (src/PyExner/domain/boundary_registry.py:183-187).
//
// The generic application runs each handler as a gather of all donor values into a
// scratch buffer followed by a scatter into the boundary cells, which is the jax
// semantics of `state.h.at[by, bx].set(state.h[iy, ix])` (reads before writes within a
// handler, later handlers overwrite earlier ones).  It is used once, at set-up; the
// stage kernels use the ring recipes resolved from the same handlers.
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

// Field slots of the generic handler kernels.
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
    T c0, c1;
    T* tmp;  // 6 * count values
};

template <class T>
__global__ void bc_gather_kernel(const BcArgs<T> a) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= a.count) return;
    const long long d = a.donors[k];
    T* t = a.tmp;
    const int n = a.count;
    switch (a.kind) {
        case PXB_BC_RE_REFLECTIVE: {  // roeexner_reflective.py:17-63
            const T hu = a.f[1][d], hv = a.f[2][d];
            const T mom_n = hu * a.nx + hv * a.ny;
            const T mom_t = -hu * a.ny + hv * a.nx;
            const T mom_r = -mom_n;
            t[0 * n + k] = a.f[0][d];
            t[1 * n + k] = mom_r * a.nx - mom_t * a.ny;
            t[2 * n + k] = mom_r * a.ny + mom_t * a.nx;
            t[3 * n + k] = a.f[3][d];
            t[4 * n + k] = a.f[4][d];
            t[5 * n + k] = a.f[5][d];
            break;
        }
        case PXB_BC_RE_TRANSMISSIVE:  // roeexner_transmissive.py:17-31
            t[0 * n + k] = a.f[0][d];
            t[1 * n + k] = a.f[1][d];
            t[2 * n + k] = a.f[2][d];
            break;
        case PXB_BC_RE_TRANSMISSIVEBED:  // roeexner_transmissivebed.py:17-27
            t[3 * n + k] = a.f[3][d];
            break;
        case PXB_BC_RE_CONSTANTINFLUX:  // roeexner_constantinflux.py:18-48
            t[1 * n + k] = a.c0;
            t[2 * n + k] = a.c1;
            break;
        case PXB_BC_ROE_REFLECTIVE:  // roe_reflective.py:18-44
            t[0 * n + k] = a.f[0][d];
            t[3 * n + k] = a.f[3][d];
            t[4 * n + k] = a.f[4][d];
            t[1 * n + k] = a.f[1][d] * (T(1) - T(2) * a.nx * a.nx);
            t[2 * n + k] = a.f[2][d] * (T(1) - T(2) * a.ny * a.ny);
            break;
        case PXB_BC_ROE_TRANSMISSIVE:  // roe_transmissive.py:17-43
            t[0 * n + k] = a.f[0][d];
            t[1 * n + k] = a.f[1][d];
            t[2 * n + k] = a.f[2][d];
            t[3 * n + k] = a.f[3][d];
            t[4 * n + k] = a.f[4][d];
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
        if ((fm >> s) & 1u) a.f[s][b] = a.tmp[s * a.count + k];
}

}  // namespace pxb
