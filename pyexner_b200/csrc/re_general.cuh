// General Roe-Exner stage path: the stage of step_fn_roeexner
// (PyExner src/PyExner/solvers/roe_exner_solver.py:80-116) as a chain of cell-parallel
// kernels over plan-owned scratch planes, for the boundary layouts that the fused stage
// kernel does not cover: boundary cells inside the array (L- and T-shaped domains, inner
// walls), handlers whose value is a formula of the time or of donor values
// (ConstantOutflux, Berthon, NormalFlowDepth, SteepFall, ZeroMomentum), and handler
// chains whose repeated application does not settle after one pass.
//
//   gen_hydro     hydro faces (roe_exner.py:535-612) -> S.h, S.hu, S.hv; S.z_b, S.G, S.n
//                 copied from the input
//   gen_corr      momentum corrections on the interior (roe_exner.py:14-62), in place
//   handlers      every handler in order, gather then scatter (boundary_registry.py:183-187)
//   gen_grass     G (roe_exner.py:85-140)
//   gen_exner     Exner faces and the z_b update (roe_exner.py:665-717) -> S.z_b2
//   handlers      second application on (S.h, S.hu, S.hv, S.z_b2, S.n, S.G)
//   gen_store     output planes, with the SSPRK2 average (SSPRK2.py:40) when asked
//
// Every face and cell formula is the device function the fused kernel uses, applied to
// the same operands in the same order, so in float64 both paths give the same bits.
// Each face is evaluated by both of its cells (twice the face work of the fused kernel);
// the path trades speed for generality.
#pragma once
#include "pxb_device.cuh"

namespace pxb {

template <class T>
struct GenArgs {
    int ny, nx;
    long long pitch;
    T dx;
    const T *h, *hu, *hv, *zb, *z, *nb, *G, *n;  // stage input (G, n may be null)
    T *sh, *shu, *shv, *szb, *sG, *sn, *szb2;     // scratch state
    const uint8_t* nodata;                         // mask[0] or null
    const T* dt;
    SedTable<T> sed;
    int mpm;
    // gen_store
    T *oh, *ohu, *ohv, *ozb, *oG, *on;            // output (oG, on may be null)
    const T *ah, *ahu, *ahv, *azb, *aG, *an;      // SSPRK2 partner or null
    int* err;
};

template <class T>
__device__ __forceinline__ bool gen_cell(const GenArgs<T>& a, int& r, int& c, long long& i) {
    c = blockIdx.x * blockDim.x + threadIdx.x;
    r = blockIdx.y * blockDim.y + threadIdx.y;
    if (r >= a.ny || c >= a.nx) return false;
    i = (long long)r * a.pitch + c;
    return true;
}

template <class T>
__device__ __forceinline__ bool gen_nodata(const GenArgs<T>& a, long long i) {
    return a.nodata ? (a.nodata[i] != 0) : false;
}

template <class T>
__device__ __forceinline__ HCell<T> gen_hcell(const GenArgs<T>& a, long long i) {
    return make_hcell(a.h[i], a.hu[i], a.hv[i], a.zb[i], a.z[i], a.nb[i]);
}

// Hydro update of one cell from its four faces, accumulated in the scatter order of
// roe_exner.py:597-602: east face upwM, west face upwP, south face upwM, north face upwP.
template <class T>
__global__ void __launch_bounds__(256) gen_hydro_kernel(const GenArgs<T> a) {
    int r, c;
    long long i;
    if (!gen_cell(a, r, c, i)) return;
    const T DRY = T(DRY_TOL);
    const T dt = *a.dt, dx = a.dx;
    const T dtdx = dt / dx;  // float path only
    const HCell<T> C = gen_hcell(a, i);
    const T hC = a.h[i];
    const bool mC = gen_nodata(a, i);
    T P[3], M[3];
    T f0 = 0, f1 = 0, f2 = 0;
    if (c + 1 < a.nx) {
        const long long j = i + 1;
        if (((hC > DRY) || (a.h[j] > DRY)) && !(mC || gen_nodata(a, j))) {
            roe_exner_face<T, false>(C, gen_hcell(a, j), dx, P, M);
            f0 = f0 + M[0]; f1 = f1 + M[1]; f2 = f2 + M[2];
        }
    }
    if (c >= 1) {
        const long long j = i - 1;
        if (((a.h[j] > DRY) || (hC > DRY)) && !(gen_nodata(a, j) || mC)) {
            roe_exner_face<T, false>(gen_hcell(a, j), C, dx, P, M);
            f0 = f0 + P[0]; f1 = f1 + P[1]; f2 = f2 + P[2];
        }
    }
    if (r + 1 < a.ny) {
        const long long j = i + a.pitch;
        if (((hC > DRY) || (a.h[j] > DRY)) && !(mC || gen_nodata(a, j))) {
            roe_exner_face<T, true>(C, gen_hcell(a, j), dx, P, M);
            f0 = f0 + M[0]; f1 = f1 + M[1]; f2 = f2 + M[2];
        }
    }
    if (r >= 1) {
        const long long j = i - a.pitch;
        if (((a.h[j] > DRY) || (hC > DRY)) && !(gen_nodata(a, j) || mC)) {
            roe_exner_face<T, true>(gen_hcell(a, j), C, dx, P, M);
            f0 = f0 + P[0]; f1 = f1 + P[1]; f2 = f2 + P[2];
        }
    }
    if constexpr (is_f32<T>()) {
        a.sh[i] = hC - dtdx * f0;
        a.shu[i] = a.hu[i] - dtdx * f1;
        a.shv[i] = a.hv[i] - dtdx * f2;
    } else {
        a.sh[i] = hC - dt * f0 / dx;
        a.shu[i] = a.hu[i] - dt * f1 / dx;
        a.shv[i] = a.hv[i] - dt * f2 / dx;
    }
    a.szb[i] = a.zb[i];
    a.sG[i] = a.G ? a.G[i] : T(0);
    a.sn[i] = a.n ? a.n[i] : T(0);
}

// Momentum corrections (roe_exner.py:14-62) on rows and columns 1 .. n-2.  They read
// the updated depths of the neighbours and write only the own momenta: in place.
template <class T>
__global__ void __launch_bounds__(256) gen_corr_kernel(const GenArgs<T> a) {
    int r, c;
    long long i;
    if (!gen_cell(a, r, c, i)) return;
    if (r < 1 || r > a.ny - 2 || c < 1 || c > a.nx - 2) return;
    const T DRY = T(DRY_TOL);
    const long long E = i + 1, W = i - 1, N = i - a.pitch, S = i + a.pitch;
    const T eta = a.sh[i] + (a.z[i] + a.zb[i]);
    const bool stop_u = ((eta < a.z[E] + a.zb[E]) && (a.sh[E] < DRY)) ||
                        ((eta < a.z[W] + a.zb[W]) && (a.sh[W] < DRY)) || gen_nodata(a, E) || gen_nodata(a, W);
    const bool stop_v = ((eta < a.z[N] + a.zb[N]) && (a.sh[N] < DRY)) ||
                        ((eta < a.z[S] + a.zb[S]) && (a.sh[S] < DRY)) || gen_nodata(a, N) || gen_nodata(a, S);
    const bool active = (a.sh[i] > DRY) && !gen_nodata(a, i);
    if (!(active && !stop_u)) a.shu[i] = T(0);
    if (!(active && !stop_v)) a.shv[i] = T(0);
}

// Grass factor after the first boundary application (roe_exner_solver.py:106).
template <class T>
__global__ void __launch_bounds__(256) gen_grass_kernel(const GenArgs<T> a) {
    int r, c;
    long long i;
    if (!gen_cell(a, r, c, i)) return;
    const bool m = gen_nodata(a, i);
    a.sG[i] = a.mpm ? mpm_grass(a.sh[i], a.shu[i], a.shv[i], m, a.sed) : const_grass(a.sh[i], a.sG[i], m);
}

template <class T>
__device__ __forceinline__ ECell<T> gen_ecell(const GenArgs<T>& a, long long i) {
    return make_ecell(a.sh[i], a.shu[i], a.shv[i], a.szb[i], a.sG[i]);
}

// z_b update (roe_exner.py:708-715): -F west, +F east, then -F north, +F south.
template <class T>
__global__ void __launch_bounds__(256) gen_exner_kernel(const GenArgs<T> a) {
    int r, c;
    long long i;
    if (!gen_cell(a, r, c, i)) return;
    const T dt = *a.dt, dx = a.dx;
    const T dtdx = dt / dx;  // float path only
    const ECell<T> C = gen_ecell(a, i);
    const bool mC = gen_nodata(a, i);
    T xe = 0;
    if (c >= 1) {
        const long long j = i - 1;
        const ECell<T> w = gen_ecell(a, j);
        if (exner_active(w, C, gen_nodata(a, j), mC)) xe = xe + (-exner_face<T, false>(w, C));
    }
    if (c + 1 < a.nx) {
        const long long j = i + 1;
        const ECell<T> e = gen_ecell(a, j);
        if (exner_active(C, e, mC, gen_nodata(a, j))) xe = xe + exner_face<T, false>(C, e);
    }
    T fn = 0, fs = 0;
    if (r >= 1) {
        const long long j = i - a.pitch;
        const ECell<T> nn = gen_ecell(a, j);
        if (exner_active(nn, C, gen_nodata(a, j), mC)) fn = exner_face<T, true>(nn, C);
    }
    if (r + 1 < a.ny) {
        const long long j = i + a.pitch;
        const ECell<T> ss = gen_ecell(a, j);
        if (exner_active(C, ss, mC, gen_nodata(a, j))) fs = exner_face<T, true>(C, ss);
    }
    T acc = xe;
    acc = acc + (-fn);
    acc = acc + fs;
    if constexpr (is_f32<T>()) a.szb2[i] = C.zb - dtdx * acc;
    else a.szb2[i] = C.zb - dt * acc / dx;
}

// Output planes; the SSPRK2 average is pointwise, so `out` may alias `avg`.
template <class T>
__global__ void __launch_bounds__(256) gen_store_kernel(const GenArgs<T> a) {
    int r, c;
    long long i;
    if (!gen_cell(a, r, c, i)) return;
    T oh = a.sh[i], ou = a.shu[i], ov = a.shv[i], oz = a.szb2[i], og = a.sG[i], on = a.sn[i];
    if (a.ah) {
        oh = T(0.5) * a.ah[i] + T(0.5) * oh;
        ou = T(0.5) * a.ahu[i] + T(0.5) * ou;
        ov = T(0.5) * a.ahv[i] + T(0.5) * ov;
        oz = T(0.5) * a.azb[i] + T(0.5) * oz;
        if (a.aG) og = T(0.5) * a.aG[i] + T(0.5) * og;
        if (a.an) on = T(0.5) * a.an[i] + T(0.5) * on;
    }
    a.oh[i] = oh;
    a.ohu[i] = ou;
    a.ohv[i] = ov;
    a.ozb[i] = oz;
    if (a.oG) a.oG[i] = og;
    if (a.on) a.on[i] = on;
    if (!(d_isfinite(oh) && d_isfinite(ou) && d_isfinite(ov) && d_isfinite(oz))) atomicOr(a.err, 1);
}

}  // namespace pxb
