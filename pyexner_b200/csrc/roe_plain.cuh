// Plain Roe shallow-water step (no Exner): PyExner src/PyExner/solvers/kernels/roe.py
// and src/PyExner/solvers/roe_solver.py.
//
// Four threads per cell, one face each (every face is evaluated by both of its cells).
// Ring cells with boundary recipes recompute the update of their donor cell instead of
// reading it, so the stage is one launch with no global synchronisation.  The plain Roe
// configuration is small (258 x 258) and latency-bound; the Roe-Exner stage is the one
// built for bandwidth.
#pragma once
#include "pxb_device.cuh"

namespace pxb {

template <class T>
struct RoeArgs {
    int ny, nx;
    long long pitch;
    T dx;
    const T *h, *hu, *hv, *z, *n;
    T *oh, *ohu, *ohv, *oz, *on;
    const T *ah, *ahu, *ahv, *az, *an;
    const T* dt;
    const pxb_ring_recipe* ring;
    int* err;
};

// Roe fluctuations with the wet/dry thrust and beta limiter (roe.py:32-249).  YF (the
// y-face orientation) is a runtime flag, so that the four threads of a cell, two on
// x-faces and two on y-faces, run one code path.
template <class T>
__device__ __forceinline__ void roe_plain_face(T hi, T hui, T hvi, T zi, T ni, T hj, T huj, T hvj, T zj, T nj, T dx,
                                               const bool YF, T P[3], T M[3]) {
    const T DRY = T(DRY_TOL);
    hi = hi > DRY ? hi : T(0);
    hj = hj > DRY ? hj : T(0);
    const T sqi = d_sqrt(hi), sqj = d_sqrt(hj);
    const T ui = hi > T(0) ? hui / hi : T(0);
    const T vi = hi > T(0) ? hvi / hi : T(0);
    const T uj = hj > T(0) ? huj / hj : T(0);
    const T vj = hj > T(0) ? hvj / hj : T(0);
    const T uhi = YF ? -vi : ui, vhi = YF ? ui : vi;
    const T uhj = YF ? -vj : uj, vhj = YF ? uj : vj;
    const T hsum = T(0.5) * (hi + hj);
    const T ht = hsum > DRY ? hsum : T(0);
    const T ct = d_sqrt(T(G_ACC) * ht);
    const T ut = (uhi * sqi + uhj * sqj) / (sqi + sqj);
    const T vt = (vhi * sqi + vhj * sqj) / (sqi + sqj);
    T l1 = ut - ct;
    const T l2 = ut;
    T l3 = ut + ct;
    // Harten-Hyman: the fixed speed replaces lambda, then the entropy speed uses it (roe.py:77-92)
    T lE1 = T(0), lE3 = T(0);
    {
        const T ei = uhi - d_sqrt(T(G_ACC) * hi), ej = uhj - d_sqrt(T(G_ACC) * hj);
        const bool m = (ei < T(0)) && (ej > T(0));
        if (m) {
            l1 = ei * (ej - l1) / ((ej - ei) + T(VEL_TOL));
            lE1 = l1 - ei * (ej - l1) / ((ej - ei) + T(VEL_TOL));
        }
    }
    {
        const T ei = uhi + d_sqrt(T(G_ACC) * hi), ej = uhj + d_sqrt(T(G_ACC) * hj);
        const bool m = (ei < T(0)) && (ej > T(0));
        if (m) {
            l3 = ej * (l3 - ei) / ((ej - ei) + T(VEL_TOL));
            lE3 = l3 - ej * (l3 - ei) / ((ej - ei) + T(VEL_TOL));
        }
    }
    const T den = l1 - l3 + T(VEL_TOL);
    const T p00 = -l3 / den, p01 = T(1) / den;
    const T p10 = -vt / ct, p12 = T(1) / ct;
    const T p20 = l1 / den, p21 = T(-1) / den;
    const T dh = hj - hi;
    const T dhu = hj * uhj - hi * uhi;
    const T dhv = hj * vhj - hi * vhi;
    // P^-1 dU accumulated over the inner index in order (roe.py:127)
    const T a1 = p00 * dh + p01 * dhu + T(0) * dhv;
    const T a2 = p10 * dh + T(0) * dhu + p12 * dhv;
    const T a3 = p20 * dh + p21 * dhu + T(0) * dhv;
    const T dz = zj - zi;
    const T di = hi + zi, dj = hj + zj;
    const T dd = dj - di;
    const T thrust_a = -T(G_ACC) * ht * dz;
    const bool k1 = (dz >= T(0)) && (di < zj);
    const bool k2 = (dz < T(0)) && (dj < zi);
    const T dzt = k1 ? hi : (k2 ? hj : dz);
    const T hr = dz >= T(0) ? hi : hj;
    const T thrust_b = -T(G_ACC) * (hr - T(0.5) * fabs(dzt)) * dzt;
    const bool mt = (dz * dd >= T(0)) && (ut * dz > T(0));
    const T thrust = mt ? nan_max(thrust_a, thrust_b) : thrust_b;
    const T nt = T(0.5) * (ni + nj);
    const T sf = (nt * nt * d_sqrt(ut * ut + vt * vt) * ut) / clamp_lo(d_pow(ht, T(4.0 / 3.0)), T(DRY_TOL));
    const T tau = T(G_ACC) * ht * sf * dx;
    const T T1 = thrust - tau;
    // P^-1 (0, T1, 0) (roe.py:159-165)
    T b1 = p00 * T(0) + p01 * T1 + T(0) * T(0);
    const T b2 = p10 * T(0) + T(0) * T1 + p12 * T(0);
    T b3 = p20 * T(0) + p21 * T1 + T(0) * T(0);
    const T hs1 = hi + a1 - (b1 / l1);
    const T hs3 = hj - a3 + (b3 / l3);
    const T b1min = -(hi + a1) * fabs(l1);
    const T b3min = -(hi - a1) * fabs(l3);
    const T dtf = dx / nan_max(nan_max(fabs(l1), fabs(l2)), fabs(l3));
    const T dt1s = (dx / T(2) * l1) * (hi / (hi - hs1 + T(VEL_TOL)));
    const T dt3s = (dx / T(2) * l3) * (hj / (hj - hs3 + T(VEL_TOL)));
    if ((hs1 < T(0)) && (hs3 > T(0)) && (dt1s < dtf)) {
        b1 = (-b1min >= b3min) ? b1min : b1;
        b3 = -b1;
    }
    if ((hs1 > T(0)) && (hs3 < T(0)) && (dt3s < dtf)) {
        b3 = (-b3min >= b3min) ? b1min : b3;
        b1 = -b3;
    }
    const bool mk1 = (hi < DRY) && (hs1 < T(0));
    const bool mk2 = (hj < DRY) && (hs3 < T(0));
    T p0 = 0, p1 = 0, p2 = 0, n0 = 0, n1 = 0, n2 = 0;
    const T lam[3] = {l1, l2, l3};
    const T alp[3] = {a1, a2, a3};
    const T bet[3] = {b1, b2, b3};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const T w = lam[k] * alp[k] - bet[k];
        const T f0 = (k == 1) ? w * T(0) : w;
        const T f1 = (k == 0) ? w * l1 : (k == 2 ? w * l3 : w * T(0));
        const T f2 = (k == 1) ? w * ct : w * vt;
        const bool pos = mk2 ? false : (mk1 ? true : (lam[k] > T(0)));
        const bool neg = mk2 ? true : (mk1 ? false : (lam[k] <= T(0)));
        if (pos) { p0 = p0 + f0; p1 = p1 + f1; p2 = p2 + f2; }
        if (neg) { n0 = n0 + f0; n1 = n1 + f1; n2 = n2 + f2; }
    }
    {
        const T e = lE1 * a1;
        if (lE1 > T(0)) { p0 = p0 + e; p1 = p1 + e * l1; p2 = p2 + e * vt; }
        else if (lE1 <= T(0)) { n0 = n0 + e; n1 = n1 + e * l1; n2 = n2 + e * vt; }
    }
    {
        const T e = lE3 * a3;
        if (lE3 > T(0)) { p0 = p0 + e; p1 = p1 + e * l3; p2 = p2 + e * vt; }
        else if (lE3 <= T(0)) { n0 = n0 + e; n1 = n1 + e * l3; n2 = n2 + e * vt; }
    }
    if (YF) {
        P[0] = p0; P[1] = p2; P[2] = -p1;
        M[0] = n0; M[1] = n2; M[2] = -n1;
    } else {
        P[0] = p0; P[1] = p1; P[2] = p2;
        M[0] = n0; M[1] = n1; M[2] = n2;
    }
}

// Update of cell (r, c) from its four faces (roe.py:251-315), order of roe.py:296-299.
// Update of cell (r, c) by the four threads of its quad (adjacent lanes qbase..qbase+3):
// thread q evaluates face q of the cell (0 east, 1 west, 2 south = row + 1, 3 north =
// row - 1) and the sums run in that order, the scatter order of roe.py (east upwM, west
// upwP, south upwM, north upwP).  One face per thread: the 66 k-cell configuration of
// this path is latency-bound, and four threads per cell keep four times as many in
// flight as one thread evaluating the four faces in turn.
template <class T>
__device__ __forceinline__ void roe_quad_update(const RoeArgs<T>& a, int r, int c, T dt, int q, unsigned qmask,
                                                int qbase, T out[3]) {
    const long long p = a.pitch;
    const long long i = (long long)r * p + c;
    const bool first = (q & 1) == 0;  // the cell is the face's i side (east, south faces)
    const bool yf = q >= 2;
    const bool has = q == 0 ? (c + 1 < a.nx) : q == 1 ? (c >= 1) : q == 2 ? (r + 1 < a.ny) : (r >= 1);
    const long long j = q == 0 ? i + 1 : q == 1 ? i - 1 : q == 2 ? i + p : i - p;
    T v[3] = {T(0), T(0), T(0)};
    if (has) {
        const long long ii = first ? i : j, jj = first ? j : i;
        T P[3], M[3];
        roe_plain_face<T>(a.h[ii], a.hu[ii], a.hv[ii], a.z[ii], a.n[ii], a.h[jj], a.hu[jj], a.hv[jj], a.z[jj], a.n[jj],
                          a.dx, yf, P, M);
#pragma unroll
        for (int m = 0; m < 3; ++m) v[m] = first ? M[m] : P[m];
    }
    T f[3] = {T(0), T(0), T(0)};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const bool hk = __shfl_sync(qmask, (int)has, qbase + k) != 0;
#pragma unroll
        for (int m = 0; m < 3; ++m) {
            const T vk = __shfl_sync(qmask, v[m], qbase + k);
            if (hk) f[m] = f[m] + vk;
        }
    }
    out[0] = a.h[i] - dt * f[0] / a.dx;
    out[1] = a.hu[i] - dt * f[1] / a.dx;
    out[2] = a.hv[i] - dt * f[2] / a.dx;
}

// The larger of the two speeds of compute_dt for plain Roe (roe.py:13-30) at one cell,
// |u| + c + VEL_TOL and |v| + c + VEL_TOL, as an IEEE bit pattern (speeds are positive or
// NaN, so unsigned order is float order and NaN wins).
template <class T>
__device__ __forceinline__ unsigned long long roe_cell_speed_bits(T h0, T hu0, T hv0) {
    const bool wet = h0 > T(DRY_TOL);
    const T h = wet ? h0 : T(0);
    const T hv = wet ? hv0 : T(0);
    const T hu = wet ? hu0 : T(0);
    const T u = hu / (h + T(DRY_TOL));
    const T v = hv / (h + T(DRY_TOL));
    const T cc = d_sqrt(T(G_ACC) * h);
    const T sx = fabs(u) + cc + T(VEL_TOL);
    const T sy = fabs(v) + cc + T(VEL_TOL);
    const unsigned long long bx = speed_bits(sx), by = speed_bits(sy);
    return bx > by ? bx : by;
}

// Max over the launch of the threads' speed bits (warp max, block max through shared
// memory, one atomicMax per block), and the last block to finish turns it into
// dt = cfl * dx / smax (no floor), logs it and resets the accumulator.  Every thread of
// every block calls it once, at its end.
template <class T>
__device__ __forceinline__ void roe_dt_reduce(unsigned long long best, CflScratch* scr, T cfl, T dx, T* dt_out,
                                              T* dt_log) {
    const int lane = threadIdx.x & 31;
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long other = __shfl_xor_sync(FULL, best, o);
        best = other > best ? other : best;
    }
    __shared__ unsigned long long wmax[32];
    if (lane == 0) wmax[threadIdx.x >> 5] = best;
    __syncthreads();
    if (threadIdx.x != 0) return;
    for (int w = 1; w < (int)((blockDim.x + 31) >> 5); ++w) best = wmax[w] > best ? wmax[w] : best;
    if (best != 0ull) atomicMax(&scr->maxbits, best);
    __threadfence();  // the block's maximum before its ticket
    const unsigned int ticket = atomicAdd(&scr->done, 1u);
    if (ticket != gridDim.x - 1) return;
    __threadfence();
    const unsigned long long bits = atomicAdd(&scr->maxbits, 0ull);
    const T smax = bits_speed(bits, T(0));
    const T dt = cfl * (dx / smax);
    *dt_out = dt;
    if (dt_log) dt_log[scr->step] = dt;
    scr->step += 1;
    if (!d_isfinite(dt)) scr->err |= 2;
    scr->maxbits = 0ull;
    scr->done = 0u;
    __threadfence();
}

// One stage; four threads per cell.  Ring cells with boundary recipes recompute the
// update of their donor cell instead of reading it, so the stage is one launch with no
// global synchronisation.
// Resident 256-thread blocks per SM the stage is register-limited to (tuning knob): 4
// (64 registers, a few hundred bytes of spills) runs the 256^2 dam break's 266 k threads
// in 2 waves instead of 2.3, 3 % faster than 3 (80 registers) and 8 % faster than 2.
#ifndef PXB_ROE_MIN_BLOCKS
#define PXB_ROE_MIN_BLOCKS 4
#endif

template <class T, bool AVG>
__global__ void __launch_bounds__(256, PXB_ROE_MIN_BLOCKS) roe_stage_kernel(const RoeArgs<T> a) {
    const int lane = threadIdx.x & 31;
    const int qbase = lane & ~3;
    const unsigned qmask = 0xFu << qbase;
    const long long tid = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long cell = tid >> 2;
    const int q = (int)(tid & 3);
    if (cell >= (long long)a.ny * a.nx) return;  // whole quads leave together
    const int r = (int)(cell / a.nx), c = (int)(cell - (long long)r * a.nx);
    const T dt = *a.dt;
    const long long i = (long long)r * a.pitch + c;
    const bool on_ring = (r == 0) || (r == a.ny - 1) || (c == 0) || (c == a.nx - 1);
    // The same for the four threads of the quad: Roe handlers write h, z and n from one
    // donor (flags bit 0) and the momentum from another (bit 1: a 2x2 map of the donor's,
    // or constants with bit 2).
    unsigned flags = 0u;
    int hdy = 0, hdx = 0, mdy = 0, mdx = 0;
    T m0 = T(0), m1 = T(0), m2 = T(0), m3 = T(0);
    if (on_ring && a.ring != nullptr) {
        const pxb_ring_recipe& rc = a.ring[ring_slot(r, c, a.ny, a.nx)];
        flags = rc.flags;
        hdy = rc.h_dy, hdx = rc.h_dx, mdy = rc.m_dy, mdx = rc.m_dx;
        m0 = T(rc.m[0]), m1 = T(rc.m[1]), m2 = T(rc.m[2]), m3 = T(rc.m[3]);
    }
    // Updates evaluated in turn by one inlined copy of the quad update: the cell itself
    // (unless both of its parts come from donors), the h donor, the momentum donor.
    T u[3] = {T(0), T(0), T(0)}, dh[3] = {T(0), T(0), T(0)}, dm[3] = {T(0), T(0), T(0)};
#pragma unroll 1
    for (int pass = 0; pass < 3; ++pass) {
        int rr = r, cc = c;
        if (pass == 0 && (flags & 3u) == 3u) continue;
        if (pass == 1) {
            if (!(flags & 1u)) continue;
            rr = r + hdy, cc = c + hdx;
        }
        if (pass == 2) {
            if (!(flags & 2u) || (flags & 4u)) continue;
            rr = r + mdy, cc = c + mdx;
        }
        T d[3];
        roe_quad_update(a, rr, cc, dt, q, qmask, qbase, d);
#pragma unroll
        for (int m = 0; m < 3; ++m) {
            u[m] = pass == 0 ? d[m] : u[m];
            dh[m] = pass == 1 ? d[m] : dh[m];
            dm[m] = pass == 2 ? d[m] : dm[m];
        }
    }
    T zo = a.z[i], no = a.n[i];
    if (flags & 1u) {
        u[0] = dh[0];
        const long long j = (long long)(r + hdy) * a.pitch + (c + hdx);
        zo = a.z[j];
        no = a.n[j];
    }
    if (flags & 2u) {
        if (flags & 4u) {
            u[1] = m0;
            u[2] = m1;
        } else {
            u[1] = m0 * dm[1] + m1 * dm[2];
            u[2] = m2 * dm[1] + m3 * dm[2];
        }
    }
    if (q != 0) return;  // the quad's first thread writes the cell
    if (AVG) {
        u[0] = T(0.5) * a.ah[i] + T(0.5) * u[0];
        u[1] = T(0.5) * a.ahu[i] + T(0.5) * u[1];
        u[2] = T(0.5) * a.ahv[i] + T(0.5) * u[2];
        zo = T(0.5) * a.az[i] + T(0.5) * zo;
        no = T(0.5) * a.an[i] + T(0.5) * no;
    }
    a.oh[i] = u[0];
    a.ohu[i] = u[1];
    a.ohv[i] = u[2];
    if (on_ring) {
        a.oz[i] = zo;
        a.on[i] = no;
    }
    if (!(d_isfinite(u[0]) && d_isfinite(u[1]) && d_isfinite(u[2]))) atomicOr(a.err, 1);
}

// compute_dt for plain Roe (roe.py:13-30): cfl * dx / max over ALL cells of
// (|u| + c + VEL_TOL) and (|v| + c + VEL_TOL); no floor.
template <class T>
__global__ void __launch_bounds__(256) roe_cfl_kernel(const CflArgs<T> a) {
    unsigned long long best = 0ull;
    const long long ncell = (long long)a.ny * a.nx;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < ncell; k += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(k / a.nx), c = (int)(k - (long long)r * a.nx);
        const long long i = (long long)r * a.pitch + c;
        const unsigned long long b = roe_cell_speed_bits(a.h[i], a.hu[i], a.hv[i]);
        best = b > best ? b : best;
    }
    roe_dt_reduce<T>(best, a.scr, a.cfl, a.dx, a.dt_out, a.dt_log);
}

}  // namespace pxb
