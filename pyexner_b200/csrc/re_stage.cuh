// Fused Roe-Exner stage kernel (one launch per Runge-Kutta stage).
//
// Replaces step_fn_roeexner (PyExner src/PyExner/solvers/roe_exner_solver.py:80-116) on
// one rank: hydro update (roe_exner.py:535-612) -> momentum corrections (:14-62) ->
// boundary handlers -> grass factor (:85-140) -> Exner update (:665-717) -> boundary
// handlers, and for the second SSPRK2 stage the 0.5/0.5 combination (SSPRK2.py:40).
//
// Layout of the work: a warp owns a strip of 32 columns (3 halo | 26 owned | 3 halo) and
// marches down a band of rows.  Each iteration consumes one new row, copied into the
// warp's shared buffer by cp.async during the previous iteration (together with the
// partner-state values the averaging stage stores in this one), and advances a software
// pipeline held in registers:
//   A  row r   : cell precompute, x-face fluxes (east neighbour by shuffle), y-face (r-1|r)
//   B  row r-1 : hydro update (all four faces known)
//   C  row r-2 : momentum corrections (needs updated depths of rows r-3..r-1)
//   D  row r-3 : first boundary application on ring cells (donors in rows r-4..r-2)
//   E  row r-3 : grass factor, Exner cell, Exner x-faces and y-face (r-4|r-3)
//   F  row r-4 : z_b update
//   G  row r-5 : second boundary application on z_b and G, then the z_b / G stores
// Hydro fields are stored after D (the second application leaves them unchanged for
// the layouts the host accepts).  Every face is evaluated once per warp; the only
// redundant work is the 6 halo columns of each strip and 6 halo rows of each band.
#pragma once
#include <type_traits>

#include "pxb_device.cuh"

// Resident 128-thread blocks per SM the build is register-limited to (tuning knobs,
// measured on the 2048^2 and 8192^2 Gaussian-bed cases): 4 (128 registers, no spills)
// for both the plain stage and the averaging second SSPRK2 stage; 5 (96 registers) is
// 1% faster at 8192^2 and 4% slower at 2048^2, where fewer resident warps mean taller
// bands and fewer redundant halo rows.
#ifndef PXB_STAGE_MIN_BLOCKS
#define PXB_STAGE_MIN_BLOCKS 4
#endif
#ifndef PXB_STAGE_MIN_BLOCKS_AVG
#define PXB_STAGE_MIN_BLOCKS_AVG 4
#endif
// float64 state (twice the registers per value)
#ifndef PXB_STAGE_MIN_BLOCKS_F64
#define PXB_STAGE_MIN_BLOCKS_F64 5
#endif
// Unroll factor of the steady row loop (tuning knob).
#ifndef PXB_STAGE_UNROLL
#define PXB_STAGE_UNROLL 1
#endif
#define PXB_PRAGMA(x) _Pragma(#x)
#define PXB_UNROLL(n) PXB_PRAGMA(unroll n)
#define PXB_STAGE_BOUNDS(T, AVG) \
    (sizeof(T) == 8 ? PXB_STAGE_MIN_BLOCKS_F64 : ((AVG) ? PXB_STAGE_MIN_BLOCKS_AVG : PXB_STAGE_MIN_BLOCKS))

namespace pxb {

template <class T>
struct REStageArgs {
    int ny, nx;
    long long pitch;
    T dx;
    const T *h, *hu, *hv, *zb, *z, *nb, *G;  // stage input (G read in constant-G mode)
    const uint8_t* nodata;                    // mask[0] or null
    T *oh, *ohu, *ohv, *ozb, *oG;            // stage output (oG may be null)
    const T *ah, *ahu, *ahv, *azb, *aG;      // SSPRK2 partner u^n (AVG)
    const T* dt;
    const pxb_ring_recipe* ring;              // null when there are no handlers
    SedTable<T> sed;
    int band_rows, nstrips, nbands;
    int* err;
    unsigned int* queue;  // {next dynamic item, finished blocks}, zero between launches
};

// Asynchronous global -> shared copies of one element (cp.async, completion by group).
template <class T>
__device__ __forceinline__ void cp_async_elem(T* smem, const T* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    if constexpr (sizeof(T) == 4) asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
    else asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
static_assert(sizeof(pxb_ring_recipe) == 48, "ring recipes are copied as three 16-byte chunks");

// Fields of the second boundary application (z_b and G donors) packed into one word by
// the first: flags bits 3-4 and the four offsets (each in [-1, 1]) biased by 8.
__device__ __forceinline__ unsigned pack_zg(unsigned flags, int zdy, int zdx, int gdy, int gdx) {
    return (flags & 24u) | ((unsigned)(zdy + 8) << 8) | ((unsigned)(zdx + 8) << 12) | ((unsigned)(gdy + 8) << 16) |
           ((unsigned)(gdx + 8) << 20);
}
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

template <class T>
__device__ __forceinline__ T pick_row(int dy, T above, T mid, T below) {
    return dy < 0 ? above : (dy > 0 ? below : mid);
}

template <class T>
__device__ __forceinline__ HCell<T> shfl_down_hcell(const HCell<T>& p) {
    HCell<T> q;
    q.h = __shfl_down_sync(FULL, p.h, 1);
    q.u = __shfl_down_sync(FULL, p.u, 1);
    q.v = __shfl_down_sync(FULL, p.v, 1);
    q.sq = __shfl_down_sync(FULL, p.sq, 1);
    q.c = __shfl_down_sync(FULL, p.c, 1);
    q.zt = __shfl_down_sync(FULL, p.zt, 1);
    q.nb = __shfl_down_sync(FULL, p.nb, 1);
    return q;
}

template <class T>
__device__ __forceinline__ ECell<T> shfl_down_ecell(const ECell<T>& p) {
    ECell<T> q;
    q.h = __shfl_down_sync(FULL, p.h, 1);
    q.zb = __shfl_down_sync(FULL, p.zb, 1);
    q.zbe = __shfl_down_sync(FULL, p.zbe, 1);
    q.sq = __shfl_down_sync(FULL, p.sq, 1);
    q.u = __shfl_down_sync(FULL, p.u, 1);
    q.v = __shfl_down_sync(FULL, p.v, 1);
    q.um = __shfl_down_sync(FULL, p.um, 1);
    q.G = __shfl_down_sync(FULL, p.G, 1);
    return q;
}

// One work item (a strip of one band) of a stage; the single-grid kernel and the
// ensemble kernel (ens_stage.cuh) both loop over items and call this.
template <class T, bool MPM, bool HAS_MASK, bool AVG>
__device__ __forceinline__ void re_stage_item(const REStageArgs<T>& a, const int item, bool& bad) {
    const int lane = threadIdx.x & 31;
    const int ny = a.ny, nx = a.nx;
    const unsigned upitch = (unsigned)a.pitch;  // planes are < 2^31 elements (checked at plan creation)
    const T dt = *a.dt;
    const T dx = a.dx;
    const T dtdx = dt / dx;  // float path only
    const T DRY = T(DRY_TOL);
    {
        const int ipb = pxb_stage_items_per_band(a.nstrips);
        const int band = item / ipb;
        const int k = item - band * ipb;
        int strip = k - 1, half = -1;  // half: 0 / 1 = upper / lower half of a boundary strip
        if (ipb == 1) strip = 0;
        else if (k < 2) { strip = 0; half = k; }
        else if (k >= a.nstrips) { strip = a.nstrips - 1; half = k - a.nstrips; }
        const int c = strip * PXB_STRIP_OUT - PXB_HALO + lane;
        const bool colok = (c >= 0) && (c < nx);
        const bool has_e = colok && (c + 1 < nx) && (lane < 31);
        const bool last_strip = strip == a.nstrips - 1;
        const bool out_col = colok && lane >= PXB_HALO && (lane < PXB_HALO + PXB_STRIP_OUT || last_strip);
        const bool interior_col = (c >= 1) && (c <= nx - 2);
        const int B0 = band * a.band_rows;
        const int B1 = (band == a.nbands - 1) ? ny : B0 + a.band_rows;
        const int Bm = B0 + (B1 - B0 + 1) / 2;
        const int R0 = half == 1 ? Bm : B0;
        const int R1 = half == 0 ? Bm : B1;
        const int L0 = max(0, R0 - 3), L1 = min(ny, R1 + 3);
        // boundary recipes can only apply in the first/last strip or on rows 0 / ny-1
        const bool bc_strip = (a.ring != nullptr) && (strip == 0 || last_strip);
        const bool bc_rows = (a.ring != nullptr) && (R0 == 0 || R1 == ny);

        // ---- carried pipeline state
        HCell<T> pA = make_hcell(T(0), T(0), T(0), T(0), T(0), T(0));
        T hA = 0, huA = 0, hvA = 0, ztA = 0;
        T xfA0 = 0, xfA1 = 0, xfA2 = 0, nfA0 = 0, nfA1 = 0, nfA2 = 0;
        T hr3 = 0, hr2 = 0, hur2 = 0, hvr2 = 0, zt3 = 0, zt2 = 0;
        unsigned mwin = 0;  // bit k = nodata of row r-1-k
        T zin1 = 0, zin2 = 0, zin3 = 0, zin4 = 0;
        T gin1 = 0, gin2 = 0, gin3 = 0, gin4 = 0;
        T hf4h = 0, hf4u = 0, hf4v = 0, hf3h = 0, hf3u = 0, hf3v = 0;
        ECell<T> e4 = make_ecell(T(0), T(0), T(0), T(0), T(0));
        T xe4 = 0, fn4 = 0;
        T zbp6 = 0, zbp5 = 0, gg6 = 0, gg5 = 0;

        // Row r+1 is fetched while row r is computed: the loads of one iteration are in
        // flight during the ~thousand instructions of the previous one.  In float32 they
        // are cp.async copies into this warp's shared buffer (no registers held); in
        // float64 (measured: faster there) plain loads into registers.
        constexpr bool ASYNC_ROWS = is_f32<T>();
        constexpr int NP = MPM ? 6 : 7;
        __shared__ T rbuf[4][ASYNC_ROWS ? 2 : 1][ASYNC_ROWS ? NP : 1][32];
        T(*rb)[ASYNC_ROWS ? NP : 1][32] = rbuf[threadIdx.x >> 5];
        T nh = 0, nhu = 0, nhv = 0, nzb = 0, nz = 0, nnb = 0, ng = 0;
        bool nm = false;
        auto load_row = [&](int rr) {
            const int b = rr & 1;
            if constexpr (!ASYNC_ROWS) {
                if (rr < L1 && colok) {
                    const unsigned i = (unsigned)rr * upitch + (unsigned)c;
                    nh = __ldg(a.h + i);
                    nhu = __ldg(a.hu + i);
                    nhv = __ldg(a.hv + i);
                    nzb = __ldg(a.zb + i);
                    nz = __ldg(a.z + i);
                    nnb = __ldg(a.nb + i);
                    if (!MPM) ng = __ldg(a.G + i);
                    if (HAS_MASK) nm = __ldg(a.nodata + i) != 0;
                } else {
                    nh = nhu = nhv = nzb = nz = nnb = ng = T(0);
                    nm = false;
                }
            } else {
                if (rr < L1 && colok) {
                    const unsigned i = (unsigned)rr * upitch + (unsigned)c;
                    cp_async_elem(&rb[b][0][lane], a.h + i);
                    cp_async_elem(&rb[b][1][lane], a.hu + i);
                    cp_async_elem(&rb[b][2][lane], a.hv + i);
                    cp_async_elem(&rb[b][3][lane], a.zb + i);
                    cp_async_elem(&rb[b][4][lane], a.z + i);
                    cp_async_elem(&rb[b][5][lane], a.nb + i);
                    if constexpr (!MPM) cp_async_elem(&rb[b][NP - 1][lane], a.G + i);
                    if (HAS_MASK) nm = __ldg(a.nodata + i) != 0;
                } else {
#pragma unroll
                    for (int k = 0; k < NP; ++k) rb[b][k][lane] = T(0);
                    nm = false;
                }
            }
        };
        load_row(L0);
        // Averaging stage: the partner state's values of the cells stored in iteration r
        // (rows r-3 and r-5).  In float32 they are copied asynchronously into this warp's
        // shared buffer during iteration r-1, so they cost neither registers nor a wait at
        // the store; in float64 (measured: the shared-buffer form is slower there) they
        // are loaded into registers at the start of iteration r.  Only the owning lane
        // reads and then writes these cells, so both are safe when the output aliases the
        // partner.
        constexpr bool ASYNC_PARTNER = AVG && is_f32<T>();
        __shared__ T pbuf[4][ASYNC_PARTNER ? 2 : 1][5][32];
        T(*pb)[5][32] = pbuf[threadIdx.x >> 5];
        auto partner_copy = [&](const int rr) {  // the rows stored in iteration rr
            const int q0 = rr - 3, p0 = rr - 5;
            const int b = rr & 1;
            if (q0 >= L0 && q0 < L1 && q0 >= R0 && q0 < R1 && out_col) {
                const unsigned i = (unsigned)q0 * upitch + (unsigned)c;
                cp_async_elem(&pb[b][0][lane], a.ah + i);
                cp_async_elem(&pb[b][1][lane], a.ahu + i);
                cp_async_elem(&pb[b][2][lane], a.ahv + i);
            }
            if (p0 >= L0 && p0 < L1 && p0 >= R0 && p0 < R1 && out_col) {
                const unsigned i = (unsigned)p0 * upitch + (unsigned)c;
                cp_async_elem(&pb[b][3][lane], a.azb + i);
                if (a.oG) cp_async_elem(&pb[b][4][lane], a.aG + i);
            }
        };
        if (ASYNC_PARTNER) partner_copy(L0);
        cp_async_commit();
        // Boundary recipes (first / last strip, first / last row): the recipe of the row
        // that the first boundary application treats in iteration r (q = r-3) is copied
        // into this warp's shared buffer during iteration r-1, so no recipe load is waited
        // on inside the pipeline; the first application leaves the z_b / G fields of the
        // second (row p = r-5, two iterations later) in a packed word.  Float32 only, as
        // the row copies.
        constexpr bool ASYNC_RECIPES = ASYNC_ROWS;
        __shared__ __align__(16) pxb_ring_recipe rcbuf[4][ASYNC_RECIPES ? 2 : 1][32];
        __shared__ unsigned zgbuf[4][ASYNC_RECIPES ? 4 : 1][32];
        pxb_ring_recipe(*rcb)[32] = rcbuf[threadIdx.x >> 5];
        unsigned(*zgb)[32] = zgbuf[threadIdx.x >> 5];
        auto recipe_copy = [&](const int rr) {  // the recipes used in iteration rr
            const int qn = rr - 3;
            if (qn >= L0 && qn < L1 && (bc_strip || (bc_rows && (qn == 0 || qn == ny - 1)))) {
                const int slot = colok ? ring_slot(qn, c, ny, nx) : -1;
                pxb_ring_recipe* d = &rcb[rr & 1][lane];
                if (slot >= 0) {
                    const char* src = reinterpret_cast<const char*>(a.ring + slot);
                    char* dst = reinterpret_cast<char*>(d);
                    cp_async16(dst, src);
                    cp_async16(dst + 16, src + 16);
                    cp_async16(dst + 32, src + 32);
                } else {
                    d->flags = 0u;
                }
            }
        };

        // One pipeline iteration.  In the steady state (rows L0+5 .. L1-1) every phase has
        // valid rows, so the row checks compile away.
        auto iterate = [&](const int r, auto steady_tag) {
            constexpr bool S = decltype(steady_tag)::value;
            const bool rowA = S || r < L1;
            // ================= A: row r (prefetched), x-faces of row r, y-face (r-1 | r)
            T h_r, hu_r, hv_r, zb_r, z_r, nb_r, g_r = T(0);
            if constexpr (ASYNC_ROWS) {
                cp_async_wait<0>();  // row r (and the partner rows stored in this iteration)
                const int rbb = r & 1;
                h_r = rb[rbb][0][lane];
                hu_r = rb[rbb][1][lane];
                hv_r = rb[rbb][2][lane];
                zb_r = rb[rbb][3][lane];
                z_r = rb[rbb][4][lane];
                nb_r = rb[rbb][5][lane];
                if constexpr (!MPM) g_r = rb[rbb][NP - 1][lane];
            } else {
                h_r = nh, hu_r = nhu, hv_r = nhv, zb_r = nzb, z_r = nz, nb_r = nnb, g_r = ng;
            }
            const bool m_r = nm;
            load_row(r + 1);
            if (ASYNC_PARTNER) partner_copy(r + 1);
            if (ASYNC_RECIPES) recipe_copy(r + 1);
            cp_async_commit();
            T pah = 0, pahu = 0, pahv = 0, pazb = 0, paG = 0;
            if (ASYNC_PARTNER) {
                // read at the stores below
            } else if (AVG) {
                const int q0 = r - 3, p0 = r - 5;
                if ((S || (q0 >= L0 && q0 < L1)) && q0 >= R0 && q0 < R1 && out_col) {
                    const unsigned i = (unsigned)q0 * upitch + (unsigned)c;
                    pah = a.ah[i];
                    pahu = a.ahu[i];
                    pahv = a.ahv[i];
                }
                if ((S || (p0 >= L0 && p0 < L1)) && p0 >= R0 && p0 < R1 && out_col) {
                    const unsigned i = (unsigned)p0 * upitch + (unsigned)c;
                    pazb = a.azb[i];
                    if (a.oG) paG = a.aG[i];
                }
            }
            const HCell<T> pr = make_hcell(h_r, hu_r, hv_r, zb_r, z_r, nb_r);
            const T zt_r = z_r + zb_r;
            T xf0 = 0, xf1 = 0, xf2 = 0;
            // In the prologue / drain iterations of a band the faces of invalid rows are
            // skipped for the whole warp (r is warp-uniform); their results would be masked.
            if (S || rowA) {
                const HCell<T> pe = shfl_down_hcell(pr);
                const T he = __shfl_down_sync(FULL, h_r, 1);
                const bool me = HAS_MASK ? (__shfl_down_sync(FULL, (int)m_r, 1) != 0) : false;
                const bool xact = rowA && has_e && ((h_r > DRY) || (he > DRY)) && !(m_r || me);
                T P[3], M[3];
                roe_exner_face<T, false>(pr, pe, dx, P, M);
#pragma unroll
                for (int k = 0; k < 3; ++k) { P[k] = xact ? P[k] : T(0); M[k] = xact ? M[k] : T(0); }
                const T w0 = __shfl_up_sync(FULL, P[0], 1);
                const T w1 = __shfl_up_sync(FULL, P[1], 1);
                const T w2 = __shfl_up_sync(FULL, P[2], 1);
                const bool wact = (__shfl_up_sync(FULL, (int)xact, 1) != 0) && lane > 0;
                // scatter order of roe_exner.py:599-600: east upwM first, then west upwP
                if (xact) { xf0 = xf0 + M[0]; xf1 = xf1 + M[1]; xf2 = xf2 + M[2]; }
                if (wact) { xf0 = xf0 + w0; xf1 = xf1 + w1; xf2 = xf2 + w2; }
            }
            T yP[3] = {T(0), T(0), T(0)}, yM[3] = {T(0), T(0), T(0)};
            const bool yact = rowA && (S || r - 1 >= L0) && colok && ((hA > DRY) || (h_r > DRY)) && !((mwin & 1u) || m_r);
            if (S || (rowA && r - 1 >= L0)) {
                roe_exner_face<T, true>(pA, pr, dx, yP, yM);
#pragma unroll
                for (int k = 0; k < 3; ++k) { yP[k] = yact ? yP[k] : T(0); yM[k] = yact ? yM[k] : T(0); }
            }

            // ================= B: hydro update of row r-1
            T hr1 = 0, hur1 = 0, hvr1 = 0;
            if (S || (r - 1 >= L0 && r - 1 < L1)) {
                T f0 = xfA0, f1 = xfA1, f2 = xfA2;
                f0 = f0 + yM[0]; f1 = f1 + yM[1]; f2 = f2 + yM[2];      // south face upwM
                f0 = f0 + nfA0; f1 = f1 + nfA1; f2 = f2 + nfA2;         // north face upwP
                if constexpr (is_f32<T>()) {
                    hr1 = hA - dtdx * f0;
                    hur1 = huA - dtdx * f1;
                    hvr1 = hvA - dtdx * f2;
                } else {
                    hr1 = hA - dt * f0 / dx;
                    hur1 = huA - dt * f1 / dx;
                    hvr1 = hvA - dt * f2 / dx;
                }
            }

            // ================= C: momentum corrections of row r-2
            T hf2h = 0, hf2u = 0, hf2v = 0;
            {
                const int q2 = r - 2;
                const T hE = __shfl_down_sync(FULL, hr2, 1), hW = __shfl_up_sync(FULL, hr2, 1);
                const T zE = __shfl_down_sync(FULL, zt2, 1), zW = __shfl_up_sync(FULL, zt2, 1);
                const bool m2 = HAS_MASK && ((mwin >> 1) & 1u);
                const bool mE = HAS_MASK ? (__shfl_down_sync(FULL, (int)m2, 1) != 0) : false;
                const bool mW = HAS_MASK ? (__shfl_up_sync(FULL, (int)m2, 1) != 0) : false;
                if (S || (q2 >= L0 && q2 < L1)) {
                    hf2h = hr2;
                    hf2u = hur2;
                    hf2v = hvr2;
                    if (interior_col && q2 >= 1 && q2 <= ny - 2) {
                        const bool mN = HAS_MASK && ((mwin >> 2) & 1u);
                        const bool mS = HAS_MASK && (mwin & 1u);
                        const T eta = hr2 + zt2;
                        const bool stop_u = ((eta < zE) && (hE < DRY)) || ((eta < zW) && (hW < DRY)) || mE || mW;
                        const bool stop_v = ((eta < zt3) && (hr3 < DRY)) || ((eta < ztA) && (hr1 < DRY)) || mN || mS;
                        const bool active = (hr2 > DRY) && !m2;
                        hf2u = (active && !stop_u) ? hur2 : T(0);
                        hf2v = (active && !stop_v) ? hvr2 : T(0);
                    }
                }
            }

            // ================= D: boundary passes for the hydro fields of row q = r-3
            // The first pass maps pre-boundary values (HF, input z_b / G) of the donors; the
            // stored h, hu, hv are the second pass, which maps first-pass values: a donor in
            // the same row contributes its first-pass value, a donor in another row is never
            // a hydro boundary cell (checked at plan creation), so its value is HF.
            const int q = r - 3;
            const bool rowD = S || ((q >= L0) && (q < L1));
            T hbh = hf3h, hbu = hf3u, hbv = hf3v, zb1 = zin3, gb1 = gin3;
            T sbh = hf3h, sbu = hf3u, sbv = hf3v;
            if (rowD && (bc_strip || (bc_rows && (q == 0 || q == ny - 1)))) {
                unsigned flags = 0;
                int hdy = 0, hdx = 0, mdy = 0, mdx = 0, zdy = 0, zdx = 0, gdy = 0, gdx = 0;
                T m0 = 0, m1 = 0, m2c = 0, m3 = 0;
                auto take = [&](const pxb_ring_recipe& rc) {
                    flags = rc.flags;
                    hdy = rc.h_dy; hdx = rc.h_dx; mdy = rc.m_dy; mdx = rc.m_dx;
                    zdy = rc.zb_dy; zdx = rc.zb_dx; gdy = rc.g_dy; gdx = rc.g_dx;
                    m0 = T(rc.m[0]); m1 = T(rc.m[1]); m2c = T(rc.m[2]); m3 = T(rc.m[3]);
                };
                if constexpr (ASYNC_RECIPES) {
                    const pxb_ring_recipe& rc = rcb[r & 1][lane];  // copied in iteration r-1
                    if (rc.flags != 0u) take(rc);
                    zgb[r & 3][lane] = pack_zg(flags, zdy, zdx, gdy, gdx);
                } else {
                    const int slot = colok ? ring_slot(q, c, ny, nx) : -1;
                    if (slot >= 0) take(a.ring[slot]);
                }
                if (__any_sync(FULL, flags != 0)) {
                    // Donor value at (row q+dy, column c+dx); the row is chosen by the
                    // receiver.  Donors lie in another row only for cells of the first and
                    // last rows (plan creation checks it), so other rows shuffle one value.
                    const bool dyrow = (q == 0) || (q == ny - 1);
                    auto fetch = [&](int dy, int dx_, T above, T mid, T below) {
                        const T vm = __shfl_sync(FULL, mid, lane + dx_);
                        if (!dyrow) return vm;
                        const T va = __shfl_sync(FULL, above, lane + dx_);
                        const T vb = __shfl_sync(FULL, below, lane + dx_);
                        return pick_row(dy, va, vm, vb);
                    };
                    const T vh = fetch(hdy, hdx, hf4h, hf3h, hf2h);
                    const T vu = fetch(mdy, mdx, hf4u, hf3u, hf2u);
                    const T vv = fetch(mdy, mdx, hf4v, hf3v, hf2v);
                    const T vz = fetch(zdy, zdx, zin4, zin3, zin2);
                    if (flags & 1u) hbh = vh;
                    if (flags & 2u) {
                        if (flags & 4u) { hbu = m0; hbv = m1; }
                        else { hbu = sum2(m0, vu, m1, vv); hbv = sum2(m2c, vu, m3, vv); }
                    }
                    if (flags & 8u) zb1 = vz;
                    if (!MPM) {
                        const T vg = fetch(gdy, gdx, gin4, gin3, gin2);
                        if (flags & 16u) gb1 = vg;
                    }
                    // second pass
                    const T wh = fetch(hdy, hdx, hf4h, hbh, hf2h);
                    const T wu = fetch(mdy, mdx, hf4u, hbu, hf2u);
                    const T wv = fetch(mdy, mdx, hf4v, hbv, hf2v);
                    sbh = hbh;
                    sbu = hbu;
                    sbv = hbv;
                    if (flags & 1u) sbh = wh;
                    if ((flags & 2u) && !(flags & 4u)) {
                        sbu = sum2(m0, wu, m1, wv);
                        sbv = sum2(m2c, wu, m3, wv);
                    }
                }
            }

            // ================= E: grass factor, Exner cell and faces of row q
            const bool mq = HAS_MASK && ((mwin >> 2) & 1u);
            const bool mq1 = HAS_MASK && ((mwin >> 3) & 1u);
            ECell<T> e3{};
            T xe3 = 0, Fy = 0;
            if (S || rowD) {  // warp-uniform: row q is outside the band's rows in some prologue / drain iterations
            const T Gq = MPM ? mpm_grass(hbh, hbu, hbv, mq, a.sed) : const_grass(hbh, gb1, mq);
            e3 = make_ecell(hbh, hbu, hbv, zb1, Gq);
            {
                const ECell<T> ee = shfl_down_ecell(e3);
                const bool mqe = HAS_MASK ? (__shfl_down_sync(FULL, (int)mq, 1) != 0) : false;
                const bool xact = rowD && has_e && exner_active(e3, ee, mq, mqe);
                const T Fx = exner_face<T, false>(e3, ee);
                const T F = xact ? Fx : T(0);
                const T Fw = __shfl_up_sync(FULL, F, 1);
                const bool wact = (__shfl_up_sync(FULL, (int)xact, 1) != 0) && lane > 0;
                // roe_exner.py:710-711: -F of the west face first, then +F of the east face
                if (wact) xe3 = xe3 + (-Fw);
                if (xact) xe3 = xe3 + F;
            }
            const bool yex = rowD && (S || q - 1 >= L0) && colok && exner_active(e4, e3, mq1, mq);
            const T Fyv = exner_face<T, true>(e4, e3);
            Fy = yex ? Fyv : T(0);
            }

            // ================= F: z_b update of row r-4
            T zbp4 = 0;
            if (S || (r - 4 >= L0 && r - 4 < L1)) {
                T acc = xe4;
                acc = acc + (-fn4);  // north face (roe_exner.py:712)
                acc = acc + Fy;      // south face (roe_exner.py:713)
                if constexpr (is_f32<T>()) zbp4 = e4.zb - dtdx * acc;
                else zbp4 = e4.zb - dt * acc / dx;
            }
            const T gg4 = e4.G;

            // ================= G: second boundary application and stores of row p = r-5
            const int p = r - 5;
            const bool rowG = S || ((p >= L0) && (p < L1));
            T zfin = zbp5, gfin = gg5;
            if (rowG && (bc_strip || (bc_rows && (p == 0 || p == ny - 1)))) {
                unsigned flags = 0;
                int zdy = 0, zdx = 0, gdy = 0, gdx = 0;
                if constexpr (ASYNC_RECIPES) {
                    const unsigned w = zgb[(r - 2) & 3][lane];  // left by the first application of row p
                    flags = w & 24u;
                    zdy = (int)((w >> 8) & 15u) - 8;
                    zdx = (int)((w >> 12) & 15u) - 8;
                    gdy = (int)((w >> 16) & 15u) - 8;
                    gdx = (int)((w >> 20) & 15u) - 8;
                } else {
                    const int slot = colok ? ring_slot(p, c, ny, nx) : -1;
                    if (slot >= 0) {
                        const pxb_ring_recipe& rc = a.ring[slot];
                        flags = rc.flags;
                        zdy = rc.zb_dy; zdx = rc.zb_dx; gdy = rc.g_dy; gdx = rc.g_dx;
                    }
                }
                if (__any_sync(FULL, (flags & 24u) != 0)) {
                    T zv = __shfl_sync(FULL, zbp5, lane + zdx), gv = __shfl_sync(FULL, gg5, lane + gdx);
                    if ((p == 0) || (p == ny - 1)) {  // donors in another row: first / last row only
                        const T z6 = __shfl_sync(FULL, zbp6, lane + zdx), z4 = __shfl_sync(FULL, zbp4, lane + zdx);
                        const T g6 = __shfl_sync(FULL, gg6, lane + gdx), g4 = __shfl_sync(FULL, gg4, lane + gdx);
                        zv = pick_row(zdy, z6, zv, z4);
                        gv = pick_row(gdy, g6, gv, g4);
                    }
                    if (flags & 8u) zfin = zv;
                    if (flags & 16u) gfin = gv;
                }
            }
            if (rowG && p >= R0 && p < R1 && out_col) {
                const unsigned i = (unsigned)p * upitch + (unsigned)c;
                if (AVG) {
                    if (ASYNC_PARTNER) {
                        pazb = pb[r & 1][3][lane];
                        if (a.oG) paG = pb[r & 1][4][lane];
                    }
                    zfin = T(0.5) * pazb + T(0.5) * zfin;
                    if (a.oG) gfin = T(0.5) * paG + T(0.5) * gfin;
                }
                a.ozb[i] = zfin;
                if (a.oG) a.oG[i] = gfin;
                bad |= !d_isfinite(zfin);
            }
            if (rowD && q >= R0 && q < R1 && out_col) {
                const unsigned i = (unsigned)q * upitch + (unsigned)c;
                T oh = sbh, ou = sbu, ov = sbv;
                if (AVG) {
                    if (ASYNC_PARTNER) {
                        pah = pb[r & 1][0][lane];
                        pahu = pb[r & 1][1][lane];
                        pahv = pb[r & 1][2][lane];
                    }
                    oh = T(0.5) * pah + T(0.5) * oh;
                    ou = T(0.5) * pahu + T(0.5) * ou;
                    ov = T(0.5) * pahv + T(0.5) * ov;
                }
                a.oh[i] = oh;
                a.ohu[i] = ou;
                a.ohv[i] = ov;
                bad |= !(d_isfinite(oh) && d_isfinite(ou) && d_isfinite(ov));
            }

            // ================= shift the windows
            pA = pr; hA = h_r; huA = hu_r; hvA = hv_r;
            xfA0 = xf0; xfA1 = xf1; xfA2 = xf2;
            nfA0 = yP[0]; nfA1 = yP[1]; nfA2 = yP[2];
            zt3 = zt2; zt2 = ztA; ztA = zt_r;
            hr3 = hr2; hr2 = hr1; hur2 = hur1; hvr2 = hvr1;
            mwin = (mwin << 1) | (m_r ? 1u : 0u);
            zin4 = zin3; zin3 = zin2; zin2 = zin1; zin1 = zb_r;
            if (!MPM) { gin4 = gin3; gin3 = gin2; gin2 = gin1; gin1 = g_r; }
            hf4h = hf3h; hf4u = hf3u; hf4v = hf3v;
            hf3h = hf2h; hf3u = hf2u; hf3v = hf2v;
            e4 = e3; xe4 = xe3; fn4 = Fy;
            zbp6 = zbp5; zbp5 = zbp4;
            gg6 = gg5; gg5 = gg4;
        };
        const int steady0 = min(L0 + 5, L1), steady1 = L1;
        int r = L0;
        for (; r < steady0; ++r) iterate(r, std::false_type{});
        PXB_UNROLL(PXB_STAGE_UNROLL)
        for (; r < steady1; ++r) iterate(r, std::true_type{});
        for (; r < L1 + 5; ++r) iterate(r, std::false_type{});
        cp_async_wait<0>();  // the buffers are reused by the next item
    }
}

// The grid is sized to the resident capacity of the device.  A warp's first item is its
// warp index; further items come from a grid-wide queue (one atomic per item), so warps
// on lightly loaded SMs take more of them and no SM waits on a fixed share.  The last
// block to finish resets the queue for the next launch on the stream.
template <class T, bool MPM, bool HAS_MASK, bool AVG>
__global__ void __launch_bounds__(128, PXB_STAGE_BOUNDS(T, AVG)) re_stage_kernel(const REStageArgs<T> a) {
    const int lane = threadIdx.x & 31;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    const int nitems = pxb_stage_items_per_band(a.nstrips) * a.nbands;
    bool bad = false;
    int item = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    while (item < nitems) {
        re_stage_item<T, MPM, HAS_MASK, AVG>(a, item, bad);
        unsigned next = 0;
        if (lane == 0) next = atomicAdd(&a.queue[0], 1u);
        item = nw + (int)__shfl_sync(FULL, next, 0);
    }
    if (bad) atomicOr(a.err, 1);
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(&a.queue[1], 1u) == gridDim.x - 1) {
            atomicExch(&a.queue[0], 0u);
            atomicExch(&a.queue[1], 0u);
        }
    }
}

}  // namespace pxb
