// Fused Roe-Exner stage kernel (one launch per Runge-Kutta stage).
//
// Replaces step_fn_roeexner (PyExner src/PyExner/solvers/roe_exner_solver.py:80-116) on
// one rank: hydro update (roe_exner.py:535-612) -> momentum corrections (:14-62) ->
// boundary handlers -> grass factor (:85-140) -> Exner update (:665-717) -> boundary
// handlers, and for the second SSPRK2 stage the 0.5/0.5 combination (SSPRK2.py:40).
//
// Layout of the work: a warp owns a strip of 32 x CPT columns (3 halo | owned | 3 halo;
// CPT consecutive columns per lane, one by default, two as a float32 build knob) and
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
// Warp votes skip work whose result is known for the whole warp: the entropy-fix terms
// without a transonic face, the momentum corrections where every cell is wet, the Exner
// block where no cell of the two rows carries sediment (see the phases below).
#pragma once
#include <type_traits>

#include "pxb_device.cuh"

// Resident 128-thread blocks per SM the float32 build is register-limited to, for the
// plain stage and the averaging second SSPRK2 stage (tuning knobs, measured on the
// 2048^2 and 8192^2 Gaussian-bed cases): 4 (128 registers, no spills) with one column
// per lane; 5 (96 registers) is 1% faster at 8192^2 and 4% slower at 2048^2, where fewer
// resident warps mean taller bands and fewer redundant halo rows.  With two columns per
// lane the state needs about 200 registers: 3 blocks (168, some spills) or 2.
#ifndef PXB_STAGE_MIN_BLOCKS
#define PXB_STAGE_MIN_BLOCKS (PXB_STAGE_CPT_F32 == 2 ? 3 : 4)
#endif
#ifndef PXB_STAGE_MIN_BLOCKS_AVG
#define PXB_STAGE_MIN_BLOCKS_AVG (PXB_STAGE_CPT_F32 == 2 ? 3 : 4)
#endif
// float64 state (twice the registers per value): 3 blocks (168 registers, a few hundred
// bytes of spills) measured 12 % faster than 5 (96 registers, 2.8 KB of spills) and than
// 2 (no spills, too few warps) at 2048^2
#ifndef PXB_STAGE_MIN_BLOCKS_F64
#define PXB_STAGE_MIN_BLOCKS_F64 3
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
    // Volume budget (null: off): per work item, the outflow through the outer boundary of
    // the physical cells (rows and columns 1 .. n-2) of water (sum of the mass fluxes of
    // the boundary faces) and of sediment (Exner fluxes), in the state's flux units; item
    // k writes bud[2k], bud[2k+1] on every launch.
    double* bud;
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
// cp.async of 16 bytes with zero fill: the first src_bytes (0-16) bytes are read, the
// rest of the 16 is set to zero; with src_bytes = 0 nothing is read.
__device__ __forceinline__ void cp_async16_zfill(unsigned smem, const void* gmem, unsigned src_bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(smem), "l"(gmem), "r"(src_bytes) : "memory");
}
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

// Donor values of the boundary passes for the CPT columns of this lane: column k takes
// the value at (row q+dy[k], column +dxo[k]) with dy, dxo in [-1, 1].  The candidates
// are this lane's own columns and the last column of the west lane / first column of
// the east lane (one shuffle each); the row is chosen by the receiver.  Donors lie in
// another row only for cells of the first and last rows (plan creation checks it), so
// elsewhere (dyrow false) only the middle row is fetched.
template <int CPT, class T>
__device__ __forceinline__ T pick_col(const T (&cand)[CPT + 2], int s) {
    T v = cand[0];
#pragma unroll
    for (int t = 1; t < CPT + 2; ++t) v = (s == t) ? cand[t] : v;
    return v;
}

template <int CPT, class T>
__device__ __forceinline__ void donor_candidates(const T (&x)[CPT], T (&cd)[CPT + 2]) {
    cd[0] = __shfl_up_sync(FULL, x[CPT - 1], 1);
#pragma unroll
    for (int k = 0; k < CPT; ++k) cd[k + 1] = x[k];
    cd[CPT + 1] = __shfl_down_sync(FULL, x[0], 1);
}

template <int CPT, class T>
__device__ __forceinline__ void fetch_donor(bool dyrow, const int (&dy)[CPT], const int (&dxo)[CPT],
                                            const T (&above)[CPT], const T (&mid)[CPT], const T (&below)[CPT],
                                            T (&out)[CPT]) {
    T cm[CPT + 2];
    donor_candidates<CPT>(mid, cm);
    if (!dyrow) {
#pragma unroll
        for (int k = 0; k < CPT; ++k) out[k] = pick_col<CPT>(cm, k + dxo[k] + 1);
        return;
    }
    T ca[CPT + 2], cbl[CPT + 2];
    donor_candidates<CPT>(above, ca);
    donor_candidates<CPT>(below, cbl);
#pragma unroll
    for (int k = 0; k < CPT; ++k) {
        const int s = k + dxo[k] + 1;
        out[k] = pick_row(dy[k], pick_col<CPT>(ca, s), pick_col<CPT>(cm, s), pick_col<CPT>(cbl, s));
    }
}

// CPT consecutive elements of a shared row buffer laid out by column (lane * CPT + k).
template <int CPT, class T>
__device__ __forceinline__ void read_cols(const T* rowp, int lane, T (&v)[CPT]) {
    if constexpr (CPT == 2 && sizeof(T) == 4) {
        const float2 t = *reinterpret_cast<const float2*>(rowp + 2 * lane);
        v[0] = t.x;
        v[1] = t.y;
    } else {
#pragma unroll
        for (int k = 0; k < CPT; ++k) v[k] = rowp[CPT * lane + k];
    }
}

// One work item (a strip of one band) of a stage; the single-grid kernel and the
// ensemble kernel (ens.cuh) both loop over items and call this.  Each lane owns CPT
// consecutive columns (pxb_stage_cpt): a strip is 32 * CPT columns, 3 halo | owned | 3
// halo.  Neighbour values inside a lane are plain registers; across lanes one shuffle
// moves the first (east) or last (west) column.
// A block's shared buffer of the stage kernel (TAG: 0 row copies, 1 partner copies),
// one object for every instantiation of re_stage_item with these dimensions, so that
// the interior and the boundary instantiations in one kernel share it.
template <class T, int TAG, int D0, int D1, int D2, int D3>
__device__ __forceinline__ T (&stage_smem())[D0][D1][D2][D3] {
    __shared__ __align__(16) T buf[D0][D1][D2][D3];
    return buf;
}

// INTERIOR: the instantiation for items away from the grid's boundary (no boundary strip
// or row), which carries none of the boundary-recipe code.
template <class T, bool MPM, bool HAS_MASK, bool AVG, bool BUD = false, bool INTERIOR = false>
__device__ __forceinline__ void re_stage_item(const REStageArgs<T>& a, const int item, bool& bad) {
    constexpr int CPT = pxb_stage_cpt((int)sizeof(T));
    constexpr int W = 32 * CPT;
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
        const int kb = item - band * ipb;
        int strip = kb - 1, half = -1;  // half: 0 / 1 = upper / lower half of a boundary strip
        if (ipb == 1) strip = 0;
        else if (kb < 2) { strip = 0; half = kb; }
        else if (kb >= a.nstrips) { strip = a.nstrips - 1; half = kb - a.nstrips; }
        const bool last_strip = !INTERIOR && strip == a.nstrips - 1;
        const int cb = strip * (W - 2 * PXB_HALO) - PXB_HALO + CPT * lane;  // column of this lane's first element
        bool colok[CPT], has_e[CPT], out_col[CPT], interior_col[CPT];
#pragma unroll
        for (int k = 0; k < CPT; ++k) {
            const int c = cb + k, j = CPT * lane + k;
            // an interior strip lies inside the grid's columns 1 .. nx-2 (it is neither the
            // first nor the last strip, and every strip but the last ends two columns
            // short of column nx - 1)
            colok[k] = INTERIOR || ((c >= 0) && (c < nx));
            has_e[k] = colok[k] && (INTERIOR || c + 1 < nx) && (j < W - 1);
            out_col[k] = colok[k] && j >= PXB_HALO && (j < W - PXB_HALO || last_strip);
            interior_col[k] = INTERIOR || ((c >= 1) && (c <= nx - 2));
        }
        const int B0 = band * a.band_rows;
        const int B1 = (band == a.nbands - 1) ? ny : B0 + a.band_rows;
        const int Bm = B0 + (B1 - B0 + 1) / 2;
        const int R0 = half == 1 ? Bm : B0;
        const int R1 = half == 0 ? Bm : B1;
        const int L0 = max(0, R0 - 3), L1 = min(ny, R1 + 3);
        // boundary recipes can only apply in the first/last strip or on rows 0 / ny-1
        const bool bc_strip = !INTERIOR && (a.ring != nullptr) && (strip == 0 || last_strip);
        const bool bc_rows = !INTERIOR && (a.ring != nullptr) && (R0 == 0 || R1 == ny);
        // Budget: only items that own boundary faces of physical cells add to the lane slots.
        // A face counts once: in the item that owns its row (x-faces; y-faces (r-1|r) by row
        // r) and, for columns, by the lane that owns the column.  The outflow of a face with
        // left cell I (west / north side) is F = h_I u_n,I + upwM_0, the flux whose
        // differences the fluctuations of roe_exner.py:597-606 telescope to; F leaves the
        // physical cells through the east / south boundary and enters them through the west
        // / north one.  Exner: the upwind face flux of roe_exner.py:708-715.
        // (BUD: the budget instantiation, launched only when a.bud is set)
        __shared__ double budbuf[4][BUD ? 2 : 1][BUD ? 32 : 1];
        const bool bud_item = BUD && (bc_strip || bc_rows);
        if constexpr (BUD) {
            budbuf[threadIdx.x >> 5][0][lane] = 0.0;
            budbuf[threadIdx.x >> 5][1][lane] = 0.0;
        }

        // ---- carried pipeline state, per column
        HCell<T> pA[CPT];
        T hA[CPT], huA[CPT], hvA[CPT], ztA[CPT];
        T xfA[CPT][3], nfA[CPT][3];
        T hr3[CPT], hr2[CPT], hur2[CPT], hvr2[CPT], zt3[CPT], zt2[CPT];
        unsigned mwin[CPT];  // bit i = nodata of row r-1-i
        T zin1[CPT], zin2[CPT], zin3[CPT], zin4[CPT];
        T gin1[CPT], gin2[CPT], gin3[CPT], gin4[CPT];
        T hf4h[CPT], hf4u[CPT], hf4v[CPT], hf3h[CPT], hf3u[CPT], hf3v[CPT];
        ECell<T> e4[CPT];
        T xe4[CPT], fn4[CPT];
        T zbp6[CPT], zbp5[CPT], gg6[CPT], gg5[CPT];
#pragma unroll
        for (int k = 0; k < CPT; ++k) {
            pA[k] = make_hcell(T(0), T(0), T(0), T(0), T(0), T(0));
            hA[k] = huA[k] = hvA[k] = ztA[k] = T(0);
#pragma unroll
            for (int m = 0; m < 3; ++m) xfA[k][m] = nfA[k][m] = T(0);
            hr3[k] = hr2[k] = hur2[k] = hvr2[k] = zt3[k] = zt2[k] = T(0);
            mwin[k] = 0u;
            zin1[k] = zin2[k] = zin3[k] = zin4[k] = T(0);
            gin1[k] = gin2[k] = gin3[k] = gin4[k] = T(0);
            hf4h[k] = hf4u[k] = hf4v[k] = hf3h[k] = hf3u[k] = hf3v[k] = T(0);
            e4[k] = make_ecell(T(0), T(0), T(0), T(0), T(0));
            xe4[k] = fn4[k] = T(0);
            zbp6[k] = zbp5[k] = gg6[k] = gg5[k] = T(0);
        }

        // Row r+1 is fetched while row r is computed: the loads of one iteration are in
        // flight during the ~thousand instructions of the previous one.  In float32 they
        // are cp.async copies into this warp's shared buffer (no registers held); in
        // float64 (measured: faster there) plain loads into registers.
        constexpr bool ASYNC_ROWS = is_f32<T>();
        constexpr int NP = MPM ? 6 : 7;
        auto& rbuf = stage_smem<T, 0, 4, ASYNC_ROWS ? 2 : 1, ASYNC_ROWS ? NP : 1, ASYNC_ROWS ? W : 1>();
        T(*rb)[ASYNC_ROWS ? NP : 1][ASYNC_ROWS ? W : 1] = rbuf[threadIdx.x >> 5];
        T nh[CPT], nhu[CPT], nhv[CPT], nzb[CPT], nz[CPT], nnb[CPT], ng[CPT];
        bool nm[CPT];
#pragma unroll
        for (int k = 0; k < CPT; ++k) {
            nh[k] = nhu[k] = nhv[k] = nzb[k] = nz[k] = nnb[k] = ng[k] = T(0);
            nm[k] = false;
        }
        auto load_row = [&](int rr) __attribute__((always_inline)) {
            const int b = rr & 1;
#pragma unroll
            for (int k = 0; k < CPT; ++k) {
                const bool ok = rr < L1 && colok[k];
                const unsigned i = (unsigned)rr * upitch + (unsigned)(cb + k);
                if constexpr (!ASYNC_ROWS) {
                    if (ok) {
                        nh[k] = __ldg(a.h + i);
                        nhu[k] = __ldg(a.hu + i);
                        nhv[k] = __ldg(a.hv + i);
                        nzb[k] = __ldg(a.zb + i);
                        nz[k] = __ldg(a.z + i);
                        nnb[k] = __ldg(a.nb + i);
                        if (!MPM) ng[k] = __ldg(a.G + i);
                        if (HAS_MASK) nm[k] = __ldg(a.nodata + i) != 0;
                    } else {
                        nh[k] = nhu[k] = nhv[k] = nzb[k] = nz[k] = nnb[k] = ng[k] = T(0);
                        nm[k] = false;
                    }
                } else {
                    const int e = CPT * lane + k;
                    if (ok) {
                        cp_async_elem(&rb[b][0][e], a.h + i);
                        cp_async_elem(&rb[b][1][e], a.hu + i);
                        cp_async_elem(&rb[b][2][e], a.hv + i);
                        cp_async_elem(&rb[b][3][e], a.zb + i);
                        cp_async_elem(&rb[b][4][e], a.z + i);
                        cp_async_elem(&rb[b][5][e], a.nb + i);
                        if constexpr (!MPM) cp_async_elem(&rb[b][NP - 1][e], a.G + i);
                        if (HAS_MASK) nm[k] = __ldg(a.nodata + i) != 0;
                    } else {
#pragma unroll
                        for (int pl = 0; pl < NP; ++pl) rb[b][pl][e] = T(0);
                        nm[k] = false;
                    }
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
        auto& pbuf = stage_smem<T, 1, 4, ASYNC_PARTNER ? 2 : 1, 5, ASYNC_PARTNER ? W : 1>();
        T(*pb)[5][ASYNC_PARTNER ? W : 1] = pbuf[threadIdx.x >> 5];
        auto partner_copy = [&](const int rr) __attribute__((always_inline)) {  // the rows stored in iteration rr
            const int q0 = rr - 3, p0 = rr - 5;
            const int b = rr & 1;
#pragma unroll
            for (int k = 0; k < CPT; ++k) {
                const int e = CPT * lane + k;
                if (q0 >= L0 && q0 < L1 && q0 >= R0 && q0 < R1 && out_col[k]) {
                    const unsigned i = (unsigned)q0 * upitch + (unsigned)(cb + k);
                    cp_async_elem(&pb[b][0][e], a.ah + i);
                    cp_async_elem(&pb[b][1][e], a.ahu + i);
                    cp_async_elem(&pb[b][2][e], a.ahv + i);
                }
                if (p0 >= L0 && p0 < L1 && p0 >= R0 && p0 < R1 && out_col[k]) {
                    const unsigned i = (unsigned)p0 * upitch + (unsigned)(cb + k);
                    cp_async_elem(&pb[b][3][e], a.azb + i);
                    if (a.oG) cp_async_elem(&pb[b][4][e], a.aG + i);
                }
            }
        };
        if constexpr (ASYNC_PARTNER) partner_copy(L0);
        cp_async_commit();
        // Boundary recipes of the side columns (first / last strip, rows other than the
        // first and last): the recipe of the ring cell of the row that the first boundary
        // application treats in iteration r (q = r-3) is copied into this warp's shared
        // buffer during iteration r-1 (one slot per side), so no recipe load is waited on
        // inside the pipeline; the first and last rows, where every column is a ring cell,
        // read theirs directly.  The first application leaves the z_b / G fields of the
        // second (row p = r-5, two iterations later) in a packed word.  Float32 only, as
        // the row copies.
        constexpr bool ASYNC_RECIPES = ASYNC_ROWS && !INTERIOR;
        __shared__ __align__(16) pxb_ring_recipe rcbuf[4][ASYNC_RECIPES ? 2 : 1][2];
        __shared__ unsigned zgbuf[4][ASYNC_RECIPES ? 4 : 1][ASYNC_RECIPES ? W : 1];
        pxb_ring_recipe(*rcb)[2] = rcbuf[threadIdx.x >> 5];
        unsigned(*zgb)[ASYNC_RECIPES ? W : 1] = zgbuf[threadIdx.x >> 5];
        auto recipe_copy = [&](const int rr) __attribute__((always_inline)) {  // the recipes used in iteration rr
            const int qn = rr - 3;
            if (bc_strip && qn >= L0 && qn < L1 && qn != 0 && qn != ny - 1) {
#pragma unroll
                for (int k = 0; k < CPT; ++k) {
                    const int c = cb + k;
                    if (c == 0 || c == nx - 1) {
                        const char* src = reinterpret_cast<const char*>(a.ring + ring_slot(qn, c, ny, nx));
                        char* dst = reinterpret_cast<char*>(&rcb[rr & 1][c == 0 ? 0 : 1]);
                        cp_async16(dst, src);
                        cp_async16(dst + 16, src + 16);
                        cp_async16(dst + 32, src + 32);
                    }
                }
            }
        };

        // One pipeline iteration.  In the steady state (rows L0+5 .. L1-1) every phase has
        // valid rows, so the row checks compile away.
        auto iterate = [&](const int r, auto steady_tag) __attribute__((always_inline)) {
            constexpr bool S = decltype(steady_tag)::value;
            const bool rowA = S || r < L1;
            // ================= A: row r (prefetched), x-faces of row r, y-face (r-1 | r)
            T h_r[CPT], hu_r[CPT], hv_r[CPT], zb_r[CPT], z_r[CPT], nb_r[CPT], g_r[CPT];
            if constexpr (ASYNC_ROWS) {
                cp_async_wait<0>();  // row r (and the partner rows stored in this iteration)
                const int rbb = r & 1;
                read_cols<CPT>(rb[rbb][0], lane, h_r);
                read_cols<CPT>(rb[rbb][1], lane, hu_r);
                read_cols<CPT>(rb[rbb][2], lane, hv_r);
                read_cols<CPT>(rb[rbb][3], lane, zb_r);
                read_cols<CPT>(rb[rbb][4], lane, z_r);
                read_cols<CPT>(rb[rbb][5], lane, nb_r);
                if constexpr (!MPM) {
                    read_cols<CPT>(rb[rbb][NP - 1], lane, g_r);
                } else {
#pragma unroll
                    for (int k = 0; k < CPT; ++k) g_r[k] = T(0);
                }
            } else {
#pragma unroll
                for (int k = 0; k < CPT; ++k) {
                    h_r[k] = nh[k], hu_r[k] = nhu[k], hv_r[k] = nhv[k], zb_r[k] = nzb[k];
                    z_r[k] = nz[k], nb_r[k] = nnb[k], g_r[k] = ng[k];
                }
            }
            bool m_r[CPT];
#pragma unroll
            for (int k = 0; k < CPT; ++k) m_r[k] = nm[k];
            load_row(r + 1);
            if constexpr (ASYNC_PARTNER) partner_copy(r + 1);
            if constexpr (ASYNC_RECIPES) recipe_copy(r + 1);
            cp_async_commit();
            T pah[CPT], pahu[CPT], pahv[CPT], pazb[CPT], paG[CPT];
#pragma unroll
            for (int k = 0; k < CPT; ++k) pah[k] = pahu[k] = pahv[k] = pazb[k] = paG[k] = T(0);
            if constexpr (!ASYNC_PARTNER && AVG) {
                const int q0 = r - 3, p0 = r - 5;
#pragma unroll
                for (int k = 0; k < CPT; ++k) {
                    if ((S || (q0 >= L0 && q0 < L1)) && q0 >= R0 && q0 < R1 && out_col[k]) {
                        const unsigned i = (unsigned)q0 * upitch + (unsigned)(cb + k);
                        pah[k] = a.ah[i];
                        pahu[k] = a.ahu[i];
                        pahv[k] = a.ahv[i];
                    }
                    if ((S || (p0 >= L0 && p0 < L1)) && p0 >= R0 && p0 < R1 && out_col[k]) {
                        const unsigned i = (unsigned)p0 * upitch + (unsigned)(cb + k);
                        pazb[k] = a.azb[i];
                        if (a.oG) paG[k] = a.aG[i];
                    }
                }
            }
            HCell<T> pr[CPT];
            T zt_r[CPT];
#pragma unroll
            for (int k = 0; k < CPT; ++k) {
                pr[k] = make_hcell(h_r[k], hu_r[k], hv_r[k], zb_r[k], z_r[k], nb_r[k]);
                zt_r[k] = z_r[k] + zb_r[k];
            }
            T xf[CPT][3];
#pragma unroll
            for (int k = 0; k < CPT; ++k) xf[k][0] = xf[k][1] = xf[k][2] = T(0);
            // In the prologue / drain iterations of a band the faces of invalid rows are
            // skipped for the whole warp (r is warp-uniform); their results would be masked.
            if (S || rowA) {
                HCell<T> pe[CPT];
                bool me[CPT];
#pragma unroll
                for (int k = 0; k + 1 < CPT; ++k) { pe[k] = pr[k + 1]; me[k] = m_r[k + 1]; }
                pe[CPT - 1] = shfl_down_hcell(pr[0]);
                me[CPT - 1] = HAS_MASK ? (__shfl_down_sync(FULL, (int)m_r[0], 1) != 0) : false;
                T P[CPT][3], M[CPT][3];
                bool xact[CPT];
#pragma unroll
                for (int k = 0; k < CPT; ++k) {
                    // pr.h = max(h, DRY_TOL) > DRY_TOL exactly when h > DRY_TOL (false for NaN)
                    xact[k] = rowA && has_e[k] && ((pr[k].h > DRY) || (pe[k].h > DRY)) && !(m_r[k] || me[k]);
                    roe_exner_face<T, false>(pr[k], pe[k], dx, P[k], M[k]);
#pragma unroll
                    for (int m = 0; m < 3; ++m) {
                        P[k][m] = xact[k] ? P[k][m] : T(0);
                        M[k][m] = xact[k] ? M[k][m] : T(0);
                    }
                    if (bud_item && xact[k] && out_col[k] && r >= R0 && r < R1 && r >= 1 && r <= ny - 2 &&
                        (cb + k == 0 || cb + k == nx - 2)) {
                        const double F = (double)mul_rn(pr[k].h, pr[k].u) + (double)M[k][0];
                        if constexpr (BUD) budbuf[threadIdx.x >> 5][0][lane] += cb + k == 0 ? -F : F;
                    }
                }
                // upwP of the west face of column k: own column k-1, or the west lane's last
                // (lane 0 has no west face in the warp).  P and M are zero on inactive faces,
                // and the sums start at +0, so adding them unconditionally gives the same bits
                // as adding only the active ones.
                T wP[CPT][3];
#pragma unroll
                for (int k = 1; k < CPT; ++k)
#pragma unroll
                    for (int m = 0; m < 3; ++m) wP[k][m] = P[k - 1][m];
#pragma unroll
                for (int m = 0; m < 3; ++m) {
                    const T w = __shfl_up_sync(FULL, P[CPT - 1][m], 1);
                    wP[0][m] = lane > 0 ? w : T(0);
                }
                // scatter order of roe_exner.py:599-600: east upwM first, then west upwP
#pragma unroll
                for (int k = 0; k < CPT; ++k) {
#pragma unroll
                    for (int m = 0; m < 3; ++m) xf[k][m] = (xf[k][m] + M[k][m]) + wP[k][m];
                }
            }
            T yP[CPT][3], yM[CPT][3];
#pragma unroll
            for (int k = 0; k < CPT; ++k)
#pragma unroll
                for (int m = 0; m < 3; ++m) yP[k][m] = yM[k][m] = T(0);
            if (S || (rowA && r - 1 >= L0)) {
#pragma unroll
                for (int k = 0; k < CPT; ++k) {
                    const bool yact = rowA && (S || r - 1 >= L0) && colok[k] && ((hA[k] > DRY) || (h_r[k] > DRY)) &&
                                      !((mwin[k] & 1u) || m_r[k]);
                    roe_exner_face<T, true>(pA[k], pr[k], dx, yP[k], yM[k]);
#pragma unroll
                    for (int m = 0; m < 3; ++m) {
                        yP[k][m] = yact ? yP[k][m] : T(0);
                        yM[k][m] = yact ? yM[k][m] : T(0);
                    }
                    if (bud_item && (r == 1 || r == ny - 1) && r >= R0 && r < R1) {
                        const int c = cb + k;
                        if (out_col[k] && yact && c >= 1 && c <= nx - 2) {
                            // y-faces have the normal (0, -1): u_n = -v
                            const double F = -(double)mul_rn(pA[k].h, pA[k].v) + (double)yM[k][0];
                            if constexpr (BUD) budbuf[threadIdx.x >> 5][0][lane] += r == 1 ? -F : F;
                        }
                    }
                }
            }

            // ================= B: hydro update of row r-1
            T hr1[CPT], hur1[CPT], hvr1[CPT];
#pragma unroll
            for (int k = 0; k < CPT; ++k) {
                hr1[k] = hur1[k] = hvr1[k] = T(0);
                if (S || (r - 1 >= L0 && r - 1 < L1)) {
                    T f0 = xfA[k][0], f1 = xfA[k][1], f2 = xfA[k][2];
                    f0 = f0 + yM[k][0]; f1 = f1 + yM[k][1]; f2 = f2 + yM[k][2];    // south face upwM
                    f0 = f0 + nfA[k][0]; f1 = f1 + nfA[k][1]; f2 = f2 + nfA[k][2];  // north face upwP
                    if constexpr (is_f32<T>()) {
                        hr1[k] = hA[k] - dtdx * f0;
                        hur1[k] = huA[k] - dtdx * f1;
                        hvr1[k] = hvA[k] - dtdx * f2;
                    } else {
                        hr1[k] = hA[k] - dt * f0 / dx;
                        hur1[k] = huA[k] - dt * f1 / dx;
                        hvr1[k] = hvA[k] - dt * f2 / dx;
                    }
                }
            }

            // ================= C: momentum corrections of row r-2
            T hf2h[CPT], hf2u[CPT], hf2v[CPT];
            // Where every cell of the warp is wet and its north / south neighbours are not
            // dry (no nodata mask), no correction applies: a warp vote skips the tests and
            // their shuffles.  Exact: NaN depths fail the vote, as they fail `active`.
            bool allwet = false;
            if constexpr (!HAS_MASK) {
                bool dry = false;
#pragma unroll
                for (int k = 0; k < CPT; ++k)
                    dry = dry || (colok[k] && (!(hr2[k] > DRY) || (hr3[k] < DRY) || (hr1[k] < DRY)));
                allwet = !__any_sync(FULL, dry);
            }
            if (allwet) {
#pragma unroll
                for (int k = 0; k < CPT; ++k) {
                    const bool ok = S || (r - 2 >= L0 && r - 2 < L1);
                    hf2h[k] = ok ? hr2[k] : T(0);
                    hf2u[k] = ok ? hur2[k] : T(0);
                    hf2v[k] = ok ? hvr2[k] : T(0);
                }
            } else {
                const int q2 = r - 2;
                T hE[CPT], hW[CPT], zE[CPT], zW[CPT];
                bool m2[CPT], mE[CPT], mW[CPT];
#pragma unroll
                for (int k = 0; k < CPT; ++k) m2[k] = HAS_MASK && ((mwin[k] >> 1) & 1u);
#pragma unroll
                for (int k = 0; k + 1 < CPT; ++k) { hE[k] = hr2[k + 1]; zE[k] = zt2[k + 1]; mE[k] = m2[k + 1]; }
#pragma unroll
                for (int k = 1; k < CPT; ++k) { hW[k] = hr2[k - 1]; zW[k] = zt2[k - 1]; mW[k] = m2[k - 1]; }
                hE[CPT - 1] = __shfl_down_sync(FULL, hr2[0], 1);
                zE[CPT - 1] = __shfl_down_sync(FULL, zt2[0], 1);
                hW[0] = __shfl_up_sync(FULL, hr2[CPT - 1], 1);
                zW[0] = __shfl_up_sync(FULL, zt2[CPT - 1], 1);
                mE[CPT - 1] = HAS_MASK ? (__shfl_down_sync(FULL, (int)m2[0], 1) != 0) : false;
                mW[0] = HAS_MASK ? (__shfl_up_sync(FULL, (int)m2[CPT - 1], 1) != 0) : false;
#pragma unroll
                for (int k = 0; k < CPT; ++k) {
                    hf2h[k] = hf2u[k] = hf2v[k] = T(0);
                    if (S || (q2 >= L0 && q2 < L1)) {
                        hf2h[k] = hr2[k];
                        hf2u[k] = hur2[k];
                        hf2v[k] = hvr2[k];
                        if (interior_col[k] && q2 >= 1 && q2 <= ny - 2) {
                            const bool mN = HAS_MASK && ((mwin[k] >> 2) & 1u);
                            const bool mS = HAS_MASK && (mwin[k] & 1u);
                            const T eta = hr2[k] + zt2[k];
                            const bool stop_u = ((eta < zE[k]) && (hE[k] < DRY)) || ((eta < zW[k]) && (hW[k] < DRY)) || mE[k] || mW[k];
                            const bool stop_v = ((eta < zt3[k]) && (hr3[k] < DRY)) || ((eta < ztA[k]) && (hr1[k] < DRY)) || mN || mS;
                            const bool active = (hr2[k] > DRY) && !m2[k];
                            hf2u[k] = (active && !stop_u) ? hur2[k] : T(0);
                            hf2v[k] = (active && !stop_v) ? hvr2[k] : T(0);
                        }
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
            T hbh[CPT], hbu[CPT], hbv[CPT], zb1[CPT], gb1[CPT], sbh[CPT], sbu[CPT], sbv[CPT];
#pragma unroll
            for (int k = 0; k < CPT; ++k) {
                hbh[k] = sbh[k] = hf3h[k];
                hbu[k] = sbu[k] = hf3u[k];
                hbv[k] = sbv[k] = hf3v[k];
                zb1[k] = zin3[k];
                gb1[k] = gin3[k];
            }
            if (rowD && (bc_strip || (bc_rows && (q == 0 || q == ny - 1)))) {
                unsigned flags[CPT];
                int hdy[CPT], hdx[CPT], mdy[CPT], mdx[CPT], zdy[CPT], zdx[CPT], gdy[CPT], gdx[CPT];
                T m0[CPT], m1[CPT], m2c[CPT], m3[CPT];
                bool anyf = false;
#pragma unroll
                for (int k = 0; k < CPT; ++k) {
                    flags[k] = 0u;
                    hdy[k] = hdx[k] = mdy[k] = mdx[k] = zdy[k] = zdx[k] = gdy[k] = gdx[k] = 0;
                    m0[k] = m1[k] = m2c[k] = m3[k] = T(0);
                    auto take = [&](const pxb_ring_recipe& rc) __attribute__((always_inline)) {
                        flags[k] = rc.flags;
                        hdy[k] = rc.h_dy; hdx[k] = rc.h_dx; mdy[k] = rc.m_dy; mdx[k] = rc.m_dx;
                        zdy[k] = rc.zb_dy; zdx[k] = rc.zb_dx; gdy[k] = rc.g_dy; gdx[k] = rc.g_dx;
                        m0[k] = T(rc.m[0]); m1[k] = T(rc.m[1]); m2c[k] = T(rc.m[2]); m3[k] = T(rc.m[3]);
                    };
                    const int c = cb + k;
                    bool direct = true;
                    if constexpr (ASYNC_RECIPES) {
                        if (q != 0 && q != ny - 1) {  // side rows: the ring column's recipe, copied in iteration r-1
                            direct = false;
                            if (c == 0 || c == nx - 1) take(rcb[r & 1][c == 0 ? 0 : 1]);
                        }
                    }
                    if (direct) {
                        const int slot = colok[k] ? ring_slot(q, c, ny, nx) : -1;
                        if (slot >= 0) take(a.ring[slot]);
                    }
                    if constexpr (ASYNC_RECIPES) zgb[r & 3][CPT * lane + k] = pack_zg(flags[k], zdy[k], zdx[k], gdy[k], gdx[k]);
                    anyf = anyf || (flags[k] != 0u);
                }
                if (__any_sync(FULL, anyf)) {
                    const bool dyrow = (q == 0) || (q == ny - 1);
                    T vh[CPT], vu[CPT], vv[CPT], vz[CPT];
                    fetch_donor<CPT>(dyrow, hdy, hdx, hf4h, hf3h, hf2h, vh);
                    fetch_donor<CPT>(dyrow, mdy, mdx, hf4u, hf3u, hf2u, vu);
                    fetch_donor<CPT>(dyrow, mdy, mdx, hf4v, hf3v, hf2v, vv);
                    fetch_donor<CPT>(dyrow, zdy, zdx, zin4, zin3, zin2, vz);
#pragma unroll
                    for (int k = 0; k < CPT; ++k) {
                        if (flags[k] & 1u) hbh[k] = vh[k];
                        if (flags[k] & 2u) {
                            if (flags[k] & 4u) { hbu[k] = m0[k]; hbv[k] = m1[k]; }
                            else { hbu[k] = sum2(m0[k], vu[k], m1[k], vv[k]); hbv[k] = sum2(m2c[k], vu[k], m3[k], vv[k]); }
                        }
                        if (flags[k] & 8u) zb1[k] = vz[k];
                    }
                    if (!MPM) {
                        T vg[CPT];
                        fetch_donor<CPT>(dyrow, gdy, gdx, gin4, gin3, gin2, vg);
#pragma unroll
                        for (int k = 0; k < CPT; ++k)
                            if (flags[k] & 16u) gb1[k] = vg[k];
                    }
                    // second pass
                    T wh[CPT], wu[CPT], wv[CPT];
                    fetch_donor<CPT>(dyrow, hdy, hdx, hf4h, hbh, hf2h, wh);
                    fetch_donor<CPT>(dyrow, mdy, mdx, hf4u, hbu, hf2u, wu);
                    fetch_donor<CPT>(dyrow, mdy, mdx, hf4v, hbv, hf2v, wv);
#pragma unroll
                    for (int k = 0; k < CPT; ++k) {
                        sbh[k] = hbh[k];
                        sbu[k] = hbu[k];
                        sbv[k] = hbv[k];
                        if (flags[k] & 1u) sbh[k] = wh[k];
                        if ((flags[k] & 2u) && !(flags[k] & 4u)) {
                            sbu[k] = sum2(m0[k], wu[k], m1[k], wv[k]);
                            sbv[k] = sum2(m2c[k], wu[k], m3[k], wv[k]);
                        }
                    }
                }
            }

            // ================= E: grass factor, Exner cell and faces of row q
            bool mq[CPT], mq1[CPT];
#pragma unroll
            for (int k = 0; k < CPT; ++k) {
                mq[k] = HAS_MASK && ((mwin[k] >> 2) & 1u);
                mq1[k] = HAS_MASK && ((mwin[k] >> 3) & 1u);
            }
            ECell<T> e3[CPT];
            T xe3[CPT], Fy[CPT];
#pragma unroll
            for (int k = 0; k < CPT; ++k) {
                e3[k] = ECell<T>{};
                xe3[k] = Fy[k] = T(0);
            }
            if (S || rowD) {  // warp-uniform: row q is outside the band's rows in some prologue / drain iterations
#pragma unroll
                for (int k = 0; k < CPT; ++k) {
                    const T Gq = MPM ? mpm_grass(hbh[k], hbu[k], hbv[k], mq[k], a.sed) : const_grass(hbh[k], gb1[k], mq[k]);
                    e3[k] = make_ecell(hbh[k], hbu[k], hbv[k], zb1[k], Gq);
                }
                // Below the Shields threshold G is 0 and every Exner flux is 0 (q = G |u|^2 u):
                // a warp whose rows q and q-1 carry no G skips the Exner faces, their shuffles
                // and activity tests; xe3 and Fy keep their +0.  Exact in both precisions: the
                // skipped fluxes are +-0, which leave z_b unchanged bit for bit, and a NaN G
                // (NaN depth or velocity in the MPM factor) is not 0, so it still propagates.
                bool anyG = false;
#pragma unroll
                for (int k = 0; k < CPT; ++k) anyG = anyG || !(e3[k].G == T(0)) || !(e4[k].G == T(0));
                if (__any_sync(FULL, anyG)) {
                    ECell<T> ee[CPT];
                    bool mqe[CPT];
#pragma unroll
                    for (int k = 0; k + 1 < CPT; ++k) { ee[k] = e3[k + 1]; mqe[k] = mq[k + 1]; }
                    ee[CPT - 1] = shfl_down_ecell(e3[0]);
                    mqe[CPT - 1] = HAS_MASK ? (__shfl_down_sync(FULL, (int)mq[0], 1) != 0) : false;
                    T F[CPT];
                    bool xact[CPT];
#pragma unroll
                    for (int k = 0; k < CPT; ++k) {
                        xact[k] = rowD && has_e[k] && exner_active(e3[k], ee[k], mq[k], mqe[k]);
                        const T Fx = exner_face<T, false>(e3[k], ee[k]);
                        F[k] = xact[k] ? Fx : T(0);
                        if (bud_item && xact[k] && out_col[k] && q >= R0 && q < R1 && q >= 1 && q <= ny - 2 &&
                            (cb + k == 0 || cb + k == nx - 2))
                            if constexpr (BUD) budbuf[threadIdx.x >> 5][1][lane] += cb + k == 0 ? -(double)F[k] : (double)F[k];
                    }
                    T Fw[CPT];
                    bool wact[CPT];
#pragma unroll
                    for (int k = 1; k < CPT; ++k) { Fw[k] = F[k - 1]; wact[k] = xact[k - 1]; }
                    Fw[0] = __shfl_up_sync(FULL, F[CPT - 1], 1);
                    wact[0] = (__shfl_up_sync(FULL, (int)xact[CPT - 1], 1) != 0) && lane > 0;
#pragma unroll
                    for (int k = 0; k < CPT; ++k) {
                        // roe_exner.py:710-711: -F of the west face first, then +F of the east face
                        if (wact[k]) xe3[k] = xe3[k] + (-Fw[k]);
                        if (xact[k]) xe3[k] = xe3[k] + F[k];
                        const bool yex = rowD && (S || q - 1 >= L0) && colok[k] && exner_active(e4[k], e3[k], mq1[k], mq[k]);
                        const T Fyv = exner_face<T, true>(e4[k], e3[k]);
                        Fy[k] = yex ? Fyv : T(0);
                        if (bud_item && yex && out_col[k] && (q == 1 || q == ny - 1) && q >= R0 && q < R1 &&
                            cb + k >= 1 && cb + k <= nx - 2)
                            if constexpr (BUD) budbuf[threadIdx.x >> 5][1][lane] += q == 1 ? -(double)Fy[k] : (double)Fy[k];
                    }
                }
            }

            // ================= F: z_b update of row r-4
            T zbp4[CPT], gg4[CPT];
#pragma unroll
            for (int k = 0; k < CPT; ++k) {
                zbp4[k] = T(0);
                if (S || (r - 4 >= L0 && r - 4 < L1)) {
                    T acc = xe4[k];
                    acc = acc + (-fn4[k]);  // north face (roe_exner.py:712)
                    acc = acc + Fy[k];      // south face (roe_exner.py:713)
                    if constexpr (is_f32<T>()) zbp4[k] = e4[k].zb - dtdx * acc;
                    else zbp4[k] = e4[k].zb - dt * acc / dx;
                }
                gg4[k] = e4[k].G;
            }

            // ================= G: second boundary application and stores of row p = r-5
            const int p = r - 5;
            const bool rowG = S || ((p >= L0) && (p < L1));
            T zfin[CPT], gfin[CPT];
#pragma unroll
            for (int k = 0; k < CPT; ++k) { zfin[k] = zbp5[k]; gfin[k] = gg5[k]; }
            if (rowG && (bc_strip || (bc_rows && (p == 0 || p == ny - 1)))) {
                unsigned flags[CPT];
                int zdy[CPT], zdx[CPT], gdy[CPT], gdx[CPT];
                bool anyf = false;
#pragma unroll
                for (int k = 0; k < CPT; ++k) {
                    flags[k] = 0u;
                    zdy[k] = zdx[k] = gdy[k] = gdx[k] = 0;
                    if constexpr (ASYNC_RECIPES) {
                        const unsigned w = zgb[(r - 2) & 3][CPT * lane + k];  // left by the first application of row p
                        flags[k] = w & 24u;
                        zdy[k] = (int)((w >> 8) & 15u) - 8;
                        zdx[k] = (int)((w >> 12) & 15u) - 8;
                        gdy[k] = (int)((w >> 16) & 15u) - 8;
                        gdx[k] = (int)((w >> 20) & 15u) - 8;
                    } else {
                        const int slot = colok[k] ? ring_slot(p, cb + k, ny, nx) : -1;
                        if (slot >= 0) {
                            const pxb_ring_recipe& rc = a.ring[slot];
                            flags[k] = rc.flags;
                            zdy[k] = rc.zb_dy; zdx[k] = rc.zb_dx; gdy[k] = rc.g_dy; gdx[k] = rc.g_dx;
                        }
                    }
                    anyf = anyf || ((flags[k] & 24u) != 0u);
                }
                if (__any_sync(FULL, anyf)) {
                    const bool dyrow = (p == 0) || (p == ny - 1);
                    T zv[CPT], gv[CPT];
                    fetch_donor<CPT>(dyrow, zdy, zdx, zbp6, zbp5, zbp4, zv);
                    fetch_donor<CPT>(dyrow, gdy, gdx, gg6, gg5, gg4, gv);
#pragma unroll
                    for (int k = 0; k < CPT; ++k) {
                        if (flags[k] & 8u) zfin[k] = zv[k];
                        if (flags[k] & 16u) gfin[k] = gv[k];
                    }
                }
            }
            if (rowG && p >= R0 && p < R1) {
                if constexpr (ASYNC_PARTNER) {
                    read_cols<CPT>(pb[r & 1][3], lane, pazb);
                    if (a.oG) read_cols<CPT>(pb[r & 1][4], lane, paG);
                }
#pragma unroll
                for (int k = 0; k < CPT; ++k) {
                    if (!out_col[k]) continue;
                    const unsigned i = (unsigned)p * upitch + (unsigned)(cb + k);
                    T zo = zfin[k], go = gfin[k];
                    if (AVG) {
                        zo = T(0.5) * pazb[k] + T(0.5) * zo;
                        if (a.oG) go = T(0.5) * paG[k] + T(0.5) * go;
                    }
                    a.ozb[i] = zo;
                    if (a.oG) a.oG[i] = go;
                    bad |= !d_isfinite(zo);
                }
            }
            if (rowD && q >= R0 && q < R1) {
                if constexpr (ASYNC_PARTNER) {
                    read_cols<CPT>(pb[r & 1][0], lane, pah);
                    read_cols<CPT>(pb[r & 1][1], lane, pahu);
                    read_cols<CPT>(pb[r & 1][2], lane, pahv);
                }
#pragma unroll
                for (int k = 0; k < CPT; ++k) {
                    if (!out_col[k]) continue;
                    const unsigned i = (unsigned)q * upitch + (unsigned)(cb + k);
                    T oh = sbh[k], ou = sbu[k], ov = sbv[k];
                    if (AVG) {
                        oh = T(0.5) * pah[k] + T(0.5) * oh;
                        ou = T(0.5) * pahu[k] + T(0.5) * ou;
                        ov = T(0.5) * pahv[k] + T(0.5) * ov;
                    }
                    a.oh[i] = oh;
                    a.ohu[i] = ou;
                    a.ohv[i] = ov;
                    bad |= !(d_isfinite(oh) && d_isfinite(ou) && d_isfinite(ov));
                }
            }

            // ================= shift the windows
#pragma unroll
            for (int k = 0; k < CPT; ++k) {
                pA[k] = pr[k]; hA[k] = h_r[k]; huA[k] = hu_r[k]; hvA[k] = hv_r[k];
#pragma unroll
                for (int m = 0; m < 3; ++m) { xfA[k][m] = xf[k][m]; nfA[k][m] = yP[k][m]; }
                zt3[k] = zt2[k]; zt2[k] = ztA[k]; ztA[k] = zt_r[k];
                hr3[k] = hr2[k]; hr2[k] = hr1[k]; hur2[k] = hur1[k]; hvr2[k] = hvr1[k];
                mwin[k] = (mwin[k] << 1) | (m_r[k] ? 1u : 0u);
                zin4[k] = zin3[k]; zin3[k] = zin2[k]; zin2[k] = zin1[k]; zin1[k] = zb_r[k];
                if (!MPM) { gin4[k] = gin3[k]; gin3[k] = gin2[k]; gin2[k] = gin1[k]; gin1[k] = g_r[k]; }
                hf4h[k] = hf3h[k]; hf4u[k] = hf3u[k]; hf4v[k] = hf3v[k];
                hf3h[k] = hf2h[k]; hf3u[k] = hf2u[k]; hf3v[k] = hf2v[k];
                e4[k] = e3[k]; xe4[k] = xe3[k]; fn4[k] = Fy[k];
                zbp6[k] = zbp5[k]; zbp5[k] = zbp4[k];
                gg6[k] = gg5[k]; gg5[k] = gg4[k];
            }
        };
        const int steady0 = min(L0 + 5, L1), steady1 = L1;
        int r = L0;
        for (; r < steady0; ++r) iterate(r, std::false_type{});
        PXB_UNROLL(PXB_STAGE_UNROLL)
        for (; r < steady1; ++r) iterate(r, std::true_type{});
        // drain until phase G has stored the band's last row (p = R1 - 1 at r = R1 + 4);
        // later iterations would only advance the halo rows below the band
        for (; r < R1 + 5; ++r) iterate(r, std::false_type{});
        cp_async_wait<0>();  // the buffers are reused by the next item
        if constexpr (BUD) {  // this item's outflow: the warp's slots in a fixed order
            double bh = budbuf[threadIdx.x >> 5][0][lane], bz = budbuf[threadIdx.x >> 5][1][lane];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                bh += __shfl_down_sync(FULL, bh, o);
                bz += __shfl_down_sync(FULL, bz, o);
            }
            if (lane == 0) {
                a.bud[2 * item] = bh;
                a.bud[2 * item + 1] = bz;
            }
        }
    }
}

// Whether an item lies away from the grid's boundary: an interior strip (boundary strips
// are the first two and the last two items of a band, as half-height items) of an
// interior band, or any item of a grid without boundary recipes.  Such items take the
// re_stage_item instantiation without boundary code, whose columns are all inside the
// grid (the same bits, fewer instructions per row).
template <class T>
__device__ __forceinline__ bool stage_item_interior(const REStageArgs<T>& a, const int item) {
    const int ipb = pxb_stage_items_per_band(a.nstrips);
    const int band = item / ipb, kb = item - band * ipb;
    return a.ring == nullptr || (ipb > 1 && kb >= 2 && kb < a.nstrips && band > 0 && band < a.nbands - 1);
}

// Work-queue order of the items: those that run the generic instantiation (the first and
// the last band, then in every band its boundary strips) come first, so that the items
// handed out last, which set the kernel's tail, are the uniform interior ones.  A
// permutation of the item numbers: the results do not depend on it.
template <class T>
__device__ __forceinline__ int stage_item_order(const REStageArgs<T>& a, const int q) {
    const int ipb = pxb_stage_items_per_band(a.nstrips);
    const int bq = q / ipb, k = q - bq * ipb;
    const int nb = a.nbands;
    const int band = (nb < 2 || bq == 0) ? 0 : (bq == 1 ? nb - 1 : bq - 1);
    // boundary items of a band: kb 0, 1 (first strip) and ipb-2, ipb-1 (last strip)
    const int kb = (ipb < 4 || k < 2) ? k : (k < 4 ? ipb - 4 + k : k - 2);
    return band * ipb + kb;
}

// The grid is sized to the resident capacity of the device.  A warp's first item is its
// warp index; further items come from a grid-wide queue (one atomic per item), so warps
// on lightly loaded SMs take more of them and no SM waits on a fixed share.  The last
// block to finish resets the queue for the next launch on the stream.
template <class T, bool MPM, bool HAS_MASK, bool AVG, bool BUD = false>
__global__ void __launch_bounds__(128, PXB_STAGE_BOUNDS(T, AVG)) re_stage_kernel(const REStageArgs<T> a) {
    const int lane = threadIdx.x & 31;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    const int nitems = pxb_stage_items_per_band(a.nstrips) * a.nbands;
    bool bad = false;
    int item = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    while (item < nitems) {
        const int it = stage_item_order(a, item);
        if (stage_item_interior(a, it)) re_stage_item<T, MPM, HAS_MASK, AVG, BUD, true>(a, it, bad);
        else re_stage_item<T, MPM, HAS_MASK, AVG, BUD, false>(a, it, bad);
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
