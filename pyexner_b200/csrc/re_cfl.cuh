// CFL reduction for the Roe-Exner bundle (compute_dt_roeexner,
// PyExner src/PyExner/solvers/roe_exner_solver.py:118-122 with compute_dt_2D,
// roe_exner.py:257-310).
//
// min over active faces of dx / speed_f equals dx / max_f speed_f exactly (division by
// a positive number is monotone under round-to-nearest), so the kernel reduces the
// maximum speed: a warp-level max of the IEEE bit patterns (speeds are >= 0 or NaN, so
// unsigned order is float order and NaN wins like jnp.min's NaN), a block max through
// shared memory, one 64-bit atomicMax per block, and the last block to finish turns it
// into dt = max(cfl * dx / smax, 1e-6),
// resets the accumulator and logs dt.  Deterministic and free of host round trips.
//
// Work layout: a warp covers 32 columns and the 31 x-faces between them (strips overlap
// by one column) and marches down a band of rows; y-faces (r | r+1) belong to row r's band.
#pragma once
#include "pxb_device.cuh"
#include "re_stage.cuh"  // cp.async helpers

namespace pxb {

struct CflScratch {
    unsigned long long maxbits;  // running max of speed bits
    unsigned int done;           // finished blocks of the current launch
    unsigned int step;           // index into the dt log
    int err;                     // sticky error word
    int pad;
    double t_step;               // simulation time at the start of the current step
    double t_next;               // t_step + dt: the time the next dt is added to
    unsigned int queue[2];       // stage kernel work queue: items handed out, blocks finished
    unsigned int cfl_queue;      // CFL kernel work queue: items handed out (reset by the last block)
    unsigned int pad2;
};

// Start of a fixed-step run at time t0 (the first CFL launch moves it into t_step).
template <class T>
__global__ void set_time_kernel(CflScratch* scr, double t0) {
    scr->t_step = t0;
    scr->t_next = t0;
}

template <class T>
struct CflArgs {
    int ny, nx;
    long long pitch;
    const T *h, *hu, *hv, *G;
    const uint8_t* nodata;
    T dx, cfl, floor_dt;  // floor_dt = 1e-6 (Roe-Exner); <= 0 disables the floor
    CflScratch* scr;
    T* dt_out;   // device scalar
    T* dt_log;   // optional: dt_log[scr->step++] = dt
    int band_rows, nstrips, nbands;
};

// Rows in flight ahead of the one the float32 CFL item evaluates (tuning knob; the item
// does little arithmetic per row, so the copies must cover the memory latency).
#ifndef PXB_CFL_AHEAD
#define PXB_CFL_AHEAD 2
#endif

// Float32 work item of the CFL reduction (a 31-column strip of one band; the 32nd lane
// is the first column of the next strip, for the strip's last x-face).  Rows arrive in
// shared slots of this warp, PXB_CFL_AHEAD rows ahead.  With 16-byte aligned planes and a
// pitch that is a multiple of 4 elements (VEC), one 16-byte cp.async per lane copies a
// whole row of the four planes (9 chunks of 4 columns per plane, starting from lane 0's
// column rounded down to a multiple of 4; the 36 chunks are lanes 0-31 plus lanes 0-3
// again), so lanes read columns that other lanes copied, after a warp barrier; otherwise
// each lane copies its own column of each plane, 4 bytes at a time.  Two rows per loop
// iteration: the cells of the previous row stay where they are.  Columns beyond the grid
// read as G = 0 (the warp vote below) and never enter a face.
constexpr int PXB_CFL_RW = 36;  // floats per plane row in a shared slot of the float32 CFL item
constexpr int PXB_CFL_SLOTS = PXB_CFL_AHEAD < 4 ? 4 : (PXB_CFL_AHEAD < 8 ? 8 : 16);  // a power of two above AHEAD

// cb: this warp's slots (PXB_CFL_SLOTS rows of the four planes, PXB_CFL_RW floats each)
template <bool HAS_MASK, bool VEC>
__device__ __forceinline__ void re_cfl_item_f32(const CflArgs<float>& a, const int item, unsigned& best,
                                                float (*cb)[4][PXB_CFL_RW]) {
    constexpr int RW = PXB_CFL_RW;
    const int lane = threadIdx.x & 31;
    const int ny = a.ny, nx = a.nx;
    const float DRY = float(DRY_TOL);
    const int band = item / a.nstrips;
    const int strip = item - band * a.nstrips;
    const int c0 = strip * 31;
    const int c = c0 + lane;
    const bool colok = c < nx;
    const bool has_e = colok && (c + 1 < nx) && lane < 31;
    const int R0 = band * a.band_rows;
    const int R1 = min(ny, R0 + a.band_rows);
    const int rend = min(ny, R1 + 1);
    const unsigned upitch = (unsigned)a.pitch;  // planes are < 2^31 elements
    constexpr int AHEAD = PXB_CFL_AHEAD;
    constexpr int SLOTS = PXB_CFL_SLOTS;
    const int al = VEC ? (c0 & ~3) : c0;
    const int off = c0 - al;
    // VEC: this lane's chunks k = lane and k = 32 + lane (lanes 0-3): plane k / 9, columns al + 4 (k % 9)
    const float* csrc[2];
    unsigned cdst[2], cbytes[2];
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        const int k = lane + 32 * q;
        const int pl = min(k / 9, 3), j = k - 9 * (k / 9);
        const float* base = pl == 0 ? a.h : (pl == 1 ? a.hu : (pl == 2 ? a.hv : a.G));
        const int col = al + 4 * j;
        const bool ok = k < 36 && col + 4 <= (int)upitch;  // a chunk never straddles two rows
        csrc[q] = base + (ok ? col : 0);
        cbytes[q] = ok ? 16u : 0u;
        cdst[q] = (unsigned)__cvta_generic_to_shared(&cb[0][pl][4 * (j < 9 ? j : 0)]);
    }
    constexpr unsigned SLOT = 4 * RW * sizeof(float);
    auto issue = [&](int rr) __attribute__((always_inline)) {  // row rr into slot rr % SLOTS
        if (rr < rend) {
            const unsigned ro = (unsigned)rr * upitch;
            const unsigned so = (unsigned)(rr & (SLOTS - 1)) * SLOT;
            if constexpr (VEC) {
                cp_async16_zfill(cdst[0] + so, csrc[0] + ro, cbytes[0]);
                if (lane < 4) cp_async16_zfill(cdst[1] + so, csrc[1] + ro, cbytes[1]);
            } else if (colok) {
                float* d = &cb[rr & (SLOTS - 1)][0][lane];
                cp_async_elem(d, a.h + ro + c);
                cp_async_elem(d + RW, a.hu + ro + c);
                cp_async_elem(d + 2 * RW, a.hv + ro + c);
                cp_async_elem(d + 3 * RW, a.G + ro + c);
            }
        }
        cp_async_commit();
    };
    bool nm = false;
    auto fetch_mask = [&](int rr) __attribute__((always_inline)) {
        nm = false;
        if (HAS_MASK && colok && rr < rend) nm = __ldg(a.nodata + (unsigned)rr * upitch + (unsigned)c) != 0;
    };
    auto row = [&](const int r, CCell<float>& cur, bool& mc, const CCell<float>& prev, const bool mp)
                   __attribute__((always_inline)) {
        cp_async_wait<AHEAD - 1>();  // row r landed (rows r+1 .. r+AHEAD-1 may be in flight)
        if constexpr (VEC) __syncwarp();  // chunks copied by other lanes
        const float* sr = &cb[r & (SLOTS - 1)][0][off + lane];
        const float h = sr[0], hu = sr[RW], hv = sr[2 * RW];
        const float g = colok ? sr[3 * RW] : 0.f;
        issue(r + AHEAD);
        mc = nm;
        fetch_mask(r + 1);
        cur = make_ccell(h, hu, hv, g);
        // rows r-1 and r of the warp without G (below the Shields threshold) take
        // face_speed_nog, the same value without a~ and the cubic (a NaN G is not 0)
        const bool nog = !__any_sync(FULL, !(g == 0.f) || !(prev.G == 0.f));
        if (r < R1) {  // x-face (c | c+1) of row r
            CCell<float> e;
            e.h = __shfl_down_sync(FULL, cur.h, 1);
            e.sq = __shfl_down_sync(FULL, cur.sq, 1);
            e.u = __shfl_down_sync(FULL, cur.u, 1);
            e.v = __shfl_down_sync(FULL, cur.v, 1);
            const bool me = HAS_MASK ? (__shfl_down_sync(FULL, (int)mc, 1) != 0) : false;
            // cur.h = max(h, DRY_TOL) > DRY_TOL exactly when h > DRY_TOL (false for NaN)
            const bool act = has_e && ((cur.h > DRY) || (e.h > DRY)) && !(mc || me);
            if (nog) {  // branch-free: every lane evaluates, inactive ones are masked
                const unsigned b = __float_as_uint(face_speed_nog<float, false>(cur, e));
                best = (act && b > best) ? b : best;
            } else {
                e.G = __shfl_down_sync(FULL, cur.G, 1);
                e.rs = __shfl_down_sync(FULL, cur.rs, 1);
                // only active faces enter the cubic: a lane without a face (the strip's last, or
                // beyond the grid) could otherwise send the warp into the float64 fallback
                if (act) {
                    const unsigned b = __float_as_uint(face_speed<float, false>(cur, e));
                    best = b > best ? b : best;
                }
            }
        }
        if (r > R0) {  // y-face (r-1 | r)
            const bool act = colok && ((prev.h > DRY) || (cur.h > DRY)) && !(mp || mc);
            if (nog) {
                const unsigned b = __float_as_uint(face_speed_nog<float, true>(prev, cur));
                best = (act && b > best) ? b : best;
            } else if (act) {
                const unsigned b = __float_as_uint(face_speed<float, true>(prev, cur));
                best = b > best ? b : best;
            }
        }
    };
#pragma unroll
    for (int k = 0; k < AHEAD; ++k) issue(R0 + k);
    fetch_mask(R0);
    CCell<float> pa = make_ccell(1.f, 0.f, 0.f, 0.f), pb = pa;
    bool ma = false, mb = false;
    int r = R0;
    for (; r + 1 < rend; r += 2) {
        row(r, pb, mb, pa, ma);
        row(r + 1, pa, ma, pb, mb);
    }
    if (r < rend) row(r, pb, mb, pa, ma);
    cp_async_wait<0>();  // the slots are reused by the next item
    __syncwarp();
}

// Largest face-speed bit pattern seen by this lane over one work item (a 32-column strip
// of one band) folded into `best`; shared by the single-grid and the ensemble kernels.
template <class T, bool HAS_MASK>
__device__ __forceinline__ void re_cfl_item(const CflArgs<T>& a, const int item, unsigned long long& best) {
  if constexpr (is_f32<T>()) {
    const bool vec = ((((uintptr_t)a.h | (uintptr_t)a.hu | (uintptr_t)a.hv | (uintptr_t)a.G) & 15u) == 0) &&
                     ((a.pitch & 3) == 0);
    unsigned b = 0u;
    __shared__ __align__(16) float cbuf[8][PXB_CFL_SLOTS][4][PXB_CFL_RW];
    float(*cb)[4][PXB_CFL_RW] = cbuf[(threadIdx.x >> 5) & 7];
    if (vec) re_cfl_item_f32<HAS_MASK, true>(a, item, b, cb);
    else re_cfl_item_f32<HAS_MASK, false>(a, item, b, cb);
    best = (unsigned long long)b > best ? (unsigned long long)b : best;
  } else {
    const int lane = threadIdx.x & 31;
    const int ny = a.ny, nx = a.nx;
    const T DRY = T(DRY_TOL);
    {
        const int band = item / a.nstrips;
        const int strip = item - band * a.nstrips;
        const int c = strip * 31 + lane;
        const bool colok = c < nx;
        const bool has_e = colok && (c + 1 < nx) && lane < 31;
        const int R0 = band * a.band_rows;
        const int R1 = min(ny, R0 + a.band_rows);
        CCell<T> prev = make_ccell(T(1), T(0), T(0), T(0));
        T hprev = 0;
        bool mprev = false;
        const int rend = min(ny, R1 + 1);
        // float32: rows arrive by cp.async in this warp's shared slots two rows ahead (the
        // kernel is memory-latency bound with one row of register prefetch); float64 keeps
        // the register prefetch of row r+1.  The nodata byte is a register prefetch.
        constexpr bool ASYNC = is_f32<T>();
        __shared__ T cbuf[8][ASYNC ? 3 : 1][4][32];
        T(*cb)[4][32] = cbuf[(threadIdx.x >> 5) & 7];
        T nh = 1, nhu = 0, nhv = 0, ng = 0;
        bool nm = false;
        auto issue = [&](int rr) __attribute__((always_inline)) {  // float32: row rr into slot rr % 3
            T* d = &cb[rr % 3][0][lane];
            if (colok && rr < rend) {
                const long long i = (long long)rr * a.pitch + c;
                cp_async_elem(d, a.h + i);
                cp_async_elem(d + 32, a.hu + i);
                cp_async_elem(d + 64, a.hv + i);
                cp_async_elem(d + 96, a.G + i);
            } else {
                d[0] = T(1);
                d[32] = d[64] = d[96] = T(0);
            }
            cp_async_commit();
        };
        auto fetch = [&](int rr) __attribute__((always_inline)) {
            nm = false;
            if constexpr (!ASYNC) {
                nh = 1;
                nhu = nhv = ng = 0;
            }
            if (colok && rr < rend) {
                const long long i = (long long)rr * a.pitch + c;
                if constexpr (!ASYNC) {
                    nh = __ldg(a.h + i);
                    nhu = __ldg(a.hu + i);
                    nhv = __ldg(a.hv + i);
                    ng = __ldg(a.G + i);
                }
                if (HAS_MASK) nm = __ldg(a.nodata + i) != 0;
            }
        };
        if constexpr (ASYNC) {
            issue(R0);
            issue(R0 + 1);
        }
        fetch(R0);
        for (int r = R0; r < rend; ++r) {
            T h = nh, hu = nhu, hv = nhv, g = ng;
            if constexpr (ASYNC) {
                cp_async_wait<1>();  // row r landed (row r+1 may be in flight); each lane reads its own slots
                const T* sr = &cb[r % 3][0][lane];
                h = sr[0];
                hu = sr[32];
                hv = sr[64];
                g = sr[96];
                issue(r + 2);
            }
            const bool m = nm;
            fetch(r + 1);
            const CCell<T> cur = make_ccell(h, hu, hv, g);
            // rows r-1 and r of the warp without G (below the Shields threshold) take
            // face_speed_nog, the same value without a~ and the cubic (a NaN G is not 0)
            const bool nog = !__any_sync(FULL, !(g == T(0)) || !(prev.G == T(0)));
            if (r < R1) {  // x-face (c | c+1) of row r
                CCell<T> e;
                e.h = __shfl_down_sync(FULL, cur.h, 1);
                e.sq = __shfl_down_sync(FULL, cur.sq, 1);
                e.u = __shfl_down_sync(FULL, cur.u, 1);
                e.v = __shfl_down_sync(FULL, cur.v, 1);
                e.G = __shfl_down_sync(FULL, cur.G, 1);
                e.rs = __shfl_down_sync(FULL, cur.rs, 1);
                const T he = __shfl_down_sync(FULL, h, 1);
                const bool me = HAS_MASK ? (__shfl_down_sync(FULL, (int)m, 1) != 0) : false;
                if (has_e && ((h > DRY) || (he > DRY)) && !(m || me)) {
                    const unsigned long long b =
                        speed_bits(nog ? face_speed_nog<T, false>(cur, e) : face_speed<T, false>(cur, e));
                    best = b > best ? b : best;
                }
            }
            if (r > R0 && colok && ((hprev > DRY) || (h > DRY)) && !(mprev || m)) {  // y-face (r-1 | r)
                const unsigned long long b =
                    speed_bits(nog ? face_speed_nog<T, true>(prev, cur) : face_speed<T, true>(prev, cur));
                best = b > best ? b : best;
            }
            prev = cur;
            hprev = h;
            mprev = m;
        }
        if constexpr (ASYNC) cp_async_wait<0>();  // the slots are reused by the next item
    }
  }
}

// Resident 256-thread blocks per SM the CFL kernel is compiled for (tuning knob; by
// default the compiler's register choice sets it).
#ifdef PXB_CFL_MIN_BLOCKS
#define PXB_CFL_BOUNDS __launch_bounds__(256, PXB_CFL_MIN_BLOCKS)
#else
#define PXB_CFL_BOUNDS __launch_bounds__(256)
#endif

template <class T, bool HAS_MASK>
__global__ void PXB_CFL_BOUNDS re_cfl_kernel(const CflArgs<T> a) {
    const int lane = threadIdx.x & 31;
    const int wid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    unsigned long long best = 0ull;
    const int nitems = a.nstrips * a.nbands;
    // first item by warp index, the rest from a grid-wide queue (faster warps take more)
    int item = wid;
    while (item < nitems) {
        re_cfl_item<T, HAS_MASK>(a, item, best);
        unsigned next = 0;
        if (lane == 0) next = atomicAdd(&a.scr->cfl_queue, 1u);
        item = nw + (int)__shfl_sync(FULL, next, 0);
    }
    // warp max, block max through shared memory, one atomic and one fence per block
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long other = __shfl_xor_sync(FULL, best, o);
        best = other > best ? other : best;
    }
    __shared__ unsigned long long wmax[8];
    if (lane == 0) wmax[threadIdx.x >> 5] = best;
    __syncthreads();
    if (threadIdx.x != 0) return;
#pragma unroll
    for (int w = 1; w < 8; ++w) best = wmax[w] > best ? wmax[w] : best;
    if (best != 0ull) atomicMax(&a.scr->maxbits, best);
    __threadfence();  // the block's maximum before its ticket
    // last block finalises
    const unsigned int ticket = atomicAdd(&a.scr->done, 1u);
    if (ticket == gridDim.x - 1) {
        __threadfence();
        const unsigned long long bits = atomicAdd(&a.scr->maxbits, 0ull);
        const T smax = bits_speed(bits, T(0));
        // min_f dx/speed_f (inf when no face is active), then cfl * dt and the floor
        T dt = a.cfl * (a.dx / smax);
        if (a.floor_dt > T(0)) dt = clamp_lo(dt, a.floor_dt);
        *a.dt_out = dt;
        if (a.dt_log) a.dt_log[a.scr->step] = dt;
        a.scr->step += 1;
        // time of this step, accumulated in float64 like the host loops of the integrators
        a.scr->t_step = a.scr->t_next;
        a.scr->t_next = a.scr->t_next + (double)dt;
        if (!d_isfinite(dt)) a.scr->err |= 2;
        a.scr->maxbits = 0ull;
        a.scr->done = 0u;
        a.scr->cfl_queue = 0u;  // every warp has left its item loop
        __threadfence();
    }
}

}  // namespace pxb
