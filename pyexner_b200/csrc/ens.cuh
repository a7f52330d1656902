// Ragged ensembles: many independent Roe-Exner grids (each with its own size, state,
// boundary recipes and dt) advanced together, one launch per phase for all members.
//
// The work items of every member (warp strips x row bands, as in the single-grid
// kernels) are numbered consecutively, member after member; a persistent grid covers the
// global item range (first item by warp index, the rest from a work queue).  A warp finds
// the member of its item by binary search in the item offsets and keeps that member's
// argument block in a shared-memory slot of its own, refreshed only when the member
// changes, so the per-item body is exactly the single-grid one (re_stage_item /
// re_cfl_item) reading its arguments from shared memory.
//
// CFL: each item folds its face speeds into the member's maximum (one 64-bit atomicMax
// per warp and item); a one-thread-per-member launch then turns the maxima into the
// members' dts, logs and resets them.  Each member keeps its own dt, as N separate runs of
// the reference's integrator would.
#pragma once
#include "re_cfl.cuh"
#include "re_stage.cuh"

namespace pxb {

template <class T>
struct EnsStageArgs {
    const REStageArgs<T>* args;  // per member
    const int* base;             // item offset of each member, nmembers + 1 entries
    int nmembers;
    unsigned int* queue;         // {next dynamic item, finished blocks}, zero between launches
};

template <class T>
struct EnsCflArgs {
    const CflArgs<T>* args;  // per member (scr, dt_out, dt_log, cfl, dx, floor per member)
    const int* base;
    int nmembers;
    int log_stride;  // members per dt-log row
};

__device__ __forceinline__ int ens_member_of(const int* base, int nm, int item) {
    int lo = 0, hi = nm - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(base + mid) <= item) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// Warp-cooperative copy of one argument block into the warp's shared slot.
template <class A>
__device__ __forceinline__ void ens_load_slot(A* slot, const A* src) {
    static_assert(sizeof(A) % 4 == 0, "argument blocks are copied as 32-bit words");
    const unsigned* s = reinterpret_cast<const unsigned*>(src);
    unsigned* d = reinterpret_cast<unsigned*>(slot);
    __syncwarp();
    for (int k = threadIdx.x & 31; k < (int)(sizeof(A) / 4); k += 32) d[k] = __ldg(s + k);
    __syncwarp();
}

// Items beyond one per warp come from a grid-wide queue, as in re_stage_kernel.
template <class T, bool MPM, bool HAS_MASK, bool AVG>
__global__ void __launch_bounds__(128, PXB_STAGE_BOUNDS(T, AVG)) ens_stage_kernel(const EnsStageArgs<T> e) {
    __shared__ REStageArgs<T> slot[4];
    const int w = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    const int total = __ldg(e.base + e.nmembers);
    int cur = -1;
    bool bad = false;
    int item = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    while (item < total) {
        const int m = ens_member_of(e.base, e.nmembers, item);
        if (m != cur) {
            if (bad) atomicOr(slot[w].err, 1);
            bad = false;
            ens_load_slot(&slot[w], e.args + m);
            cur = m;
        }
        re_stage_item<T, MPM, HAS_MASK, AVG>(slot[w], item - __ldg(e.base + m), bad);
        unsigned next = 0;
        if (lane == 0) next = atomicAdd(&e.queue[0], 1u);
        item = nw + (int)__shfl_sync(FULL, next, 0);
    }
    if (bad) atomicOr(slot[w].err, 1);
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(&e.queue[1], 1u) == gridDim.x - 1) {
            atomicExch(&e.queue[0], 0u);
            atomicExch(&e.queue[1], 0u);
        }
    }
}

template <class T, bool HAS_MASK>
__global__ void __launch_bounds__(256) ens_cfl_kernel(const EnsCflArgs<T> e) {
    __shared__ CflArgs<T> slot[8];
    const int w = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const int wid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    const int total = __ldg(e.base + e.nmembers);
    int cur = -1;
    for (int item = wid; item < total; item += nw) {
        const int m = ens_member_of(e.base, e.nmembers, item);
        if (m != cur) {
            ens_load_slot(&slot[w], e.args + m);
            cur = m;
        }
        unsigned long long best = 0ull;
        re_cfl_item<T, HAS_MASK>(slot[w], item - __ldg(e.base + m), best);
        for (int o = 16; o > 0; o >>= 1) {
            const unsigned long long other = __shfl_xor_sync(FULL, best, o);
            best = other > best ? other : best;
        }
        if (lane == 0 && best != 0ull) atomicMax(&slot[w].scr->maxbits, best);
    }
}

// dt of every member from its maximum face speed (as the last block of re_cfl_kernel).
template <class T>
__global__ void ens_cfl_finalize_kernel(const EnsCflArgs<T> e) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= e.nmembers) return;
    const CflArgs<T>& a = e.args[m];
    CflScratch* scr = a.scr;
    const T smax = bits_speed(scr->maxbits, T(0));
    T dt = a.cfl * (a.dx / smax);
    if (a.floor_dt > T(0)) dt = clamp_lo(dt, a.floor_dt);
    *a.dt_out = dt;
    if (a.dt_log) a.dt_log[(long long)scr->step * e.log_stride + m] = dt;
    scr->step += 1;
    if (!d_isfinite(dt)) scr->err |= 2;
    scr->maxbits = 0ull;
}

}  // namespace pxb
