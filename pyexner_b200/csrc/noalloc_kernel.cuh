// Kernel of the allocation-free CFL time step (noalloc.cu): the plan-based CFL's work
// item (re_cfl_item, one 31-column strip of one band) per warp, one partial maximum per
// item in caller-provided scratch, and a last-block reduction of the partials.  Kept in
// a header so that the float64 instantiation is compiled in its own translation unit
// with --fmad=false, like every other float64 kernel of the library.
#pragma once
#include <cuda_runtime.h>

#include "re_cfl.cuh"

namespace pxb {

template <class T, bool HAS_MASK>
__global__ void __launch_bounds__(256) cfl_noalloc_kernel(CflArgs<T> a, unsigned long long* part,
                                                          unsigned int* done, int nitems) {
    const int lane = threadIdx.x & 31;
    const int item = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    unsigned long long best = 0ull;
    if (item < nitems) re_cfl_item<T, HAS_MASK>(a, item, best);
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long other = __shfl_xor_sync(FULL, best, o);
        best = other > best ? other : best;
    }
    // every item writes its own slot on every call, so the partials need no clearing
    if (lane == 0 && item < nitems) part[item] = best;
    __threadfence();
    __shared__ bool last;
    __shared__ unsigned long long red[8];
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(done, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!last) return;
    __threadfence();
    unsigned long long m = 0ull;
    for (int k = threadIdx.x; k < nitems; k += blockDim.x) {
        const unsigned long long v = ((volatile unsigned long long*)part)[k];
        m = v > m ? v : m;
    }
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long other = __shfl_xor_sync(FULL, m, o);
        m = other > m ? other : m;
    }
    if (lane == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) m = red[w] > m ? red[w] : m;
        m = red[0] > m ? red[0] : m;
        const T smax = bits_speed(m, T(0));
        // the same finalisation as re_cfl_kernel's last block
        T dt = a.cfl * (a.dx / smax);
        if (a.floor_dt > T(0)) dt = clamp_lo(dt, a.floor_dt);
        *a.dt_out = dt;
        *done = 0u;  // leave the counter at zero for the next call
    }
}

// Launches cfl_noalloc_kernel over `nitems` work items (8 warps per block); `part` holds
// at least `nitems` words and `done` is zero on entry.
template <class T>
cudaError_t launch_cfl_noalloc(const CflArgs<T>& a, unsigned long long* part, unsigned int* done, int nitems,
                               cudaStream_t s) {
    const int grid = (nitems + 7) / 8;
    if (a.nodata) cfl_noalloc_kernel<T, true><<<grid, 256, 0, s>>>(a, part, done, nitems);
    else cfl_noalloc_kernel<T, false><<<grid, 256, 0, s>>>(a, part, done, nitems);
    return cudaGetLastError();
}

}  // namespace pxb
