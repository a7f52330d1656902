// Allocation-free CFL time step for the Roe-Exner bundle.
//
// pxb_re_cfl needs a plan, and creating a plan allocates device memory.  Some callers
// cannot allocate at the moment they need dt: an XLA custom call runs inside buffers
// that XLA has already allocated and must not grab device memory of its own, a solver
// embedded in a host application may run under a policy that forbids cudaMalloc after
// start-up, and allocating inside a stream capture would break the capture.  This
// variant takes only the state planes and an output scalar, and keeps its reduction
// scratch in a fixed array in device memory that the module owns.
//
// The scratch holds one partial maximum per work item (a 31-column strip times a band
// of rows) plus the completion counter of the last-block reduction.  Work items are
// capped at PXB_NOALLOC_MAX_ITEMS, which bounds the grid width to
// 31 * PXB_NOALLOC_MAX_ITEMS columns; wider grids are rejected.  The array stays
// resident on every device that loads the library until the process exits.  All calls
// share it, so two calls whose kernels overlap on the GPU (different streams without
// ordering between them, or different host threads on one device) race on it.
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <string>

#include "pxb_launch.h"

#define PXB_NOALLOC_MAX_ITEMS 8192
#define PXB_NOALLOC_WORDS (PXB_NOALLOC_MAX_ITEMS + 32)  // partials, then the counter

static __device__ __align__(256) unsigned long long pxb_noalloc_scratch[PXB_NOALLOC_WORDS];

namespace {

int nfail(int code, const std::string& m) { return pxb::set_error(code, m); }

template <class T, bool HAS_MASK>
__global__ void __launch_bounds__(256) cfl_noalloc_kernel(pxb::CflArgs<T> a, unsigned long long* part,
                                                          unsigned int* done, int nitems) {
    using namespace pxb;
    const int lane = threadIdx.x & 31;
    const int item = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const T DRY = T(DRY_TOL);
    unsigned long long best = 0ull;
    if (item < nitems) {
        const int band = item / a.nstrips;
        const int strip = item - band * a.nstrips;
        const int c = strip * 31 + lane;
        const bool colok = c < a.nx;
        const bool has_e = colok && (c + 1 < a.nx) && lane < 31;
        const int R0 = band * a.band_rows;
        const int R1 = min(a.ny, R0 + a.band_rows);
        CCell<T> prev = make_ccell(T(1), T(0), T(0), T(0));
        T hprev = 0;
        bool mprev = false;
        for (int r = R0; r < min(a.ny, R1 + 1); ++r) {
            T h = 1, hu = 0, hv = 0, g = 0;
            bool m = false;
            if (colok) {
                const long long i = (long long)r * a.pitch + c;
                h = a.h[i];
                hu = a.hu[i];
                hv = a.hv[i];
                g = a.G[i];
                if (HAS_MASK) m = a.nodata[i] != 0;
            }
            const CCell<T> cur = make_ccell(h, hu, hv, g);
            if (r < R1) {
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
                    const unsigned long long b = speed_bits(face_speed<T, false>(cur, e));
                    best = b > best ? b : best;
                }
            }
            if (r > R0 && colok && ((hprev > DRY) || (h > DRY)) && !(mprev || m)) {
                const unsigned long long b = speed_bits(face_speed<T, true>(prev, cur));
                best = b > best ? b : best;
            }
            prev = cur;
            hprev = h;
            mprev = m;
        }
    }
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
        T dt = a.cfl * (a.dx / smax);
        dt = clamp_lo(dt, a.floor_dt);
        *a.dt_out = dt;
        *done = 0u;  // leave the counter at zero for the next call
    }
}

// Device address of the scratch array, looked up once per device (host code cannot use
// the symbol's name as a device pointer).
struct DevSlot {
    bool ready = false;
    unsigned long long* ptr = nullptr;
};
std::mutex g_mu;
DevSlot g_slots[64];

int scratch_for_current_device(unsigned long long** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return nfail(PXB_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= 64) return nfail(PXB_ERR_ARG, "device ordinal out of range");
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_slots[dev].ready) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, pxb_noalloc_scratch);
        if (e != cudaSuccess)
            return nfail(PXB_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        g_slots[dev].ptr = (unsigned long long*)p;
        g_slots[dev].ready = true;
    }
    *out = g_slots[dev].ptr;
    return PXB_OK;
}

template <class T>
int launch(int ny, int nx, long long pitch, double dx, double cfl, const void* h, const void* hu, const void* hv,
           const void* G, const uint8_t* nodata, void* dt_out, cudaStream_t s) {
    const int nstrips = (nx + 30) / 31;
    int nbands = std::max(1, std::min((ny + 7) / 8, PXB_NOALLOC_MAX_ITEMS / nstrips));
    const int band_rows = (ny + nbands - 1) / nbands;
    nbands = (ny + band_rows - 1) / band_rows;
    const int nitems = nstrips * nbands;
    unsigned long long* scr = nullptr;
    int st = scratch_for_current_device(&scr);
    if (st != PXB_OK) return st;
    unsigned int* done = (unsigned int*)(scr + PXB_NOALLOC_MAX_ITEMS);
    cudaError_t e = cudaMemsetAsync(done, 0, sizeof(unsigned int), s);
    if (e != cudaSuccess) return nfail(PXB_ERR_CUDA, std::string("cudaMemsetAsync: ") + cudaGetErrorString(e));
    pxb::CflArgs<T> a{};
    a.ny = ny;
    a.nx = nx;
    a.pitch = pitch;
    a.h = (const T*)h;
    a.hu = (const T*)hu;
    a.hv = (const T*)hv;
    a.G = (const T*)G;
    a.nodata = nodata;
    a.dx = (T)dx;
    a.cfl = (T)cfl;
    a.floor_dt = (T)pxb::DT_FLOOR;
    a.dt_out = (T*)dt_out;
    a.band_rows = band_rows;
    a.nstrips = nstrips;
    a.nbands = nbands;
    const int grid = (nitems + 7) / 8;
    if (nodata) cfl_noalloc_kernel<T, true><<<grid, 256, 0, s>>>(a, scr, done, nitems);
    else cfl_noalloc_kernel<T, false><<<grid, 256, 0, s>>>(a, scr, done, nitems);
    e = cudaGetLastError();
    if (e != cudaSuccess) return nfail(PXB_ERR_CUDA, std::string("cfl kernel launch: ") + cudaGetErrorString(e));
    return PXB_OK;
}

}  // namespace

extern "C" int pxb_re_cfl_noalloc(int32_t ny, int32_t nx, int64_t pitch, int32_t dtype, double dx, double cfl,
                                  const void* h, const void* hu, const void* hv, const void* G,
                                  const uint8_t* nodata, void* dt_dev, void* stream) {
    if (ny < 2 || nx < 2) return nfail(PXB_ERR_ARG, "grid must be at least 2 x 2 cells");
    if (pitch < nx) return nfail(PXB_ERR_ARG, "pitch smaller than nx");
    if ((nx + 30) / 31 > PXB_NOALLOC_MAX_ITEMS)
        return nfail(PXB_ERR_ARG, "nx = " + std::to_string(nx) + " exceeds the allocation-free limit of " +
                                      std::to_string(31 * PXB_NOALLOC_MAX_ITEMS) + " columns");
    if (dtype != PXB_F32 && dtype != PXB_F64) return nfail(PXB_ERR_ARG, "dtype must be PXB_F32 or PXB_F64");
    if (!(dx > 0)) return nfail(PXB_ERR_ARG, "dx must be positive");
    if (!h || !hu || !hv || !G || !dt_dev) return nfail(PXB_ERR_ARG, "h, hu, hv, G and dt_dev must be set");
    cudaStream_t s = (cudaStream_t)stream;
    return dtype == PXB_F64 ? launch<double>(ny, nx, pitch, dx, cfl, h, hu, hv, G, nodata, dt_dev, s)
                            : launch<float>(ny, nx, pitch, dx, cfl, h, hu, hv, G, nodata, dt_dev, s);
}
