// Allocation-free CFL time step for the Roe-Exner bundle.
//
// pxb_re_cfl needs a plan, and creating a plan allocates device memory.  Some callers
// cannot allocate at the moment they need dt: an XLA custom call runs inside buffers
// that XLA has already allocated and must not grab device memory of its own, and a
// solver embedded in a host application may run under a policy that forbids cudaMalloc
// after start-up.  This variant takes only the state planes and an output scalar, and
// keeps its reduction scratch in a fixed array in device memory that the module owns.
//
// The scratch holds one partial maximum per work item (a 31-column strip times a band
// of rows) plus the completion counter of the last-block reduction.  Work items are
// capped at PXB_NOALLOC_MAX_ITEMS, which bounds the grid width to
// 31 * PXB_NOALLOC_MAX_ITEMS columns; wider grids are rejected.  The array stays
// resident on every device that loads the library until the process exits.  All calls
// share it, so two calls whose kernels overlap on the GPU (different streams without
// ordering between them, or different host threads on one device) race on it.
//
// The kernel (noalloc_kernel.cuh) runs the plan-based CFL's own work item, so both entry
// points evaluate the same faces with the same arithmetic; its float64 instantiation is
// compiled in noalloc_f64.cu with --fmad=false, like the other float64 kernels.
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <string>

#include "noalloc_kernel.cuh"
#include "pxb_launch.h"

#define PXB_NOALLOC_MAX_ITEMS 8192
#define PXB_NOALLOC_WORDS (PXB_NOALLOC_MAX_ITEMS + 32)  // partials, then the counter

static __device__ __align__(256) unsigned long long pxb_noalloc_scratch[PXB_NOALLOC_WORDS];

// float32 kernel instantiated here; float64 in noalloc_f64.cu (--fmad=false)
namespace pxb {
extern template cudaError_t launch_cfl_noalloc<double>(const CflArgs<double>&, unsigned long long*, unsigned int*,
                                                       int, cudaStream_t);
template cudaError_t launch_cfl_noalloc<float>(const CflArgs<float>&, unsigned long long*, unsigned int*, int,
                                               cudaStream_t);
}  // namespace pxb

namespace {

int nfail(int code, const std::string& m) { return pxb::set_error(code, m); }

// Device address of the scratch array, looked up once per device and context (host code
// cannot use the symbol's name as a device pointer).  The address belongs to the module
// loaded into the device's current context: after cudaDeviceReset the module is loaded
// again, possibly elsewhere, so the cache is keyed on the context handle too and is
// looked up again when that handle changes.
struct DevSlot {
    bool ready = false;
    void* ctx = nullptr;
    unsigned long long* ptr = nullptr;
};
std::mutex g_mu;
DevSlot g_slots[64];

typedef int (*CtxGetCurrentFn)(void**);  // cuCtxGetCurrent(CUcontext*), through the runtime's entry-point query

int current_context(void** ctx) {
    static CtxGetCurrentFn fn = nullptr;
    if (!fn) {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q{};
        const cudaError_t e = cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q);
        if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !f)
            return nfail(PXB_ERR_CUDA, "cuCtxGetCurrent entry point not available");
        fn = (CtxGetCurrentFn)f;
    }
    *ctx = nullptr;
    if (fn(ctx) != 0) return nfail(PXB_ERR_CUDA, "cuCtxGetCurrent failed");
    return PXB_OK;
}

int scratch_for_current_device(unsigned long long** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return nfail(PXB_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= 64) return nfail(PXB_ERR_ARG, "device ordinal out of range");
    void* ctx = nullptr;
    int st = current_context(&ctx);
    if (st != PXB_OK) return st;
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_slots[dev].ready || ctx == nullptr || g_slots[dev].ctx != ctx) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, pxb_noalloc_scratch);  // sets the runtime's context up if needed
        if (e != cudaSuccess)
            return nfail(PXB_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        st = current_context(&ctx);  // the context the address belongs to
        if (st != PXB_OK) return st;
        g_slots[dev].ptr = (unsigned long long*)p;
        g_slots[dev].ctx = ctx;
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
    e = pxb::launch_cfl_noalloc<T>(a, scr, done, nitems, s);
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
