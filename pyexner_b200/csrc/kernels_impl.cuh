// Launchers shared by the float and double translation units.
#pragma once
#include "pxb_launch.h"

namespace pxb {

template <class T, bool MPM, bool HM, bool AVG>
static cudaError_t stage_variant(const REStageArgs<T>& a, int grid, cudaStream_t s) {
    // the budget variant only when its partial array is set (the others carry no budget code)
    if (a.bud) re_stage_kernel<T, MPM, HM, AVG, true><<<grid, 128, 0, s>>>(a);
    else re_stage_kernel<T, MPM, HM, AVG, false><<<grid, 128, 0, s>>>(a);
    return cudaGetLastError();
}

template <class T>
cudaError_t launch_re_stage(const REStageArgs<T>& a, bool mpm, bool hm, bool avg, int grid, cudaStream_t s) {
    const int key = (mpm ? 4 : 0) | (hm ? 2 : 0) | (avg ? 1 : 0);
    switch (key) {
        case 0: return stage_variant<T, false, false, false>(a, grid, s);
        case 1: return stage_variant<T, false, false, true>(a, grid, s);
        case 2: return stage_variant<T, false, true, false>(a, grid, s);
        case 3: return stage_variant<T, false, true, true>(a, grid, s);
        case 4: return stage_variant<T, true, false, false>(a, grid, s);
        case 5: return stage_variant<T, true, false, true>(a, grid, s);
        case 6: return stage_variant<T, true, true, false>(a, grid, s);
        default: return stage_variant<T, true, true, true>(a, grid, s);
    }
}

template <class T, bool MPM, bool HM, bool AVG>
static int stage_occ() {
    int n = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, re_stage_kernel<T, MPM, HM, AVG>, 128, 0);
    return n;
}

template <class T>
int re_stage_blocks_per_sm(bool mpm, bool hm, bool avg) {
    const int key = (mpm ? 4 : 0) | (hm ? 2 : 0) | (avg ? 1 : 0);
    switch (key) {
        case 0: return stage_occ<T, false, false, false>();
        case 1: return stage_occ<T, false, false, true>();
        case 2: return stage_occ<T, false, true, false>();
        case 3: return stage_occ<T, false, true, true>();
        case 4: return stage_occ<T, true, false, false>();
        case 5: return stage_occ<T, true, false, true>();
        case 6: return stage_occ<T, true, true, false>();
        default: return stage_occ<T, true, true, true>();
    }
}

template <class T>
cudaError_t launch_re_cfl(const CflArgs<T>& a, bool hm, int grid, cudaStream_t s) {
    if (hm) re_cfl_kernel<T, true><<<grid, 256, 0, s>>>(a);
    else re_cfl_kernel<T, false><<<grid, 256, 0, s>>>(a);
    return cudaGetLastError();
}

template <class T>
int re_cfl_blocks_per_sm(bool hm) {
    int n = 0;
    if (hm) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, re_cfl_kernel<T, true>, 256, 0);
    else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, re_cfl_kernel<T, false>, 256, 0);
    return n;
}

template <class T>
cudaError_t launch_re_init(const InitArgs<T>& a, cudaStream_t s) {
    dim3 b(32, 8), g((a.nx + 31) / 32, (a.ny + 7) / 8);
    re_init_kernel<T><<<g, b, 0, s>>>(a);
    return cudaGetLastError();
}

template <class T>
cudaError_t launch_bc(const BcArgs<T>& a, cudaStream_t s) {
    if (a.count <= 0) return cudaSuccess;
    const int g = (a.count + 255) / 256;
    bc_gather_kernel<T><<<g, 256, 0, s>>>(a);
    bc_scatter_kernel<T><<<g, 256, 0, s>>>(a);
    return cudaGetLastError();
}

template <class T, bool MPM, bool HM, bool AVG>
static cudaError_t ens_variant(const EnsStageArgs<T>& a, int grid, cudaStream_t s) {
    ens_stage_kernel<T, MPM, HM, AVG><<<grid, 128, 0, s>>>(a);
    return cudaGetLastError();
}

template <class T>
cudaError_t launch_ens_stage(const EnsStageArgs<T>& a, bool mpm, bool hm, bool avg, int grid, cudaStream_t s) {
    const int key = (mpm ? 4 : 0) | (hm ? 2 : 0) | (avg ? 1 : 0);
    switch (key) {
        case 0: return ens_variant<T, false, false, false>(a, grid, s);
        case 1: return ens_variant<T, false, false, true>(a, grid, s);
        case 2: return ens_variant<T, false, true, false>(a, grid, s);
        case 3: return ens_variant<T, false, true, true>(a, grid, s);
        case 4: return ens_variant<T, true, false, false>(a, grid, s);
        case 5: return ens_variant<T, true, false, true>(a, grid, s);
        case 6: return ens_variant<T, true, true, false>(a, grid, s);
        default: return ens_variant<T, true, true, true>(a, grid, s);
    }
}

template <class T, bool MPM, bool HM, bool AVG>
static int ens_occ() {
    int n = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, ens_stage_kernel<T, MPM, HM, AVG>, 128, 0);
    return n;
}

template <class T>
int ens_stage_blocks_per_sm(bool mpm, bool hm, bool avg) {
    const int key = (mpm ? 4 : 0) | (hm ? 2 : 0) | (avg ? 1 : 0);
    switch (key) {
        case 0: return ens_occ<T, false, false, false>();
        case 1: return ens_occ<T, false, false, true>();
        case 2: return ens_occ<T, false, true, false>();
        case 3: return ens_occ<T, false, true, true>();
        case 4: return ens_occ<T, true, false, false>();
        case 5: return ens_occ<T, true, false, true>();
        case 6: return ens_occ<T, true, true, false>();
        default: return ens_occ<T, true, true, true>();
    }
}

template <class T>
cudaError_t launch_ens_cfl(const EnsCflArgs<T>& a, bool hm, int grid, cudaStream_t s) {
    if (hm) ens_cfl_kernel<T, true><<<grid, 256, 0, s>>>(a);
    else ens_cfl_kernel<T, false><<<grid, 256, 0, s>>>(a);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    ens_cfl_finalize_kernel<T><<<(a.nmembers + 127) / 128, 128, 0, s>>>(a);
    return cudaGetLastError();
}

template <class T>
cudaError_t launch_re_general(const GenArgs<T>& a, int phase, cudaStream_t s) {
    dim3 b(32, 8), g((a.nx + 31) / 32, (a.ny + 7) / 8);
    switch (phase) {
        case GEN_HYDRO: gen_hydro_kernel<T><<<g, b, 0, s>>>(a); break;
        case GEN_CORR: gen_corr_kernel<T><<<g, b, 0, s>>>(a); break;
        case GEN_GRASS: gen_grass_kernel<T><<<g, b, 0, s>>>(a); break;
        case GEN_EXNER: gen_exner_kernel<T><<<g, b, 0, s>>>(a); break;
        default: gen_store_kernel<T><<<g, b, 0, s>>>(a); break;
    }
    return cudaGetLastError();
}

template <class T>
cudaError_t launch_set_time(CflScratch* scr, double t0, cudaStream_t s) {
    set_time_kernel<T><<<1, 1, 0, s>>>(scr, t0);
    return cudaGetLastError();
}

template <class T>
cudaError_t launch_roe_stage(const RoeArgs<T>& a, bool avg, cudaStream_t s) {
    const long long threads = 4LL * a.ny * a.nx;  // four threads per cell
    const int g = (int)((threads + 255) / 256);
    if (avg) roe_stage_kernel<T, true><<<g, 256, 0, s>>>(a);
    else roe_stage_kernel<T, false><<<g, 256, 0, s>>>(a);
    return cudaGetLastError();
}

template <class T>
cudaError_t launch_budget_stage(const double* part, int nitems, const T* dt, double w_dx, BudgetAcc* acc,
                                cudaStream_t s) {
    budget_stage_kernel<T><<<1, 256, 0, s>>>(part, nitems, dt, w_dx, acc);
    return cudaGetLastError();
}

template <class T>
cudaError_t launch_volume(int ny, int nx, long long pitch, const T* h, const T* zb, const uint8_t* nodata,
                          double* part, int nblocks, double dx2, double* out, cudaStream_t s) {
    volume_kernel<T><<<nblocks, 256, 0, s>>>(ny, nx, pitch, h, zb, nodata, part);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    volume_final_kernel<<<1, 32, 0, s>>>(part, nblocks, dx2, out);
    return cudaGetLastError();
}

template <class T>
cudaError_t launch_roe_cfl(const CflArgs<T>& a, int grid, cudaStream_t s) {
    roe_cfl_kernel<T><<<grid, 256, 0, s>>>(a);
    return cudaGetLastError();
}

#define PXB_INSTANTIATE(T)                                                                              \
    template cudaError_t launch_re_stage<T>(const REStageArgs<T>&, bool, bool, bool, int, cudaStream_t); \
    template int re_stage_blocks_per_sm<T>(bool, bool, bool);                                           \
    template cudaError_t launch_re_cfl<T>(const CflArgs<T>&, bool, int, cudaStream_t);                  \
    template int re_cfl_blocks_per_sm<T>(bool);                                                         \
    template cudaError_t launch_re_init<T>(const InitArgs<T>&, cudaStream_t);                           \
    template cudaError_t launch_bc<T>(const BcArgs<T>&, cudaStream_t);                                  \
    template cudaError_t launch_re_general<T>(const GenArgs<T>&, int, cudaStream_t);                    \
    template cudaError_t launch_ens_stage<T>(const EnsStageArgs<T>&, bool, bool, bool, int, cudaStream_t); \
    template int ens_stage_blocks_per_sm<T>(bool, bool, bool);                                          \
    template cudaError_t launch_ens_cfl<T>(const EnsCflArgs<T>&, bool, int, cudaStream_t);              \
    template cudaError_t launch_set_time<T>(CflScratch*, double, cudaStream_t);                         \
    template cudaError_t launch_roe_stage<T>(const RoeArgs<T>&, bool, cudaStream_t);                    \
    template cudaError_t launch_roe_cfl<T>(const CflArgs<T>&, int, cudaStream_t);                      \
    template cudaError_t launch_budget_stage<T>(const double*, int, const T*, double, BudgetAcc*, cudaStream_t); \
    template cudaError_t launch_volume<T>(int, int, long long, const T*, const T*, const uint8_t*, double*, int, \
                                          double, double*, cudaStream_t);

}  // namespace pxb
