// Reverse-mode (adjoint) kernels of the float64 stage and CFL step (adjoint.cuh).
// Compiled with --fmad=false, like the float64 kernels whose values they differentiate.
#include "adjoint.cuh"
#include "pxb_launch.h"

namespace pxb {

static dim3 adj_grid(int ny, int nx) { return dim3((nx + 31) / 32, (ny + 7) / 8); }

cudaError_t launch_adj_store(int ny, int nx, long long pitch, double scale, const double* const o[5], double* const S[5],
                             double* const A[5], cudaStream_t s) {
    adj_store_kernel<<<adj_grid(ny, nx), dim3(32, 8), 0, s>>>(ny, nx, pitch, scale, o[0], o[1], o[2], o[3], o[4], S[0],
                                                             S[1], S[2], S[3], S[4], A ? A[0] : nullptr,
                                                             A ? A[1] : nullptr, A ? A[2] : nullptr,
                                                             A ? A[3] : nullptr, A ? A[4] : nullptr);
    return cudaGetLastError();
}

cudaError_t launch_adj_stage(const AdjArgs& a, int phase, cudaStream_t s) {
    const dim3 g = adj_grid(a.ny, a.nx), b(32, 8);
    switch (phase) {
        case 0: adj_exner_kernel<<<g, b, 0, s>>>(a); break;
        case 1:
            if (a.tbar) adj_grass_kernel<true><<<g, b, 0, s>>>(a);
            else adj_grass_kernel<false><<<g, b, 0, s>>>(a);
            break;
        case 2: adj_corr_kernel<<<g, b, 0, s>>>(a); break;
        default:
            if (a.nbbar) adj_hydro_kernel<true><<<g, b, 0, s>>>(a);
            else adj_hydro_kernel<false><<<g, b, 0, s>>>(a);
            break;
    }
    return cudaGetLastError();
}

cudaError_t launch_adj_compute_n(int ny, int nx, long long pitch, int mpm, const double* zb, double* nbbar,
                                 double* nbar, double* npbar, cudaStream_t s) {
    adj_compute_n_kernel<<<adj_grid(ny, nx), dim3(32, 8), 0, s>>>(ny, nx, pitch, mpm, zb, nbbar, nbar, npbar);
    return cudaGetLastError();
}

cudaError_t launch_adj_bc(const AdjBcArgs& a, cudaStream_t s) {
    if (a.count <= 0) return cudaSuccess;
    const int g = (a.count + 255) / 256;
    adj_bc_read_kernel<<<g, 256, 0, s>>>(a);
    adj_bc_zero_kernel<<<g, 256, 0, s>>>(a);
    adj_bc_scatter_kernel<<<g, 256, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_adj_cfl(const AdjCflArgs& a, cudaStream_t s) {
    const dim3 g = adj_grid(a.ny, a.nx), b(32, 8);
    adj_cfl_max_kernel<<<g, b, 0, s>>>(a, 0);
    adj_cfl_max_kernel<<<g, b, 0, s>>>(a, 1);
    adj_cfl_grad_kernel<<<g, b, 0, s>>>(a);
    return cudaGetLastError();
}

}  // namespace pxb
