// Dual-number (tangent-linear) instantiations of the general stage path, the boundary
// handlers and the set-up kernel, and the dual CFL reduction.  Compiled with
// --fmad=false, like the float64 kernels, so the values are the float64 run's bits.
#include "kernels_impl.cuh"
#include "tangent.cuh"

namespace pxb {

cudaError_t launch_dual_cfl(const DualCflArgs& a, cudaStream_t s) {
    dim3 b(32, 8), g((a.nx + 31) / 32, (a.ny + 7) / 8);
    dual_cfl_max_kernel<<<g, b, 0, s>>>(a);
    dual_cfl_arg_kernel<<<g, b, 0, s>>>(a);
    dual_cfl_finalize_kernel<<<1, 1, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_dual_pack(int ny, int nx, long long pitch, const double* v, const double* t, Dual* out,
                             cudaStream_t s) {
    dim3 b(32, 8), g((nx + 31) / 32, (ny + 7) / 8);
    dual_pack_kernel<<<g, b, 0, s>>>(ny, nx, pitch, v, t, out);
    return cudaGetLastError();
}

cudaError_t launch_dual_unpack(int ny, int nx, long long pitch, const Dual* in, double* v, double* t, cudaStream_t s) {
    dim3 b(32, 8), g((nx + 31) / 32, (ny + 7) / 8);
    dual_unpack_kernel<<<g, b, 0, s>>>(ny, nx, pitch, in, v, t);
    return cudaGetLastError();
}

template cudaError_t launch_re_general<Dual>(const GenArgs<Dual>&, int, cudaStream_t);
template cudaError_t launch_bc<Dual>(const BcArgs<Dual>&, cudaStream_t);
template cudaError_t launch_re_init<Dual>(const InitArgs<Dual>&, cudaStream_t);

}  // namespace pxb
