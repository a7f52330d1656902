// Float64 instantiation of the allocation-free CFL kernel, compiled with --fmad=false
// like the other float64 kernels so that its face speeds round exactly as pxb_re_cfl's.
#include "noalloc_kernel.cuh"

namespace pxb {
template cudaError_t launch_cfl_noalloc<double>(const CflArgs<double>&, unsigned long long*, unsigned int*, int,
                                                cudaStream_t);
}  // namespace pxb
