// float64 instantiation of every kernel.  Built with --fmad=false so that each
// product and sum rounds separately, as in the reference's float64 arithmetic.
#include "kernels_impl.cuh"
namespace pxb {
PXB_INSTANTIATE(double)
}
