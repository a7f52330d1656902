// float32 instantiation of every kernel (compiled with FMA contraction on).
#include "kernels_impl.cuh"
namespace pxb {
PXB_INSTANTIATE(float)
}
