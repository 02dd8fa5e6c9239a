// stencil_h5.cu -- instantiations of the fused time-step kernels for stencil order 10.
#include "stencil.cuh"
#include "stencil_impl.cuh"

namespace rtmb {
namespace detail {
template cudaError_t launch_h<5>(const StepArgs &, bool, bool, dim3, cudaStream_t);
}  // namespace detail
}  // namespace rtmb
