// stencil_h7.cu -- instantiations of the fused time-step kernels for stencil order 14.
#include "stencil.cuh"
#include "stencil_impl.cuh"

namespace rtmb {
namespace detail {
template cudaError_t launch_h<7>(const StepArgs &, bool, bool, dim3, cudaStream_t);
}  // namespace detail
}  // namespace rtmb
