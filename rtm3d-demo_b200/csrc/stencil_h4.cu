// stencil_h4.cu -- instantiations of the fused time-step kernels for stencil order 8.
#include "stencil.cuh"
#include "stencil_impl.cuh"
#include "stencil_tma_impl.cuh"

namespace rtmb {
namespace detail {
template cudaError_t launch_h<4>(const StepArgs &, bool, bool, dim3, cudaStream_t);
template cudaError_t launch_tma_h<4>(const TmaMaps &, const StepArgs &, bool, int, bool, dim3, cudaStream_t);
template cudaError_t launch_tma_batch<float>(const BatchArgs &, bool, bool, bool, int, cudaStream_t);
}  // namespace detail
}  // namespace rtmb
