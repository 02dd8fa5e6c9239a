// stencil_store_f16.cu -- instantiations of the order-8 step kernels with __half wavefield storage.
#include "stencil.cuh"
#include "stencil_tma_impl.cuh"

namespace rtmb {
namespace detail {
template cudaError_t launch_tma_store<__half>(const TmaMaps &, const StepArgs &, int, bool, bool, dim3, cudaStream_t);
template cudaError_t launch_tma_batch<__half>(const BatchArgs &, bool, bool, bool, int, cudaStream_t);
}  // namespace detail
}  // namespace rtmb
