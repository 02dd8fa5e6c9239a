// stencil_store_bf16.cu -- instantiations of the order-8 step kernels with __nv_bfloat16 wavefield storage.
#include "stencil.cuh"
#include "stencil_tma_impl.cuh"

namespace rtmb {
namespace detail {
template cudaError_t launch_tma_store<__nv_bfloat16>(const TmaMaps &, const StepArgs &, int, bool, bool, dim3, cudaStream_t);
template cudaError_t launch_tma_batch<__nv_bfloat16>(const BatchArgs &, bool, bool, bool, int, cudaStream_t);
}  // namespace detail
}  // namespace rtmb
