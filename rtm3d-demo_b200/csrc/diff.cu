// diff.cu -- the pointwise step of the increment storage form (RTMB_FLAG_STORE_DIFF): the turn from
// the forward pass to the backward source reconstruction.
#include <algorithm>

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "ops.cuh"
#include "stencil_tma_impl.cuh"

namespace rtmb {
namespace {

// The forward pass ends in (p(nt), d(nt) = p(nt) - p(nt-1)); the reconstruction runs the same
// step backwards in time from (p(nt-1), p(nt-1) - p(nt)) = (p(nt) - d(nt), -d(nt)).  pout receives
// p(nt-1) with its own exponent (bound: max|p| + max|d|), d is negated in place (a sign flip, exact:
// its record is unchanged).  Eight values per thread and iteration (n % 8 == 0: z rows of a
// multiple of 8 values).
template <typename T>
__global__ void __launch_bounds__(256) diff_rewind_kernel(const T *__restrict__ p, T *__restrict__ d, T *__restrict__ pout,
                                                          const ScaleRec *sp, const ScaleRec *sd, ScaleRec *so,
                                                          size_t n8) {
    using ST = detail::Stor<T>;
    const ScaleRec rp = *sp, rd = *sd;
    const int e = storage_exponent(__uint_as_float(rp.amax) + __uint_as_float(rd.amax));
    const float s_p = detail::exp2i(rp.e), s_d = detail::exp2i(rd.e), inv = detail::exp2i(-e);
    if (blockIdx.x == 0 && threadIdx.x == 0) so->e = e;
    float m = 0.f;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n8; i += (size_t)gridDim.x * blockDim.x) {
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const size_t k = 8 * i + 4 * h;
            const float4 pv = ST::ld4(p + k), dv = ST::ld4(d + k);
            float4 o, nd;
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                const float v = detail::get(pv, c) * s_p - detail::get(dv, c) * s_d;
                m = fmaxf(m, fabsf(v));
                detail::put(o, c, v * inv);
                detail::put(nd, c, -detail::get(dv, c));
            }
            ST::st4(pout + k, o);
            ST::st4(d + k, nd);
        }
    }
    const unsigned mm = __reduce_max_sync(0xffffffffu, __float_as_uint(m));
    if ((threadIdx.x & 31) == 0 && mm) atomicMax(&so->amax, mm);
}

}  // namespace

cudaError_t launch_diff_rewind(int store, const void *p, void *d, void *pout, const ScaleRec *sp, const ScaleRec *sd,
                               ScaleRec *so, size_t n, cudaStream_t s) {
    if (n % 8) return cudaErrorInvalidValue;
    const size_t n8 = n / 8;
    const int blocks = (int)std::min<size_t>((n8 + 255) / 256, 148 * 16);
    if (blocks == 0) return cudaSuccess;
    if (store == kStoreF16)
        diff_rewind_kernel<__half><<<blocks, 256, 0, s>>>(static_cast<const __half *>(p), static_cast<__half *>(d),
                                                          static_cast<__half *>(pout), sp, sd, so, n8);
    else if (store == kStoreBF16)
        diff_rewind_kernel<__nv_bfloat16><<<blocks, 256, 0, s>>>(static_cast<const __nv_bfloat16 *>(p),
                                                                 static_cast<__nv_bfloat16 *>(d),
                                                                 static_cast<__nv_bfloat16 *>(pout), sp, sd, so, n8);
    else
        return cudaErrorInvalidValue;
    return cudaGetLastError();
}

}  // namespace rtmb
