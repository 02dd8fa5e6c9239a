// stencil.cu -- dispatch of the fused time-step kernel: the TMA-pipelined form
// (stencil_tma_impl.cuh) when rows are 16-byte aligned, else the plain-load form (stencil_impl.cuh).
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <cstring>

#include "stencil.cuh"
#include "stencil_tma_impl.cuh"

namespace rtmb {
namespace detail {
template <int H>
cudaError_t launch_h(const StepArgs &a, bool exact, bool aligned, dim3 grid, cudaStream_t s);
template <int H>
cudaError_t launch_tma_h(const TmaMaps &maps, const StepArgs &a, bool exact, int taper, bool img, dim3 grid,
                         cudaStream_t s);
template <typename T>
cudaError_t launch_tma_store(const TmaMaps &maps, const StepArgs &a, int taper, bool img, bool img64, dim3 grid,
                             cudaStream_t s);
}  // namespace detail

namespace {

PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}

// Map of one padded volume of element type dt (esize bytes) with a box of box_z x box_y x 1.
bool encode(PFN_cuTensorMapEncodeTiled_v12000 enc, CUtensorMap *m, const void *base, const StepArgs &a,
            int box_z, int box_y, CUtensorMapDataType dt = CU_TENSOR_MAP_DATA_TYPE_FLOAT32, size_t esize = 4) {
    const cuuint64_t dims[3] = {(cuuint64_t)a.nze, (cuuint64_t)a.nye, (cuuint64_t)a.nxe};
    const cuuint64_t strides[2] = {(cuuint64_t)a.nze * esize, (cuuint64_t)a.nye * a.nze * esize};
    const cuuint32_t box[3] = {(cuuint32_t)box_z, (cuuint32_t)box_y, 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    return enc(m, dt, 3, const_cast<void *>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
               CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// The 16-bit storage forms: order 8 only, always TMA (there is no plain-load 16-bit form).
cudaError_t store_dispatch(const StepArgs &a, dim3 grid, cudaStream_t s) {
    using S = detail::TmaShape<4, false, __half>;
    auto enc = tensor_map_encoder();
    if (!enc) return cudaErrorNotSupported;
    if (a.taper_mode == kTaperAll && a.img) return cudaErrorInvalidValue;
    const CUtensorMapDataType dt =
        a.store == kStoreF16 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16 : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16;
    detail::TmaMaps maps;
    std::memset(&maps, 0, sizeof maps);
    bool ok = encode(enc, &maps.p, a.P, a, S::SPITCH, S::SROWS, dt, 2) && encode(enc, &maps.pp, a.PP, a, kTZ, kTY, dt, 2) &&
              encode(enc, &maps.v, a.V, a, kTZ, kTY);
    if (a.img)
        ok = ok && encode(enc, &maps.ps, a.ps, a, kTZ, kTY, dt, 2) &&
             encode(enc, &maps.img, a.img, a, kTZ, kTY,
                    a.img64 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, a.img64 ? 8 : 4);
    if (!ok) return cudaErrorInvalidValue;
    if (a.store == kStoreF16)
        return detail::launch_tma_store<__half>(maps, a, a.taper_mode, a.img != nullptr, a.img64 != 0, grid, s);
    return detail::launch_tma_store<__nv_bfloat16>(maps, a, a.taper_mode, a.img != nullptr, a.img64 != 0, grid, s);
}

template <int H>
cudaError_t tma_dispatch(const StepArgs &a, bool exact, dim3 grid, cudaStream_t s, bool *used) {
    using S = detail::TmaShape<H, false>;
    *used = false;
    auto enc = tensor_map_encoder();
    if (!enc) return cudaSuccess;
    if (a.taper_mode == kTaperAll && a.img) return cudaSuccess;  // combination without a TMA form
    detail::TmaMaps maps;
    std::memset(&maps, 0, sizeof maps);
    bool ok = encode(enc, &maps.p, a.P, a, S::SPITCH, S::SROWS) && encode(enc, &maps.pp, a.PP, a, kTZ, kTY) &&
              encode(enc, &maps.v, a.V, a, kTZ, kTY);
    if (a.img) ok = ok && encode(enc, &maps.ps, a.ps, a, kTZ, kTY) && encode(enc, &maps.img, a.img, a, kTZ, kTY);
    if (!ok) return cudaSuccess;  // fall back to the plain-load form
    *used = true;
    return detail::launch_tma_h<H>(maps, a, exact, a.taper_mode, a.img != nullptr, grid, s);
}

}  // namespace

cudaError_t launch_step(const StepArgs &a, int order, bool exact, cudaStream_t s, bool allow_tma) {
    const int h = order / 2;
    const int nxi = a.nxe - 2 * h, nyi = a.nye - 2 * h;
    if (nxi <= 0 || nyi <= 0 || a.nze <= 2 * h || a.chunk <= 0) return cudaSuccess;
    dim3 grid((a.nze + kTZ - 1) / kTZ, (nyi + kTY - 1) / kTY, (nxi + a.chunk - 1) / a.chunk);
    const uintptr_t al = reinterpret_cast<uintptr_t>(a.P) | reinterpret_cast<uintptr_t>(a.PP) |
                         reinterpret_cast<uintptr_t>(a.V) | reinterpret_cast<uintptr_t>(a.img) |
                         reinterpret_cast<uintptr_t>(a.ps);
    const bool aligned = (a.nze % 4 == 0) && (al % 16 == 0);
    if (a.store != kStoreF32 || a.img64) {
        if (!storage_form_supported(order, a.nze) || al % 16 != 0 || a.store == kStoreF32)
            return cudaErrorInvalidValue;
        return store_dispatch(a, grid, s);
    }
    if (aligned && allow_tma) {
        bool used = false;
        cudaError_t e = cudaSuccess;
        switch (h) {
        case 1: e = tma_dispatch<1>(a, exact, grid, s, &used); break;
        case 2: e = tma_dispatch<2>(a, exact, grid, s, &used); break;
        case 3: e = tma_dispatch<3>(a, exact, grid, s, &used); break;
        case 4: e = tma_dispatch<4>(a, exact, grid, s, &used); break;
        default: break;  // orders above 8 use the plain-load form
        }
        if (used || e != cudaSuccess) return e;
    }
    switch (h) {
    case 1: return detail::launch_h<1>(a, exact, aligned, grid, s);
    case 2: return detail::launch_h<2>(a, exact, aligned, grid, s);
    case 3: return detail::launch_h<3>(a, exact, aligned, grid, s);
    case 4: return detail::launch_h<4>(a, exact, aligned, grid, s);
    case 5: return detail::launch_h<5>(a, exact, aligned, grid, s);
    case 6: return detail::launch_h<6>(a, exact, aligned, grid, s);
    case 7: return detail::launch_h<7>(a, exact, aligned, grid, s);
    case 8: return detail::launch_h<8>(a, exact, aligned, grid, s);
    default: return cudaErrorInvalidValue;
    }
}

bool storage_form_supported(int order, int nze) { return order == 8 && nze % 8 == 0; }

}  // namespace rtmb
