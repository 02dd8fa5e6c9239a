// stencil.cu -- dispatch of the fused time-step kernel: the TMA-pipelined form
// (stencil_tma_impl.cuh) when rows are 16-byte aligned, else the plain-load form (stencil_impl.cuh).
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <cstring>
#include <vector>

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
template <typename T>
cudaError_t launch_tma_batch(const BatchArgs &b, bool exact, bool img, bool img64, int blocks, cudaStream_t s);
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

template <int H, int V>
cudaError_t tma_dispatch_v(const StepArgs &a, bool exact, cudaStream_t s, bool *used) {
    using S = detail::TmaShape<H, false, float, float, V>;
    *used = false;
    auto enc = tensor_map_encoder();
    if (!enc) return cudaSuccess;
    if (a.taper_mode == kTaperAll && a.img) return cudaSuccess;  // combination without a TMA form
    // the FP32 forward forms of the TMA kernel sample no receivers (their drivers gather them from
    // the stored level): the plain-load form does it in the step
    if (!a.img && a.rec_mode != kRecNone) return cudaSuccess;
    const int nxi = a.nxe - 2 * H, nyi = a.nye - 2 * H;
    const dim3 grid((a.nze + S::TZ - 1) / S::TZ, (nyi + S::TY - 1) / S::TY, (nxi + a.chunk - 1) / a.chunk);
    detail::TmaMaps maps;
    std::memset(&maps, 0, sizeof maps);
    bool ok = encode(enc, &maps.p, a.P, a, S::SPITCH, S::SROWS) && encode(enc, &maps.pp, a.PP, a, S::TZ, S::TY) &&
              encode(enc, &maps.v, a.V, a, S::TZ, S::TY);
    if (a.img) ok = ok && encode(enc, &maps.ps, a.ps, a, S::TZ, S::TY) && encode(enc, &maps.img, a.img, a, S::TZ, S::TY);
    if (!ok) return cudaSuccess;  // fall back to the plain-load form
    *used = true;
    return detail::launch_tma_h<H>(maps, a, exact, a.taper_mode, a.img != nullptr, grid, s);
}

// The launch variants (tile shape, ring depths) serve the FP32 forms without taper at order 8; the
// others run variant 0.
template <int H>
cudaError_t tma_dispatch(const StepArgs &a, bool exact, cudaStream_t s, bool *used) {
    const int v = (H == 4 && a.taper_mode == kTaperNone && !a.tw) ? a.variant : 0;
    switch (v) {
    case 0: return tma_dispatch_v<H, 0>(a, exact, s, used);
    case 1: return tma_dispatch_v<H, 1>(a, exact, s, used);
    case 2: return tma_dispatch_v<H, 2>(a, exact, s, used);
    case 3: return tma_dispatch_v<H, 3>(a, exact, s, used);
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace

cudaError_t launch_step(const StepArgs &a, int order, bool exact, cudaStream_t s, bool allow_tma) {
    const int h = order / 2;
    const int nxi = a.nxe - 2 * h, nyi = a.nye - 2 * h;
    if (nxi <= 0 || nyi <= 0 || a.nze <= 2 * h || a.chunk <= 0) return cudaSuccess;
    dim3 grid((a.nze + kTZ - 1) / kTZ, (nyi + kTY - 1) / kTY, (nxi + a.chunk - 1) / a.chunk);
    const uintptr_t al = reinterpret_cast<uintptr_t>(a.P) | reinterpret_cast<uintptr_t>(a.PP) |
                         reinterpret_cast<uintptr_t>(a.V) | reinterpret_cast<uintptr_t>(a.img) |
                         reinterpret_cast<uintptr_t>(a.ps) | reinterpret_cast<uintptr_t>(a.Pout);
    const bool aligned = (a.nze % 4 == 0) && (al % 16 == 0);
    if (a.diff && a.store == kStoreF32) return cudaErrorInvalidValue;  // increment storage: 16-bit forms
    if (a.store != kStoreF32 || a.img64) {
        if (!storage_form_supported(order, a.nze) || al % 16 != 0 || a.store == kStoreF32)
            return cudaErrorInvalidValue;
        return store_dispatch(a, grid, s);
    }
    if (aligned && allow_tma) {
        bool used = false;
        cudaError_t e = cudaSuccess;
        switch (h) {
        case 1: e = tma_dispatch<1>(a, exact, s, &used); break;
        case 2: e = tma_dispatch<2>(a, exact, s, &used); break;
        case 3: e = tma_dispatch<3>(a, exact, s, &used); break;
        case 4: e = tma_dispatch<4>(a, exact, s, &used); break;
        default: break;  // orders above 8 use the plain-load form
        }
        if (used || e != cudaSuccess) return e;
    }
    if (a.tw) return cudaErrorInvalidValue;  // tapered storage is a form of the TMA kernel only
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

void variant_tile(int variant, int *tz, int *ty) {
    switch (variant) {
    case 1: *tz = detail::Variant<1>::TZ; *ty = detail::Variant<1>::TY; break;
    case 2: *tz = detail::Variant<2>::TZ; *ty = detail::Variant<2>::TY; break;
    case 3: *tz = detail::Variant<3>::TZ; *ty = detail::Variant<3>::TY; break;
    default: *tz = detail::Variant<0>::TZ; *ty = detail::Variant<0>::TY; break;
    }
}

cudaError_t launch_step_batch(const StepArgs *args, int nshots, int order, bool exact, cudaStream_t s) {
    static_assert(sizeof(detail::BatchArgs) <= 32000, "kernel parameters above the 32 KB limit");
    if (nshots <= 0 || nshots > detail::kMaxBatch || order != 8) return cudaErrorInvalidValue;
    auto enc = tensor_map_encoder();
    if (!enc) return cudaErrorNotSupported;
    const StepArgs &a0 = args[0];
    const bool img = a0.img != nullptr, img64 = a0.img64 != 0;
    const int store = a0.store;
    const bool st = store != kStoreF32;
    if (st) exact = false;  // the 16-bit storage forms always use the FMA arithmetic
    std::vector<detail::BatchArgs> hold(1);  // ~30 KB: kept off the stack
    detail::BatchArgs &b = hold[0];
    std::memset(&b, 0, sizeof b);
    b.nshots = nshots;
    b.coef = a0;
    const CUtensorMapDataType dt = store == kStoreF16 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16
                                   : store == kStoreBF16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16
                                                         : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
    const size_t es = st ? 2 : 4;
    int blocks = 0;
    for (int k = 0; k < nshots; ++k) {
        const StepArgs &a = args[k];
        if (a.taper_mode != kTaperNone || (a.img != nullptr) != img || a.img64 != a0.img64 || a.store != store ||
            a.chunk <= 0 || (!img && !st && a.rec_mode != kRecNone))
            return cudaErrorInvalidValue;
        if (a.nze % (st ? 8 : 4) != 0) return cudaErrorInvalidValue;
        const uintptr_t al = reinterpret_cast<uintptr_t>(a.P) | reinterpret_cast<uintptr_t>(a.PP) |
                             reinterpret_cast<uintptr_t>(a.V) | reinterpret_cast<uintptr_t>(a.img) |
                             reinterpret_cast<uintptr_t>(a.ps);
        if (al % 16) return cudaErrorInvalidValue;
        const int spitch = kTZ + 2 * (st ? 8 : 4), srows = kTY + 8;
        detail::TmaMaps &m = b.maps[k];
        bool ok = encode(enc, &m.p, a.P, a, spitch, srows, dt, es) && encode(enc, &m.pp, a.PP, a, kTZ, kTY, dt, es) &&
                  encode(enc, &m.v, a.V, a, kTZ, kTY);
        if (img)
            ok = ok && encode(enc, &m.ps, a.ps, a, kTZ, kTY, dt, es) &&
                 encode(enc, &m.img, a.img, a, kTZ, kTY,
                        img64 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, img64 ? 8 : 4);
        if (!ok) return cudaErrorInvalidValue;
        b.args[k] = a;
        const int nxi = a.nxe - 8, nyi = a.nye - 8;
        if (nxi <= 0 || nyi <= 0 || a.nze <= 8) return cudaErrorInvalidValue;
        b.gx[k] = (a.nze + kTZ - 1) / kTZ;
        b.gy[k] = (nyi + kTY - 1) / kTY;
        const int gz = (nxi + a.chunk - 1) / a.chunk;
        b.start[k] = blocks;
        blocks += b.gx[k] * b.gy[k] * gz;
    }
    b.start[nshots] = blocks;
    if (store == kStoreF16) return detail::launch_tma_batch<__half>(b, exact, img, img64, blocks, s);
    if (store == kStoreBF16) return detail::launch_tma_batch<__nv_bfloat16>(b, exact, img, img64, blocks, s);
    return detail::launch_tma_batch<float>(b, exact, img, img64, blocks, s);
}

}  // namespace rtmb
