// stencil_dual.cu -- host side of the dual-wavefield backward step (stencil_dual_impl.cuh).
#include <cudaTypedefs.h>

#include <cstring>

#include "stencil.cuh"
#include "stencil_dual_impl.cuh"

namespace rtmb {
namespace {

PFN_cuTensorMapEncodeTiled_v12000 dual_encoder() {
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

bool encode_f32(PFN_cuTensorMapEncodeTiled_v12000 enc, CUtensorMap *m, const float *base, const StepArgs &a, int bz,
                int by) {
    const cuuint64_t dims[3] = {(cuuint64_t)a.nze, (cuuint64_t)a.nye, (cuuint64_t)a.nxe};
    const cuuint64_t strides[2] = {(cuuint64_t)a.nze * 4, (cuuint64_t)a.nye * a.nze * 4};
    const cuuint32_t box[3] = {(cuuint32_t)bz, (cuuint32_t)by, 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    return enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float *>(base), dims, strides, box, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

}  // namespace

bool dual_step_supported(const StepArgs &src, const StepArgs &rcv, int order) {
    const uintptr_t al = reinterpret_cast<uintptr_t>(src.P) | reinterpret_cast<uintptr_t>(src.PP) |
                         reinterpret_cast<uintptr_t>(rcv.P) | reinterpret_cast<uintptr_t>(rcv.PP) |
                         reinterpret_cast<uintptr_t>(rcv.V) | reinterpret_cast<uintptr_t>(rcv.img);
    return order == 8 && rcv.nze % 4 == 0 && al % 16 == 0 && src.store == kStoreF32 && rcv.store == kStoreF32 &&
           !rcv.img64 && rcv.img && src.taper_mode == kTaperNone &&
           rcv.taper_mode == kTaperNone && src.upb_mode == kUpbNone && src.V == rcv.V &&
           (rcv.rec_mode == kRecOverwrite || rcv.rec_mode == kRecAdd || rcv.rec_mode == kRecNone) &&
           dual_encoder() != nullptr;
}

namespace {

template <int DV>
cudaError_t launch_dual_v(const StepArgs &src, const StepArgs &rcv, bool exact, cudaStream_t s) {
    using S = detail::DualShape<4, DV>;
    constexpr int TZ = S::TZ, TY = S::TY;
    auto enc = dual_encoder();
    detail::DualMaps m;
    std::memset(&m, 0, sizeof m);
    const bool ok = encode_f32(enc, &m.ps, src.P, rcv, S::SPITCH, S::SROWS) &&
                    encode_f32(enc, &m.pr, rcv.P, rcv, S::SPITCH, S::SROWS) &&
                    encode_f32(enc, &m.pps, src.PP, rcv, TZ, TY) && encode_f32(enc, &m.ppr, rcv.PP, rcv, TZ, TY) &&
                    encode_f32(enc, &m.v, rcv.V, rcv, TZ, TY) && encode_f32(enc, &m.img, rcv.img, rcv, TZ, TY);
    if (!ok) return cudaErrorInvalidValue;
    detail::DualArgs d;
    d.s = src;
    d.r = rcv;
    d.s.chunk = rcv.chunk;
    const int nxi = rcv.nxe - 8, nyi = rcv.nye - 8;
    if (nxi <= 0 || nyi <= 0 || rcv.nze <= 8) return cudaSuccess;
    dim3 grid((rcv.nze + TZ - 1) / TZ, (nyi + TY - 1) / TY, (nxi + rcv.chunk - 1) / rcv.chunk);
    return detail::launch_dual_h<4>(m, d, exact, rcv.taper_mode, DV, grid, s);
}

}  // namespace

// rcv.variant selects the dual step's launch variant (0: 64 x 8 tiles, 1: 32 x 16, 2 and 3: 32 x 16
// with deeper rings, 4 to 7: the merged form on 64 x 8, 32 x 16, 64 x 16 and 32 x 32 tiles).
cudaError_t launch_dual_step(const StepArgs &src, const StepArgs &rcv, int order, bool exact, cudaStream_t s) {
    if (!dual_step_supported(src, rcv, order) || rcv.chunk <= 0) return cudaErrorInvalidValue;
    if (rcv.img_pair != 0 && (rcv.variant < 4 || rcv.img_pair > 2)) return cudaErrorInvalidValue;  // merged form only
    switch (rcv.variant) {
    case 0: return launch_dual_v<0>(src, rcv, exact, s);
    case 1: return launch_dual_v<1>(src, rcv, exact, s);
    case 2: return launch_dual_v<2>(src, rcv, exact, s);
    case 3: return launch_dual_v<3>(src, rcv, exact, s);
    case 4: return launch_dual_v<4>(src, rcv, exact, s);
    case 5: return launch_dual_v<5>(src, rcv, exact, s);
    case 6: return launch_dual_v<6>(src, rcv, exact, s);
    case 7: return launch_dual_v<7>(src, rcv, exact, s);
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace rtmb
