// f64.cu -- the FP64 GPU oracle: rtmb_model_shot_f64 and rtmb_migrate_shot_f64.
//
// These drivers run the reference's operator sequence one launch per operator, as the reference's
// own time loops do (RTMFiniteDifferencesKernel.cpp:169-216 for modeling; ..._HBC.cpp:96-364 and
// ..._RBC.cpp:54-274 for migration): taper, step, source, receivers, upper border and image, each
// in double precision.  The discrete scheme is the FP32 one: the stencil coefficients, taper
// factors, Ricker samples and v2dt2 are the FP32 values, widened, so the only difference from the
// FP32 path is the arithmetic precision.  The error of the FP32 and 16-bit forms is measured against
// these results.  Speed is not a goal here: the step kernel reads its taps straight from global
// memory.
#include <cstdarg>
#include <cstdio>
#include <utility>

#include "ctx.hpp"
#include "ops.cuh"

namespace {

struct F64Step {
    int nxe, nye, nze, h;
    double cx[rtmb::kMaxOrder + 1], cy[rtmb::kMaxOrder + 1], cz[rtmb::kMaxOrder + 1];
};

// rtmStep3D (RTMCPUPlatform.cpp:325-395) in double: the x, y and z sums accumulate from zero in tap
// order, lap = (x + y) + z, PP = (2 P - PP) + v2dt2 * lap.  One thread per point of [h, n-h)^3.
__global__ void f64_step_kernel(const double *__restrict__ P, double *PP, const float *__restrict__ V, F64Step s,
                                unsigned *err) {
    const int z = blockIdx.x * blockDim.x + threadIdx.x + s.h;
    const int y = blockIdx.y + s.h;
    const int x = blockIdx.z + s.h;
    if (z >= s.nze - s.h) return;
    const size_t plane = (size_t)s.nye * s.nze;
    const size_t o = ((size_t)x * s.nye + y) * s.nze + z;
    double ax = 0.0, ay = 0.0, az = 0.0;
    const int order = 2 * s.h;
    for (int io = 0; io <= order; ++io) {
        ax = ax + P[o + (long long)(io - s.h) * (long long)plane] * s.cx[io];
        ay = ay + P[o + (long long)(io - s.h) * s.nze] * s.cy[io];
        az = az + P[o + (io - s.h)] * s.cz[io];
    }
    const double lap = (ax + ay) + az;
    const double r = (2.0 * P[o] - PP[o]) + (double)V[o] * lap;
    PP[o] = r;
    if (r != r && err) atomicOr(err, 1u);
}

int fail64(rtmb_ctx *c, int code, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    c->err = buf;
    return code;
}

#define CK64(call)                                                                                \
    do {                                                                                          \
        cudaError_t e_ = (call);                                                                  \
        if (e_ != cudaSuccess)                                                                    \
            return fail64(ctx, e_ == cudaErrorMemoryAllocation ? RTMB_ENOMEM : RTMB_ECUDA, "%s: %s (%s:%d)", \
                          #call, cudaGetErrorString(e_), __FILE__, __LINE__);                     \
    } while (0)

#define LAUNCH64(call)                                                                            \
    do {                                                                                          \
        ++ctx->launches;                                                                          \
        CK64(call);                                                                               \
    } while (0)

rtmb::Geom geom64(const rtmb_ctx *c) { return rtmb::Geom{c->nxe, c->nye, c->nze, (int)c->p.blen, c->h}; }

rtmb::RcvGeom rgeom64(const rtmb_ctx *c) {
    const int b = (int)c->p.blen;
    return rtmb::RcvGeom{(int)c->p.receiver_start_x + b, (int)c->p.receiver_start_y + b,
                         (int)c->p.receiver_depth_z + b, (int)c->p.receiver_distance_x,
                         (int)c->p.receiver_distance_y, (int)c->p.receiver_count_x,
                         (int)c->p.receiver_count_y, (int)c->p.ntstep};
}

F64Step step_args(const rtmb_ctx *c) {
    F64Step s{};
    s.nxe = c->nxe; s.nye = c->nye; s.nze = c->nze; s.h = c->h;
    const int o = (int)c->p.stencil_order;
    for (int i = 0; i <= o; ++i) {
        s.cx[i] = c->coefs[i];
        s.cy[i] = c->coefs[(o + 1) + i];
        s.cz[i] = c->coefs[2 * (o + 1) + i];
    }
    return s;
}

cudaError_t step64(const rtmb_ctx *c, const double *P, double *PP) {
    const F64Step s = step_args(c);
    const int nzi = c->nze - 2 * c->h, nyi = c->nye - 2 * c->h, nxi = c->nxe - 2 * c->h;
    if (nzi <= 0 || nyi <= 0 || nxi <= 0) return cudaSuccess;
    dim3 grid((nzi + 127) / 128, nyi, nxi);
    f64_step_kernel<<<grid, 128, 0, c->stream>>>(P, PP, c->d_v2dt2, s, c->d_err);
    return cudaGetLastError();
}

int alloc64(rtmb_ctx *ctx, int count) {
    for (int k = 0; k < count; ++k)
        if (!ctx->d_f64[k]) CK64(cudaMalloc(&ctx->d_f64[k], ctx->n * sizeof(double)));
    return RTMB_OK;
}

int check64(rtmb_ctx *ctx, uint32_t sx, uint32_t sy, uint32_t sz) {
    const rtmb_params &p = ctx->p;
    if (sx >= p.nx || sy >= p.ny || sz >= p.nz)
        return fail64(ctx, RTMB_EINVAL, "Invalid Source Position: (%u,%u,%u)", sx, sy, sz);
    if (!ctx->d_v2dt2) return fail64(ctx, RTMB_EINVAL, "no velocity loaded (rtmb_load_v2dt2)");
    if ((int)p.blen < ctx->h) return fail64(ctx, RTMB_EINVAL, "the per-shot drivers need blen >= stencil_order/2");
    if (p.nx == 1) return fail64(ctx, RTMB_EINVAL, "the FP64 oracle runs 3D models only (nx > 1)");
    if (p.receiver_count_x > p.nx || p.receiver_count_y > p.ny)
        return fail64(ctx, RTMB_EINVAL, "Invalid Receiver Grid Size");
    if (p.receiver_depth_z + p.blen >= (uint32_t)ctx->nze - ctx->h)
        return fail64(ctx, RTMB_EINVAL, "receiver depth outside the computed region");
    return RTMB_OK;
}

}  // namespace

extern "C" {

int rtmb_model_shot_f64(rtmb_ctx *ctx, uint32_t sx, uint32_t sy, uint32_t sz, double *rec) {
    if (!ctx || !rec) return ctx ? fail64(ctx, RTMB_EINVAL, "rtmb_model_shot_f64: null pointer") : RTMB_EINVAL;
    int rc = check64(ctx, sx, sy, sz);
    if (rc || (rc = alloc64(ctx, 2))) return rc;
    const rtmb_params &p = ctx->p;
    const rtmb::Geom g = geom64(ctx);
    const rtmb::RcvGeom r = rgeom64(ctx);
    const int quirk = !(p.flags & RTMB_FLAG_NO_TAPER_QUIRK);
    const size_t chunk = (size_t)p.receiver_count_x * p.receiver_count_y * p.ntstep;
    double *P = ctx->d_f64[0], *PP = ctx->d_f64[1];
    CK64(cudaMemsetAsync(P, 0, ctx->n * sizeof(double), ctx->stream));
    CK64(cudaMemsetAsync(PP, 0, ctx->n * sizeof(double), ctx->stream));
    const int b = (int)p.blen;
    // RTMFiniteDifferencesKernel.cpp:169-216
    for (uint32_t it = 0; it < p.nt; ++it) {
        const uint32_t lt = it % p.ntstep;
        std::swap(P, PP);
        LAUNCH64(rtmb::launch_taper(P, ctx->d_taper, g, 0, quirk, ctx->stream));
        LAUNCH64(rtmb::launch_taper(PP, ctx->d_taper, g, 0, quirk, ctx->stream));
        LAUNCH64(step64(ctx, P, PP));
        LAUNCH64(rtmb::launch_source(PP, ctx->d_wavelet, (int)it, (int)sx + b, (int)sy + b, (int)sz + b, g,
                                     ctx->stream));
        LAUNCH64(rtmb::launch_receivers(PP, rec + (size_t)(it / p.ntstep) * chunk, (int)lt, 1, r, g, ctx->stream));
    }
    return rtmb::driver::check_err_flag(ctx);
}

int rtmb_migrate_shot_f64(rtmb_ctx *ctx, uint32_t sx, uint32_t sy, uint32_t sz, const float *rec, double *img) {
    if (!ctx || !rec || !img) return ctx ? fail64(ctx, RTMB_EINVAL, "rtmb_migrate_shot_f64: null pointer") : RTMB_EINVAL;
    int rc = check64(ctx, sx, sy, sz);
    if (rc || (rc = alloc64(ctx, 4))) return rc;
    const rtmb_params &p = ctx->p;
    if (p.boundary != RTMB_BC_HBC && p.boundary != RTMB_BC_RBC)
        return fail64(ctx, RTMB_EINVAL, "migration boundary must be HBC or RBC");
    const bool hbc = p.boundary == RTMB_BC_HBC;
    const rtmb::Geom g = geom64(ctx);
    const rtmb::RcvGeom r = rgeom64(ctx);
    const size_t upb_step = (size_t)ctx->nxe * ctx->nye * ctx->h;
    if (hbc && !ctx->d_upb64) CK64(cudaMalloc(&ctx->d_upb64, upb_step * p.nt * sizeof(double)));
    const int b = (int)p.blen;
    double *P = ctx->d_f64[0], *PP = ctx->d_f64[1];
    CK64(cudaMemsetAsync(P, 0, ctx->n * sizeof(double), ctx->stream));
    CK64(cudaMemsetAsync(PP, 0, ctx->n * sizeof(double), ctx->stream));
    // forward pass (HBC.cpp:96-210 / RBC.cpp:54-144)
    for (uint32_t it = 0; it < p.nt; ++it) {
        std::swap(P, PP);
        if (hbc) {
            LAUNCH64(rtmb::launch_taper(P, ctx->d_taper, g, 1, 0, ctx->stream));
            LAUNCH64(rtmb::launch_taper(PP, ctx->d_taper, g, 1, 0, ctx->stream));
        }
        LAUNCH64(step64(ctx, P, PP));
        LAUNCH64(rtmb::launch_source(PP, ctx->d_wavelet, (int)it, (int)sx + b, (int)sy + b, (int)sz + b, g,
                                     ctx->stream));
        if (hbc) LAUNCH64(rtmb::launch_upb(PP, ctx->d_upb64 + (size_t)it * upb_step, 0, 1, g, ctx->stream));
    }
    // backward pass (HBC.cpp:212-364 / RBC.cpp:146-274).  The source pair continues in place: the
    // reference copies snap1 (= PP) and snap0 (= P) back into its buffers, which these already are.
    double *S = P, *SS = PP;  // S = snap0 = u(nt-1), SS = snap1 = u(nt)
    double *PR = ctx->d_f64[2], *PPR = ctx->d_f64[3];
    CK64(cudaMemsetAsync(PR, 0, ctx->n * sizeof(double), ctx->stream));
    CK64(cudaMemsetAsync(PPR, 0, ctx->n * sizeof(double), ctx->stream));
    CK64(cudaMemsetAsync(img, 0, ctx->n * sizeof(double), ctx->stream));
    const bool full = p.flags & RTMB_FLAG_IMG_FULL_Z;
    const int z0 = full ? 0 : b, z1 = full ? ctx->nze : ctx->nze - b;
    const int rmode = (p.flags & RTMB_FLAG_RCV_ADD) ? 3 : 2;
    const size_t chunk = (size_t)p.receiver_count_x * p.receiver_count_y * p.ntstep;
    // the reference's (P, PP) of the backward loop: after the SWAP each iteration P is the source
    // wavefield at time it
    double *BP = SS, *BPP = S;  // as if PP = snap1 had just been swapped into P at it = nt-1
    for (int it = (int)p.nt - 1; it >= 0; --it) {
        const int lt = it % (int)p.ntstep;
        if (it == (int)p.nt - 1) {
            BP = SS; BPP = S;
        } else if (it == (int)p.nt - 2) {
            BP = S; BPP = SS;
        } else {
            // step(P, PP) then SWAP: the new level lands in PP and becomes P
            LAUNCH64(step64(ctx, BP, BPP));
            if (hbc) LAUNCH64(rtmb::launch_upb(BPP, ctx->d_upb64 + (size_t)it * upb_step, 0, 0, g, ctx->stream));
            std::swap(BP, BPP);
        }
        if (hbc) {
            LAUNCH64(rtmb::launch_taper(PR, ctx->d_taper, g, 1, 0, ctx->stream));
            LAUNCH64(rtmb::launch_taper(PPR, ctx->d_taper, g, 1, 0, ctx->stream));
        }
        LAUNCH64(step64(ctx, PR, PPR));
        LAUNCH64(rtmb::launch_receivers(PPR, const_cast<float *>(rec) + (size_t)(it / p.ntstep) * chunk, lt, rmode,
                                        r, g, ctx->stream));
        LAUNCH64(rtmb::launch_image(img, BP, PPR, z0, z1, g, ctx->stream));
        std::swap(PR, PPR);
    }
    return rtmb::driver::check_err_flag(ctx);
}

}  // extern "C"
