// api.cu -- context, C ABI entry points and the per-shot time-loop drivers of librtm3d_b200.
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <utility>
#include <vector>

#include <cuda_runtime.h>

#include "ctx.hpp"
#include "ops.cuh"

namespace {

int fail(rtmb_ctx *c, int code, const char *fmt, ...) {
    if (c) {
        char buf[512];
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(buf, sizeof buf, fmt, ap);
        va_end(ap);
        c->err = buf;
    }
    return code;
}

#define CK(call)                                                                                  \
    do {                                                                                          \
        cudaError_t e_ = (call);                                                                  \
        if (e_ != cudaSuccess)                                                                    \
            return fail(ctx, e_ == cudaErrorMemoryAllocation ? RTMB_ENOMEM : RTMB_ECUDA, "%s: %s (%s:%d)", \
                        #call, cudaGetErrorString(e_), __FILE__, __LINE__);                       \
    } while (0)

#define LAUNCH(call)                                                                              \
    do {                                                                                          \
        ++ctx->launches;                                                                          \
        CK(call);                                                                                 \
    } while (0)

// A driver launch of category CAT, bracketed by profiling events when rtmb_profile is on.
#define LAUNCH_CAT(CAT, call)                                                                     \
    do {                                                                                          \
        const size_t slot_ = prof_begin(ctx, CAT);                                                \
        LAUNCH(call);                                                                             \
        prof_end(ctx, slot_);                                                                     \
    } while (0)

size_t prof_begin(rtmb_ctx *c, int cat) {
    if (!c->prof || c->capturing) return (size_t)-1;
    if (c->ev_used + 2 > c->ev.size()) {
        for (int k = 0; k < 256; ++k) {
            cudaEvent_t e;
            if (cudaEventCreate(&e) != cudaSuccess) return (size_t)-1;
            c->ev.push_back(e);
        }
        c->ev_cat.resize(c->ev.size() / 2);
    }
    const size_t slot = c->ev_used / 2;
    c->ev_cat[slot] = cat;
    cudaEventRecord(c->ev[c->ev_used], c->stream);
    c->ev_used += 2;
    return slot;
}

void prof_end(rtmb_ctx *c, size_t slot) {
    if (slot != (size_t)-1) cudaEventRecord(c->ev[2 * slot + 1], c->stream);
}

// After a stream synchronisation: fold the recorded event pairs into the per-category totals.
void prof_collect(rtmb_ctx *c) {
    for (size_t s = 0; s < c->ev_used / 2; ++s) {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, c->ev[2 * s], c->ev[2 * s + 1]) == cudaSuccess) {
            c->prof_ms[c->ev_cat[s]] += ms;
            c->prof_n[c->ev_cat[s]] += 1;
        }
    }
    c->ev_used = 0;
}

rtmb::Geom geom(const rtmb_ctx *c) { return rtmb::Geom{c->nxe, c->nye, c->nze, (int)c->p.blen, c->h}; }

rtmb::RcvGeom rgeom(const rtmb_ctx *c) {
    const int b = (int)c->p.blen;
    return rtmb::RcvGeom{(int)c->p.receiver_start_x + b, (int)c->p.receiver_start_y + b,
                         (int)c->p.receiver_depth_z + b, (int)c->p.receiver_distance_x,
                         (int)c->p.receiver_distance_y, (int)c->p.receiver_count_x,
                         (int)c->p.receiver_count_y, (int)c->p.ntstep};
}

// x planes per CTA: enough CTAs for several waves of 2 CTAs per SM on 148 SMs.
int pick_chunk(int nxi, int tiles) {
    const int target = 148 * 2 * 4;
    int nch = (target + tiles - 1) / tiles;
    const int maxch = nxi / 16 > 0 ? nxi / 16 : 1;
    if (nch > maxch) nch = maxch;
    if (nch < 1) nch = 1;
    return (nxi + nch - 1) / nch;
}

rtmb::StepArgs base_args(const rtmb_ctx *c) {
    rtmb::StepArgs a;
    std::memset(&a, 0, sizeof a);
    a.nxe = c->nxe; a.nye = c->nye; a.nze = c->nze; a.blen = (int)c->p.blen;
    a.chunk = c->chunk;
    a.variant = c->variant;
    const int o = (int)c->p.stencil_order;
    a.iso = 1;
    for (int i = 0; i <= o; ++i) {
        a.cx[i] = c->coefs[i];
        a.cy[i] = c->coefs[(o + 1) + i];
        a.cz[i] = c->coefs[2 * (o + 1) + i];
        a.iso &= a.cx[i] == a.cy[i] && a.cx[i] == a.cz[i] && c->coefs[i] == c->coefs[o - i];
    }
    if (c->p.nx == 1) {  // RTMCPUPlatform.cpp:191-256 (rtmStep2D): the plane x = blen, no x term
        for (int i = 0; i <= o; ++i) a.cx[i] = 0.f;
        a.iso = 0;
        a.x_lo = (int)c->p.blen;
        a.x_hi = (int)c->p.blen + 1;
    }
    a.taper = c->d_taper;
    a.wavelet = c->d_wavelet;
    a.sxe = a.sye = a.sze = -1;
    a.err = c->d_err;
    a.rdx = a.rdy = 1;
    return a;
}

bool exact(const rtmb_ctx *c) { return !(c->p.flags & RTMB_FLAG_FAST_FMA); }
bool tma_ok(const rtmb_ctx *c) { return !(c->p.flags & RTMB_FLAG_NO_TMA); }

}  // namespace

int rtmb::driver::check_err_flag(rtmb_ctx *ctx) {
    unsigned h = 0;
    CK(cudaMemcpyAsync(&h, ctx->d_err, sizeof h, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (ctx->prof) prof_collect(ctx);
    if (h) {
        CK(cudaMemsetAsync(ctx->d_err, 0, sizeof(unsigned), ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        if (h & 2u) return fail(ctx, RTMB_ETIMEOUT, "a bounded device wait for a tile load ran out");
        return fail(ctx, RTMB_ENAN, "Numerical Dispersion: a wavefield value became NaN");
    }
    return RTMB_OK;
}

namespace {
using rtmb::driver::check_err_flag;

int ensure_bytes(rtmb_ctx *ctx, void **buf, size_t bytes, bool zero) {
    if (!*buf) {
        CK(cudaMalloc(buf, bytes));
        if (zero) CK(cudaMemsetAsync(*buf, 0, bytes, ctx->stream));
    }
    return RTMB_OK;
}

int ensure(rtmb_ctx *ctx, float **buf, size_t count, bool zero) {
    return ensure_bytes(ctx, reinterpret_cast<void **>(buf), count * sizeof(float), zero);
}

size_t wave_bytes(const rtmb_ctx *c) { return c->n * (c->store == rtmb::kStoreF32 ? sizeof(float) : 2); }

// Scale records of the storage forms: a pool of 3 nt + 8 records per shot (forward levels, rebuilt
// source levels, receiver levels), cleared at the start of each shot.
int reset_scales(rtmb_ctx *ctx) {
    const int need = (ctx->diff ? 6 : 3) * (int)ctx->p.nt + 16;  // increment storage: two records per step
    if (ctx->sc_cap < need) {
        if (ctx->d_scale) CK(cudaFree(ctx->d_scale));
        ctx->d_scale = nullptr;
        ctx->sc_cap = 0;
        CK(cudaMalloc(&ctx->d_scale, need * sizeof(rtmb::ScaleRec)));
        ctx->sc_cap = need;
    }
    CK(cudaMemsetAsync(ctx->d_scale, 0, ctx->sc_cap * sizeof(rtmb::ScaleRec), ctx->stream));
    ctx->sc_next = 0;
    return RTMB_OK;
}

rtmb::ScaleRec *new_scale(rtmb_ctx *ctx) {
    return ctx->sc_next < ctx->sc_cap ? ctx->d_scale + ctx->sc_next++ : nullptr;
}

// RTMB_FLAG_USE_GRAPH: a driver's launches between begin() and end() are captured into a CUDA graph
// on the context's stream and replayed with one cudaGraphLaunch.  The executable graph of each
// driver kind is kept and updated in place (cudaGraphExecUpdate) when the next shot's graph has
// the same shape, so a new shot re-captures (host work only) but does not re-instantiate.  Not
// used on the legacy or per-thread default streams (which cannot be captured), while profiling,
// or when the caller is already capturing the stream (the launches then go into its graph).
struct GraphScope {
    rtmb_ctx *ctx;
    int kind;
    bool active = false;
    GraphScope(rtmb_ctx *c, int k) : ctx(c), kind(k) {}
    int begin() {
        if (!(ctx->p.flags & RTMB_FLAG_USE_GRAPH) || ctx->prof || ctx->stream == cudaStreamLegacy ||
            ctx->stream == cudaStreamPerThread || ctx->stream == nullptr)
            return RTMB_OK;
        cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
        CK(cudaStreamIsCapturing(ctx->stream, &st));
        if (st != cudaStreamCaptureStatusNone) return RTMB_OK;
        CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeRelaxed));
        active = true;
        ctx->capturing = true;
        return RTMB_OK;
    }
    int end() {
        if (!active) return RTMB_OK;
        active = false;
        ctx->capturing = false;
        cudaGraph_t g = nullptr;
        CK(cudaStreamEndCapture(ctx->stream, &g));
        cudaGraphExec_t &exec = ctx->gexec[kind];
        if (exec) {
            cudaGraphExecUpdateResultInfo info;
            if (cudaGraphExecUpdate(exec, g, &info) != cudaSuccess) {
                (void)cudaGetLastError();
                cudaGraphExecDestroy(exec);
                exec = nullptr;
            }
        }
        if (!exec) {
            const cudaError_t e = cudaGraphInstantiate(&exec, g, 0);
            if (e != cudaSuccess) {
                exec = nullptr;
                cudaGraphDestroy(g);
                return fail(ctx, RTMB_ECUDA, "cudaGraphInstantiate: %s", cudaGetErrorString(e));
            }
        }
        cudaGraphDestroy(g);
        CK(cudaGraphLaunch(exec, ctx->stream));
        return RTMB_OK;
    }
    ~GraphScope() {
        if (active) {  // an error ended the driver early: end and drop the capture
            cudaGraph_t g = nullptr;
            cudaStreamEndCapture(ctx->stream, &g);
            if (g) cudaGraphDestroy(g);
            (void)cudaGetLastError();
            ctx->capturing = false;
        }
    }
};

int check_shot(rtmb_ctx *ctx, uint32_t sx, uint32_t sy, uint32_t sz) {
    const rtmb_params &p = ctx->p;
    // RTMController.cpp:149-155 rejects sources outside the model
    if (sx >= p.nx || sy >= p.ny || sz >= p.nz)
        return fail(ctx, RTMB_EINVAL, "Invalid Source Position: (%u,%u,%u)", sx, sy, sz);
    if ((int)p.blen < ctx->h)
        return fail(ctx, RTMB_EINVAL, "the per-shot drivers need blen >= stencil_order/2");
    if (!ctx->d_v2dt2) return fail(ctx, RTMB_EINVAL, "no velocity loaded (rtmb_load_v2dt2)");
    if (p.receiver_count_x > p.nx || p.receiver_count_y > p.ny)  // RTMSeismic.cpp:15-19
        return fail(ctx, RTMB_EINVAL, "Invalid Receiver Grid Size");
    return RTMB_OK;
}

// Do all receivers lie off the tapered borders (x, y and z in [blen, n - blen))?  There the
// taper's factors are all 1, so a level stored tapered holds the raw values.
bool receivers_untapered(const rtmb_ctx *c) {
    const rtmb::RcvGeom r = rgeom(c);
    const long long b = c->p.blen;
    if (r.rcx <= 0 || r.rcy <= 0) return true;
    const long long xl = r.rx0 + (long long)(r.rcx - 1) * r.rdx, yl = r.ry0 + (long long)(r.rcy - 1) * r.rdy;
    return r.rx0 >= b && xl < c->nxe - b && r.ry0 >= b && yl < c->nye - b && r.rz >= b && r.rz < c->nze - b;
}

void set_receivers(rtmb::StepArgs &a, const rtmb_ctx *c, int mode, float *rec, int it) {
    const rtmb::RcvGeom r = rgeom(c);
    a.rec_mode = mode;
    a.rec = rec;
    a.rx0 = r.rx0; a.ry0 = r.ry0; a.rz = r.rz; a.rdx = r.rdx > 0 ? r.rdx : 1; a.rdy = r.rdy > 0 ? r.rdy : 1;
    a.rcx = r.rcx; a.rcy = r.rcy;
    const long long ntstep = c->p.ntstep;
    a.rec_si = (long long)r.rcy * ntstep;
    a.rec_sj = ntstep;
    a.rec_base = (long long)(it / ntstep) * r.rcx * r.rcy * ntstep + (it % ntstep);
}

}  // namespace

// Forward time loop shared by modeling and the migration forward pass.  Leaves the last two
// wavefields in (*P, *PP): *P = u(nt-1), *PP = u(nt), raw (untapered) except in a taper-all run
// without a hook on the TMA kernel, which stores every level tapered (T(u), StepArgs::tw).  Every
// buffer it uses must already be set in the context except the taper side buffers, which it
// allocates when missing.
int rtmb::driver::run_forward(rtmb_ctx *ctx, uint32_t sx, uint32_t sy, uint32_t sz, int taper_mode, float *rec,
                float *upb, float **P_out, float **PP_out, int cat, rtmb::ScaleRec **sc_out,
                StepHook *hook) {
    const rtmb_params &p = ctx->p;
    const size_t nb = wave_bytes(ctx);
    const bool st = ctx->store != rtmb::kStoreF32;
    float *P = ctx->d_w[0], *PP = ctx->d_w[1];
    CK(cudaMemsetAsync(P, 0, nb, ctx->stream));
    CK(cudaMemsetAsync(PP, 0, nb, ctx->stream));
    const bool quirk = taper_mode == rtmb::kTaperAll && !(p.flags & RTMB_FLAG_NO_TAPER_QUIRK) && p.blen > 0;
    if (quirk) {
        const size_t qn = (size_t)p.blen * (ctx->nze - 2 * p.blen);
        for (int k = 0; k < 3; ++k) {
            int rc = ensure(ctx, &ctx->d_quirk[k], qn > 0 ? qn : 1, false);
            if (rc) return rc;
            CK(cudaMemsetAsync(ctx->d_quirk[k], 0, (qn > 0 ? qn : 1) * sizeof(float), ctx->stream));
        }
    }
    rtmb::StepArgs a = base_args(ctx);
    a.V = ctx->d_v2dt2;
    a.taper_mode = taper_mode;
    a.quirk = quirk;
    a.sxe = (int)(sx + p.blen); a.sye = (int)(sy + p.blen); a.sze = (int)(sz + p.blen);
    a.store = ctx->store;
    a.inj = ctx->wmax;
    rtmb::ScaleRec *scP = nullptr, *scPP = nullptr;  // records of the levels in P and PP
    if (st && (!(scP = new_scale(ctx)) || !(scPP = new_scale(ctx))))
        return fail(ctx, RTMB_EINVAL, "scale record pool exhausted");
    const size_t upb_step = (size_t)ctx->nxe * ctx->nye * ctx->h;
    // FP32 storage: the record is gathered from the stored level after each step (one small launch;
    // the step kernel's forward forms carry no receiver code).  The 16-bit forms sample the FP32
    // value inside the step, before it is rounded to storage.
    const bool gather = rec && !st;
    const rtmb::RcvGeom rg = rgeom(ctx);
    const rtmb::Geom g = geom(ctx);
    // taper-all runs keep the fields tapered in HBM (StepArgs::tw) when the TMA kernel runs; a hook
    // reads the fields between steps, so it gets the raw form, and so does a gathered record with a
    // receiver in the taper region (where the stored T(u) is not u)
    const bool tw_ok = !hook && tma_ok(ctx) && p.stencil_order <= 8 && ctx->nze % 4 == 0 &&
                       !(p.flags & RTMB_FLAG_NO_TAPER_STORE);
    const bool tw = taper_mode == rtmb::kTaperAll && tw_ok && (!gather || receivers_untapered(ctx));
    a.tw = tw ? rtmb::kTwStored : 0;
    // HBC migration's forward pass (upper taper): the same, except that the last two levels, the
    // snapshots the backward pass starts from, are stored raw (the last step tapers its P on load)
    const bool tw_up = taper_mode == rtmb::kTaperUpper && tw_ok && !st;
    for (uint32_t it = 0; it < p.nt; ++it) {
        std::swap(P, PP);
        std::swap(scP, scPP);
        a.P = P; a.PP = PP; a.it = (int)it;
        rtmb::ScaleRec *lvl = nullptr;
        if (st) {
            if (!(lvl = new_scale(ctx))) return fail(ctx, RTMB_EINVAL, "scale record pool exhausted");
            a.sc_p = scP; a.sc_pp = scPP; a.sc_out = lvl;
        }
        if (rec && !gather) set_receivers(a, ctx, rtmb::kRecSample, rec, (int)it);
        if (upb) { a.upb_mode = rtmb::kUpbSave; a.upb = upb + (size_t)it * upb_step; }
        if (quirk) { a.quirk_in = ctx->d_quirk[(it + 1) % 3]; a.quirk_out = ctx->d_quirk[it % 3]; }
        if (tw_up)
            a.tw = it + 1 < p.nt ? (rtmb::kTwStored | (it + 2 == p.nt ? rtmb::kTwRawOut : 0)) : rtmb::kTwPPOnce;
        int rc;
        if (hook && (rc = hook->before((int)it, P, PP))) return rc;
        LAUNCH_CAT(cat, rtmb::launch_step(a, (int)p.stencil_order, exact(ctx), ctx->stream, tma_ok(ctx)));
        if (gather) {  // RTMCPUPlatform.cpp:133-150: record(i, j, it) = PP(rx0 + i rdx, ry0 + j rdy, rz)
            const size_t chunk = (size_t)rg.rcx * rg.rcy * p.ntstep;
            LAUNCH_CAT(RTMB_PROF_OTHER, rtmb::launch_receivers(PP, rec + (size_t)(it / p.ntstep) * chunk,
                                                               (int)(it % p.ntstep), 1, rg, g, ctx->stream));
        }
        if (hook && (rc = hook->after((int)it, P, PP))) return rc;
        if (st) scPP = lvl;
    }
    *P_out = P;
    *PP_out = PP;
    if (sc_out) { sc_out[0] = scP; sc_out[1] = scPP; }
    return RTMB_OK;
}

namespace {
using rtmb::driver::run_forward;

int alloc_driver(rtmb_ctx *ctx) {
    for (int k = 0; k < 4; ++k) {
        int rc = ensure_bytes(ctx, reinterpret_cast<void **>(&ctx->d_w[k]), wave_bytes(ctx), false);
        if (rc) return rc;
    }
    if (ctx->store != rtmb::kStoreF32) {
        int rc = ensure(ctx, &ctx->d_inj, 2, true);
        if (rc) return rc;
    }
    for (int k = 0; ctx->diff && k < 2; ++k) {
        int rc = ensure_bytes(ctx, &ctx->d_inc[k], wave_bytes(ctx), false);
        if (rc) return rc;
    }
    return RTMB_OK;
}

}  // namespace

namespace {
thread_local std::string g_noctx_error = "null context";
}  // namespace

void rtmb::driver::init_geometry(rtmb_ctx *ctx) {
    const rtmb_params &p = ctx->p;
    ctx->h = (int)p.stencil_order / 2;
    ctx->nxe = (int)(p.nx + 2 * p.blen);
    ctx->nye = (int)(p.ny + 2 * p.blen);
    ctx->nze = (int)(p.nz + 2 * p.blen);
    ctx->n = (size_t)ctx->nxe * ctx->nye * ctx->nze;
    const int nxi = ctx->nxe - 2 * ctx->h, nyi = ctx->nye - 2 * ctx->h;
    const int tiles = ((ctx->nze + rtmb::kTZ - 1) / rtmb::kTZ) * ((nyi + rtmb::kTY - 1) / rtmb::kTY);
    ctx->chunk = pick_chunk(nxi > 0 ? nxi : 1, tiles > 0 ? tiles : 1);
    // the default dual step (variant 5): 32 x 16 tiles, two CTAs per SM like the 64 x 8 split form
    const int tiles_dual = ((ctx->nze + 31) / 32) * ((nyi + 15) / 16);
    ctx->dual_chunk = pick_chunk(nxi > 0 ? nxi : 1, tiles_dual > 0 ? tiles_dual : 1);
    rtmb_stencil_coefs(p.stencil_order, p.dx, p.dy, p.dz, ctx->coefs);
}

int rtmb::driver::check_model_shot(rtmb_ctx *ctx, uint32_t sx, uint32_t sy, uint32_t sz) {
    int rc = check_shot(ctx, sx, sy, sz);
    if (rc) return rc;
    if (ctx->p.receiver_depth_z + ctx->p.blen >= (uint32_t)ctx->nze - ctx->h)
        return fail(ctx, RTMB_EINVAL, "receiver depth outside the computed region");
    return RTMB_OK;
}

int rtmb::driver::fail_noctx(int code, const char *msg) {
    g_noctx_error = msg;
    return code;
}

extern "C" {

int rtmb_abi_version(void) { return RTMB_ABI_VERSION; }

const char *rtmb_last_error(const rtmb_ctx *ctx) { return ctx ? ctx->err.c_str() : g_noctx_error.c_str(); }

uint64_t rtmb_launch_count(const rtmb_ctx *ctx) { return ctx ? ctx->launches : 0; }

int rtmb_create(const rtmb_params *params, rtmb_ctx **out) {
    if (!params || !out) return RTMB_EINVAL;
    *out = nullptr;
    const rtmb_params &p = *params;
    if (!p.nx || !p.ny || !p.nz || p.stencil_order < 2 || p.stencil_order > 16 || (p.stencil_order & 1u))
        return RTMB_EINVAL;
    if (!p.ntstep || p.nt % p.ntstep) return RTMB_EINVAL;  // RTMParam.cpp:241-245 rejects nt < ntstep
    const uint32_t sf = p.flags & (RTMB_FLAG_STORE_F16 | RTMB_FLAG_STORE_BF16);
    if (sf == (RTMB_FLAG_STORE_F16 | RTMB_FLAG_STORE_BF16))
        return rtmb::driver::fail_noctx(RTMB_EINVAL, "rtmb_create: choose one of RTMB_FLAG_STORE_F16 and _BF16");
    if ((p.flags & RTMB_FLAG_IMG_F64) && !sf)
        return rtmb::driver::fail_noctx(RTMB_EINVAL, "rtmb_create: RTMB_FLAG_IMG_F64 needs a 16-bit storage flag");
    if ((p.flags & RTMB_FLAG_STORE_DIFF) && !sf)
        return rtmb::driver::fail_noctx(RTMB_EINVAL, "rtmb_create: RTMB_FLAG_STORE_DIFF needs a 16-bit storage flag");
    if (sf && !rtmb::storage_form_supported((int)p.stencil_order, (int)(p.nz + 2 * p.blen)))
        return rtmb::driver::fail_noctx(RTMB_EINVAL,
                                        "rtmb_create: the 16-bit storage forms need stencil_order 8 and nz + 2*blen "
                                        "a multiple of 8");
    rtmb_ctx *ctx = new rtmb_ctx;
    ctx->p = p;
    ctx->store = sf == RTMB_FLAG_STORE_F16 ? rtmb::kStoreF16 : (sf ? rtmb::kStoreBF16 : rtmb::kStoreF32);
    ctx->img64 = (p.flags & RTMB_FLAG_IMG_F64) != 0;
    ctx->diff = (p.flags & RTMB_FLAG_STORE_DIFF) != 0;
    rtmb::driver::init_geometry(ctx);
    auto bail = [&](int code) {
        rtmb_destroy(ctx);
        return code;
    };
    int dev = p.device;
    if (dev < 0) {
        if (cudaGetDevice(&dev) != cudaSuccess) return bail(RTMB_ECUDA);
    } else if (cudaSetDevice(dev) != cudaSuccess) {
        return bail(RTMB_ECUDA);
    }
    ctx->device = dev;
    if (cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking) != cudaSuccess) return bail(RTMB_ECUDA);
    ctx->stream = ctx->own_stream;
    float *tap = new float[p.blen > 0 ? p.blen : 1];
    float *wav = new float[p.nt];
    rtmb_taper_vector(p.blen, p.taper_factor, tap);
    rtmb_ricker(p.nt, p.dt, p.fpeak, wav);
    for (uint32_t i = 0; i < p.nt; ++i) ctx->wmax = std::fmax(ctx->wmax, std::fabs(wav[i]));
    bool ok = cudaMalloc(&ctx->d_taper, sizeof(float) * (p.blen > 0 ? p.blen : 1)) == cudaSuccess &&
              cudaMalloc(&ctx->d_wavelet, sizeof(float) * p.nt) == cudaSuccess &&
              cudaMalloc(&ctx->d_err, sizeof(unsigned)) == cudaSuccess &&
              cudaMemcpy(ctx->d_taper, tap, sizeof(float) * (p.blen > 0 ? p.blen : 1), cudaMemcpyHostToDevice) == cudaSuccess &&
              cudaMemcpy(ctx->d_wavelet, wav, sizeof(float) * p.nt, cudaMemcpyHostToDevice) == cudaSuccess &&
              cudaMemset(ctx->d_err, 0, sizeof(unsigned)) == cudaSuccess;
    delete[] tap;
    delete[] wav;
    if (!ok) return bail(RTMB_ENOMEM);
    *out = ctx;
    return RTMB_OK;
}

int rtmb_destroy(rtmb_ctx *ctx) {
    if (!ctx) return RTMB_OK;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    for (cudaEvent_t e : ctx->ev) cudaEventDestroy(e);
    float *bufs[] = {ctx->d_taper, ctx->d_wavelet, ctx->d_v2dt2, ctx->d_w[0], ctx->d_w[1], ctx->d_w[2],
                     ctx->d_w[3], ctx->d_quirk[0], ctx->d_quirk[1], ctx->d_quirk[2], ctx->d_upb,
                     ctx->d_rec, ctx->d_img};
    for (float *b : bufs)
        if (b) cudaFree(b);
    if (ctx->d_err) cudaFree(ctx->d_err);
    if (ctx->d_scale) cudaFree(ctx->d_scale);
    if (ctx->d_inj) cudaFree(ctx->d_inj);
    if (ctx->d_img64) cudaFree(ctx->d_img64);
    for (void *b : ctx->d_inc)
        if (b) cudaFree(b);
    for (double *b : ctx->d_f64)
        if (b) cudaFree(b);
    if (ctx->d_upb64) cudaFree(ctx->d_upb64);
    if (ctx->d_fq) cudaFree(ctx->d_fq);
    for (float *b : ctx->d_fquirk)
        if (b) cudaFree(b);
    for (cudaGraphExec_t g : ctx->gexec)
        if (g) cudaGraphExecDestroy(g);
    if (ctx->d_cells) cudaFree(ctx->d_cells);
    if (ctx->d_faces) cudaFree(ctx->d_faces);
    if (ctx->d_side) cudaFree(ctx->d_side);
    if (ctx->d_cparams) cudaFree(ctx->d_cparams);
    if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
    delete ctx;
    return RTMB_OK;
}

int rtmb_set_stream(rtmb_ctx *ctx, void *cuda_stream) {
    if (!ctx) return RTMB_EINVAL;
    ctx->stream = cuda_stream ? static_cast<cudaStream_t>(cuda_stream) : ctx->own_stream;
    return RTMB_OK;
}

int rtmb_profile(rtmb_ctx *ctx, int enable) {
    if (!ctx) return RTMB_EINVAL;
    ctx->prof = enable != 0;
    ctx->ev_used = 0;
    for (int k = 0; k < RTMB_PROF_CATEGORIES; ++k) { ctx->prof_ms[k] = 0.0; ctx->prof_n[k] = 0; }
    return RTMB_OK;
}

int rtmb_profile_read(const rtmb_ctx *ctx, double *ms, uint64_t *launches) {
    if (!ctx || !ms || !launches) return RTMB_EINVAL;
    for (int k = 0; k < RTMB_PROF_CATEGORIES; ++k) { ms[k] = ctx->prof_ms[k]; launches[k] = ctx->prof_n[k]; }
    return RTMB_OK;
}

int rtmb_sync(rtmb_ctx *ctx) {
    if (!ctx) return RTMB_EINVAL;
    CK(cudaStreamSynchronize(ctx->stream));
    return check_err_flag(ctx);
}

// ------------------------------------------------------------------ per-step operators

int rtmb_step(rtmb_ctx *ctx, const float *P, float *PP, const float *v2dt2) {
    if (!ctx || !P || !PP || !v2dt2) return fail(ctx, RTMB_EINVAL, "rtmb_step: null pointer");
    rtmb::StepArgs a = base_args(ctx);
    a.P = P; a.PP = PP; a.V = v2dt2;
    LAUNCH(rtmb::launch_step(a, (int)ctx->p.stencil_order, exact(ctx), ctx->stream, tma_ok(ctx)));
    return RTMB_OK;
}

int rtmb_step_multiwave(rtmb_ctx *ctx, const float *P0, float *PP0, const float *P1, float *PP1, const float *v2dt2) {
    // RTMCPUPlatform.cpp:397-472: both wavefields, the same v2dt2, each the single-wave step's arithmetic
    int rc = rtmb_step(ctx, P0, PP0, v2dt2);
    return rc ? rc : rtmb_step(ctx, P1, PP1, v2dt2);
}

int rtmb_fmig_update_freq(rtmb_ctx *ctx, uint32_t it, uint32_t iw, uint32_t lw, const float *PS, const float *PR,
                          float *sre, float *sim, float *rre, float *rim, const float *kre, const float *kim) {
    if (!ctx || !PS || !PR || !sre || !sim || !rre || !rim || !kre || !kim)
        return fail(ctx, RTMB_EINVAL, "rtmb_fmig_update_freq: null pointer");
    if (it >= ctx->p.nt) return fail(ctx, RTMB_EINVAL, "rtmb_fmig_update_freq: time step out of range");
    LAUNCH(rtmb::launch_fmig_update(PS, PR, sre, sim, rre, rim, kre, kim, (int)it, (int)iw, (int)lw, (int)ctx->p.nt,
                                    geom(ctx), (int)ctx->p.nx, (int)ctx->p.ny, (int)ctx->p.nz, ctx->stream));
    return RTMB_OK;
}

int rtmb_fmig_image_condition(rtmb_ctx *ctx, uint32_t iw, uint32_t lw, const float *w2, float *img, const float *sre,
                              const float *sim, const float *rre, const float *rim) {
    if (!ctx || !w2 || !img || !sre || !sim || !rre || !rim)
        return fail(ctx, RTMB_EINVAL, "rtmb_fmig_image_condition: null pointer");
    LAUNCH(rtmb::launch_fmig_image(img, sre, sim, rre, rim, w2, (int)iw, (int)lw, geom(ctx), (int)ctx->p.nx,
                                   (int)ctx->p.ny, (int)ctx->p.nz, ctx->stream));
    return RTMB_OK;
}

int rtmb_taper_all_borders(rtmb_ctx *ctx, float *P) {
    if (!ctx || !P) return fail(ctx, RTMB_EINVAL, "rtmb_taper_all_borders: null pointer");
    LAUNCH(rtmb::launch_taper(P, ctx->d_taper, geom(ctx), 0, !(ctx->p.flags & RTMB_FLAG_NO_TAPER_QUIRK), ctx->stream));
    return RTMB_OK;
}

int rtmb_taper_upper_borders(rtmb_ctx *ctx, float *P) {
    if (!ctx || !P) return fail(ctx, RTMB_EINVAL, "rtmb_taper_upper_borders: null pointer");
    LAUNCH(rtmb::launch_taper(P, ctx->d_taper, geom(ctx), 1, 0, ctx->stream));
    return RTMB_OK;
}

int rtmb_apply_source(rtmb_ctx *ctx, float *PP, uint32_t sx, uint32_t sy, uint32_t sz, uint32_t it) {
    if (!ctx || !PP) return fail(ctx, RTMB_EINVAL, "rtmb_apply_source: null pointer");
    const uint32_t b = ctx->p.blen;
    if (sx + b >= (uint32_t)ctx->nxe || sy + b >= (uint32_t)ctx->nye || sz + b >= (uint32_t)ctx->nze || it >= ctx->p.nt)
        return fail(ctx, RTMB_EINVAL, "rtmb_apply_source: position or time step out of range");
    LAUNCH(rtmb::launch_source(PP, ctx->d_wavelet, (int)it, (int)(sx + b), (int)(sy + b), (int)(sz + b), geom(ctx),
                               ctx->stream));
    return RTMB_OK;
}

int rtmb_save_receiver_data(rtmb_ctx *ctx, const float *PP, float *rec, uint32_t lt) {
    if (!ctx || !PP || !rec || lt >= ctx->p.ntstep) return fail(ctx, RTMB_EINVAL, "rtmb_save_receiver_data: bad argument");
    if (ctx->p.receiver_depth_z + ctx->p.blen >= (uint32_t)ctx->nze) return fail(ctx, RTMB_EINVAL, "receiver depth out of range");
    LAUNCH(rtmb::launch_receivers(const_cast<float *>(PP), rec, (int)lt, 1, rgeom(ctx), geom(ctx), ctx->stream));
    return RTMB_OK;
}

int rtmb_restore_receiver_data(rtmb_ctx *ctx, float *PP, const float *rec, uint32_t lt) {
    if (!ctx || !PP || !rec || lt >= ctx->p.ntstep) return fail(ctx, RTMB_EINVAL, "rtmb_restore_receiver_data: bad argument");
    if (ctx->p.receiver_depth_z + ctx->p.blen >= (uint32_t)ctx->nze) return fail(ctx, RTMB_EINVAL, "receiver depth out of range");
    const int mode = (ctx->p.flags & RTMB_FLAG_RCV_ADD) ? 3 : 2;
    LAUNCH(rtmb::launch_receivers(PP, const_cast<float *>(rec), (int)lt, mode, rgeom(ctx), geom(ctx), ctx->stream));
    return RTMB_OK;
}

int rtmb_save_upper_border(rtmb_ctx *ctx, const float *P, float *upb, uint32_t lt) {
    if (!ctx || !P || !upb || lt >= ctx->p.ntstep) return fail(ctx, RTMB_EINVAL, "rtmb_save_upper_border: bad argument");
    if ((int)ctx->p.blen < ctx->h) return fail(ctx, RTMB_EINVAL, "upper border needs blen >= stencil_order/2");
    LAUNCH(rtmb::launch_upb(const_cast<float *>(P), upb, (int)lt, 1, geom(ctx), ctx->stream));
    return RTMB_OK;
}

int rtmb_restore_upper_border(rtmb_ctx *ctx, float *P, const float *upb, uint32_t lt) {
    if (!ctx || !P || !upb || lt >= ctx->p.ntstep) return fail(ctx, RTMB_EINVAL, "rtmb_restore_upper_border: bad argument");
    if ((int)ctx->p.blen < ctx->h) return fail(ctx, RTMB_EINVAL, "upper border needs blen >= stencil_order/2");
    LAUNCH(rtmb::launch_upb(P, const_cast<float *>(upb), (int)lt, 0, geom(ctx), ctx->stream));
    return RTMB_OK;
}

int rtmb_image_condition(rtmb_ctx *ctx, float *img, const float *ps, const float *pr) {
    if (!ctx || !img || !ps || !pr) return fail(ctx, RTMB_EINVAL, "rtmb_image_condition: null pointer");
    const bool full = ctx->p.flags & RTMB_FLAG_IMG_FULL_Z;
    const int z0 = full ? 0 : (int)ctx->p.blen, z1 = full ? ctx->nze : ctx->nze - (int)ctx->p.blen;
    LAUNCH(rtmb::launch_image(img, ps, pr, z0, z1, geom(ctx), ctx->stream));
    return RTMB_OK;
}

int rtmb_image_finalize(rtmb_ctx *ctx, const float *img, float *out) {
    if (!ctx || !img || !out) return fail(ctx, RTMB_EINVAL, "rtmb_image_finalize: null pointer");
    if (ctx->p.blen < 1) return fail(ctx, RTMB_EINVAL, "rtmb_image_finalize needs blen >= 1");
    float c3[9];
    rtmb_stencil_coefs(2, ctx->p.dx, ctx->p.dy, ctx->p.dz, c3);
    LAUNCH(rtmb::launch_filter_remove(img, out, c3, geom(ctx), ctx->stream));
    return RTMB_OK;
}

int rtmb_image_stack(rtmb_ctx *ctx, float *acc, const float *img) {
    if (!ctx || !acc || !img) return fail(ctx, RTMB_EINVAL, "rtmb_image_stack: null pointer");
    LAUNCH(rtmb::launch_stack(acc, img, ctx->n, ctx->stream));
    return RTMB_OK;
}

// ------------------------------------------------------------------ drivers

int rtmb_load_v2dt2(rtmb_ctx *ctx, const float *v2dt2, int from_host) {
    if (!ctx || !v2dt2) return fail(ctx, RTMB_EINVAL, "rtmb_load_v2dt2: null pointer");
    int rc = ensure(ctx, &ctx->d_v2dt2, ctx->n, false);
    if (rc) return rc;
    CK(cudaMemcpyAsync(ctx->d_v2dt2, v2dt2, ctx->n * sizeof(float),
                       from_host ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return RTMB_OK;
}

int rtmb_model_shot(rtmb_ctx *ctx, uint32_t sx, uint32_t sy, uint32_t sz, float *rec) {
    if (!ctx || !rec) return fail(ctx, RTMB_EINVAL, "rtmb_model_shot: null pointer");
    int rc = rtmb::driver::check_model_shot(ctx, sx, sy, sz);
    if (rc) return rc;
    if ((rc = alloc_driver(ctx))) return rc;
    if (ctx->store != rtmb::kStoreF32 && (rc = reset_scales(ctx))) return rc;
    float *P, *PP;
    const bool learned = ctx->p.boundary == RTMB_BC_LEARNED;
    if (learned && !ctx->d_cparams) return fail(ctx, RTMB_EINVAL, "boundary RTMB_BC_LEARNED needs rtmb_closure_set");
    if (learned && ctx->store != rtmb::kStoreF32)
        return fail(ctx, RTMB_EINVAL, "the learned closure runs with FP32 storage");
    if (ctx->diff) return fail(ctx, RTMB_EINVAL, "the increment storage form (RTMB_FLAG_STORE_DIFF) runs RBC migration only");
    // the learned closure: the strip's next level before each step, scattered after it
    struct Closure : rtmb::driver::StepHook {
        rtmb_ctx *c;
        int before(int, const float *P, float *PP) override {
            ++c->launches;
            return rtmb::driver::closure_hook_before(c, P, PP);
        }
        int after(int, const float *, float *PP) override {
            ++c->launches;
            return rtmb::driver::closure_hook_after(c, PP);
        }
    } closure;
    closure.c = ctx;
    GraphScope graph(ctx, 0);
    if ((rc = graph.begin())) return rc;
    // RTMFiniteDifferencesKernel.cpp:169-216: taper all faces, step, inject, sample.
    if ((rc = run_forward(ctx, sx, sy, sz, learned ? rtmb::kTaperNone : rtmb::kTaperAll, rec, nullptr, &P, &PP,
                          RTMB_PROF_MODEL, nullptr, learned ? &closure : nullptr)))
        return rc;
    if ((rc = graph.end())) return rc;
    return check_err_flag(ctx);
}

}  // extern "C"

namespace {

// RBC migration in the increment storage form (RTMB_FLAG_STORE_DIFF): each wavefield is a 16-bit
// level p and a 16-bit increment d = p - p_prev, each with its own exponent; the steps write
// d' = d + v2dt2 lap p in place and p' = p + d' into the other level buffer.  The same time loop
// as the two-level drivers (RBC.cpp:54-274): forward from zero, the backward pass rebuilds the
// source wavefield from the forward pass's last two levels and images it against the receiver
// wavefield.  img: the FP32 image (overwritten), the FP64 image of RTMB_FLAG_IMG_F64, or with acc64
// the caller's FP64 stack (added to).
int migrate_diff(rtmb_ctx *ctx, uint32_t sx, uint32_t sy, uint32_t sz, const float *rec, void *img_out, bool acc64) {
    const rtmb_params &p = ctx->p;
    if (p.boundary != RTMB_BC_RBC)
        return fail(ctx, RTMB_EINVAL, "the increment storage form (RTMB_FLAG_STORE_DIFF) migrates with boundary RBC");
    int rc;
    if ((rc = alloc_driver(ctx))) return rc;
    if ((rc = reset_scales(ctx))) return rc;
    if (ctx->img64 && !acc64 &&
        (rc = ensure_bytes(ctx, reinterpret_cast<void **>(&ctx->d_img64), ctx->n * sizeof(double), false)))
        return rc;
    const size_t nb = wave_bytes(ctx);
    for (int k = 0; k < 4; ++k) CK(cudaMemsetAsync(ctx->d_w[k], 0, nb, ctx->stream));
    for (int k = 0; k < 2; ++k) CK(cudaMemsetAsync(ctx->d_inc[k], 0, nb, ctx->stream));
    GraphScope graph(ctx, 1);
    if ((rc = graph.begin())) return rc;

    // one wavefield: level buffers cur / next, increment d, and their scale records
    struct Wave {
        float *cur, *next;
        void *d;
        rtmb::ScaleRec *sc_cur, *sc_d;
    };
    auto fresh = [&](Wave &w, float *a, float *b, void *d) -> int {
        w.cur = a; w.next = b; w.d = d;
        if (!(w.sc_cur = new_scale(ctx)) || !(w.sc_d = new_scale(ctx)))
            return fail(ctx, RTMB_EINVAL, "scale record pool exhausted");
        return RTMB_OK;
    };
    // one step of w: (cur, d) -> (next, d in place), the records of the new level and increment
    auto step = [&](Wave &w, rtmb::StepArgs &a, int cat) -> int {
        rtmb::ScaleRec *lp = new_scale(ctx), *ld = new_scale(ctx);
        if (!lp || !ld) return fail(ctx, RTMB_EINVAL, "scale record pool exhausted");
        a.P = w.cur; a.PP = static_cast<float *>(w.d); a.Pout = w.next;
        a.sc_p = w.sc_cur; a.sc_pp = w.sc_d; a.sc_out = lp; a.sc_out2 = ld;
        LAUNCH_CAT(cat, rtmb::launch_step(a, (int)p.stencil_order, false, ctx->stream, true));
        std::swap(w.cur, w.next);
        w.sc_cur = lp;
        w.sc_d = ld;
        return RTMB_OK;
    };
    Wave S, R;
    if ((rc = fresh(S, ctx->d_w[0], ctx->d_w[1], ctx->d_inc[0])) || (rc = fresh(R, ctx->d_w[2], ctx->d_w[3], ctx->d_inc[1])))
        return rc;

    // forward pass (RBC.cpp:54-144): source injection, no taper, no record
    rtmb::StepArgs a = base_args(ctx);
    a.V = ctx->d_v2dt2;
    a.store = ctx->store;
    a.diff = 1;
    a.inj = ctx->wmax;
    a.sxe = (int)(sx + p.blen); a.sye = (int)(sy + p.blen); a.sze = (int)(sz + p.blen);
    for (uint32_t it = 0; it < p.nt; ++it) {
        a.it = (int)it;
        if ((rc = step(S, a, RTMB_PROF_FORWARD))) return rc;
    }

    void *img = img_out;
    bool img64 = acc64;
    if (!acc64 && ctx->img64) {
        img = ctx->d_img64;
        img64 = true;
    }
    if (!acc64) CK(cudaMemsetAsync(img, 0, ctx->n * (img64 ? sizeof(double) : sizeof(float)), ctx->stream));
    const size_t nrec = (size_t)p.nt * p.receiver_count_x * p.receiver_count_y;
    LAUNCH_CAT(RTMB_PROF_OTHER, rtmb::launch_absmax(rec, nrec, ctx->d_inj, ctx->stream));

    // backward pass (RBC.cpp:146-274): it = nt-1 images p(nt); it = nt-2 images p(nt-1), rebuilt
    // from the last level and increment; below, each source step rebuilds p(it+1)
    rtmb::StepArgs src = base_args(ctx);
    src.V = ctx->d_v2dt2;
    src.store = ctx->store;
    src.diff = 1;
    rtmb::StepArgs rcv = base_args(ctx);
    rcv.V = ctx->d_v2dt2;
    rcv.store = ctx->store;
    rcv.diff = 1;
    const bool full = p.flags & RTMB_FLAG_IMG_FULL_Z;
    rcv.img = static_cast<float *>(img);
    rcv.img64 = img64;
    rcv.img_z0 = full ? 0 : (int)p.blen;
    rcv.img_z1 = full ? ctx->nze : ctx->nze - (int)p.blen;
    rcv.inj_dev = ctx->d_inj;
    const int rmode = (p.flags & RTMB_FLAG_RCV_ADD) ? rtmb::kRecAdd : rtmb::kRecOverwrite;
    for (int it = (int)p.nt - 1; it >= 0; --it) {
        if (it == (int)p.nt - 2) {
            rtmb::ScaleRec *lp = new_scale(ctx);
            if (!lp) return fail(ctx, RTMB_EINVAL, "scale record pool exhausted");
            LAUNCH_CAT(RTMB_PROF_OTHER, rtmb::launch_diff_rewind(ctx->store, S.cur, S.d, S.next, S.sc_cur, S.sc_d, lp,
                                                                 ctx->n, ctx->stream));
            std::swap(S.cur, S.next);
            S.sc_cur = lp;
        } else if (it < (int)p.nt - 2) {
            src.it = it;
            if ((rc = step(S, src, RTMB_PROF_BACKWARD_SOURCE))) return rc;
        }
        rcv.it = it;
        rcv.ps = S.cur;
        rcv.sc_ps = S.sc_cur;
        set_receivers(rcv, ctx, rmode, const_cast<float *>(rec), it);
        if ((rc = step(R, rcv, RTMB_PROF_BACKWARD_RECEIVER))) return rc;
    }
    if (img != img_out)
        LAUNCH_CAT(RTMB_PROF_OTHER, rtmb::launch_to_float(ctx->d_img64, static_cast<float *>(img_out), ctx->n,
                                                          ctx->stream));
    if ((rc = graph.end())) return rc;
    return check_err_flag(ctx);
}

// The migration of one shot.  img_out: the caller's FP32 image (overwritten) or, with acc64, the
// caller's FP64 stack (added to).
int migrate_impl(rtmb_ctx *ctx, uint32_t sx, uint32_t sy, uint32_t sz, const float *rec, void *img_out,
                 bool acc64) {
    int rc = check_shot(ctx, sx, sy, sz);
    if (rc) return rc;
    const rtmb_params &p = ctx->p;
    if (p.boundary != RTMB_BC_HBC && p.boundary != RTMB_BC_RBC)
        return fail(ctx, RTMB_EINVAL, "migration boundary must be HBC or RBC");
    if (p.receiver_depth_z + p.blen >= (uint32_t)ctx->nze - ctx->h)
        return fail(ctx, RTMB_EINVAL, "receiver depth outside the computed region");
    const bool st = ctx->store != rtmb::kStoreF32;
    if (ctx->diff) return migrate_diff(ctx, sx, sy, sz, rec, img_out, acc64);
    if (!st && acc64) {
        // FP32 storage: the FP32 shot image, then added to the FP64 stack
        if ((rc = ensure(ctx, &ctx->d_img, ctx->n, false))) return rc;
        if ((rc = migrate_impl(ctx, sx, sy, sz, rec, ctx->d_img, false))) return rc;
        LAUNCH_CAT(RTMB_PROF_OTHER, rtmb::launch_stack64(static_cast<double *>(img_out), ctx->d_img, ctx->n, ctx->stream));
        return check_err_flag(ctx);
    }
    const bool hbc = p.boundary == RTMB_BC_HBC;
    if (st && hbc) return fail(ctx, RTMB_EINVAL, "the 16-bit storage forms migrate with boundary RBC");
    if ((rc = alloc_driver(ctx))) return rc;
    if (st && (rc = reset_scales(ctx))) return rc;
    const size_t upb_step = (size_t)ctx->nxe * ctx->nye * ctx->h;
    if (hbc && (rc = ensure(ctx, &ctx->d_upb, upb_step * p.nt, true))) return rc;
    if (st && ctx->img64 && !acc64 &&
        (rc = ensure_bytes(ctx, reinterpret_cast<void **>(&ctx->d_img64), ctx->n * sizeof(double), false)))
        return rc;
    GraphScope graph(ctx, 1);
    if ((rc = graph.begin())) return rc;

    // forward pass (HBC.cpp:96-210 / RBC.cpp:54-144)
    float *sP, *sPP;
    rtmb::ScaleRec *scs[2] = {nullptr, nullptr};
    if ((rc = run_forward(ctx, sx, sy, sz, hbc ? rtmb::kTaperUpper : rtmb::kTaperNone, nullptr,
                          hbc ? ctx->d_upb : nullptr, &sP, &sPP, RTMB_PROF_FORWARD, scs)))
        return rc;
    // snap0 is P after its last in-place taper (HBC.cpp:150, 203)
    if (hbc) LAUNCH_CAT(RTMB_PROF_OTHER, rtmb::launch_taper(sP, ctx->d_taper, geom(ctx), 1, 0, ctx->stream));

    // image target: the caller's FP32 image, the caller's FP64 stack, or the FP64 image that is
    // rounded into the caller's FP32 image at the end
    void *img = img_out;
    bool img64 = false;
    if (st && acc64) {
        img64 = true;
    } else if (st && ctx->img64) {
        img = ctx->d_img64;
        img64 = true;
    }
    if (!acc64) CK(cudaMemsetAsync(img, 0, ctx->n * (img64 ? sizeof(double) : sizeof(float)), ctx->stream));

    // backward pass (HBC.cpp:212-364 / RBC.cpp:146-274)
    float *rP = ctx->d_w[2], *rPP = ctx->d_w[3];
    CK(cudaMemsetAsync(rP, 0, wave_bytes(ctx), ctx->stream));
    CK(cudaMemsetAsync(rPP, 0, wave_bytes(ctx), ctx->stream));
    rtmb::ScaleRec *sc_rP = nullptr, *sc_rPP = nullptr;
    if (st) {
        if (!(sc_rP = new_scale(ctx)) || !(sc_rPP = new_scale(ctx)))
            return fail(ctx, RTMB_EINVAL, "scale record pool exhausted");
        // the receiver levels' exponent bound includes max |record| (the injected values)
        const size_t nrec = (size_t)p.nt * p.receiver_count_x * p.receiver_count_y;
        LAUNCH_CAT(RTMB_PROF_OTHER, rtmb::launch_absmax(rec, nrec, ctx->d_inj, ctx->stream));
    }
    const bool full = p.flags & RTMB_FLAG_IMG_FULL_Z;
    float *s_cur = sPP, *s_prev = sP;  // it = nt-1 images snap1
    rtmb::ScaleRec *sc_cur = scs[1], *sc_prev = scs[0];
    rtmb::StepArgs src = base_args(ctx);
    src.V = ctx->d_v2dt2;
    src.store = ctx->store;
    if (hbc) src.upb_mode = rtmb::kUpbRestore;
    rtmb::StepArgs rcv = base_args(ctx);
    rcv.V = ctx->d_v2dt2;
    rcv.taper_mode = hbc ? rtmb::kTaperUpper : rtmb::kTaperNone;
    // HBC: the receiver wavefield stays tapered in HBM (the image takes the raw new level in the
    // step; nothing reads the receiver fields afterwards)
    if (hbc && !st && tma_ok(ctx) && p.stencil_order <= 8 && ctx->nze % 4 == 0 &&
        !(p.flags & RTMB_FLAG_NO_TAPER_STORE) && reinterpret_cast<uintptr_t>(img) % 16 == 0)
        rcv.tw = rtmb::kTwStored;
    rcv.img = static_cast<float *>(img);
    rcv.img64 = img64;
    rcv.img_z0 = full ? 0 : (int)p.blen;
    rcv.img_z1 = full ? ctx->nze : ctx->nze - (int)p.blen;
    rcv.store = ctx->store;
    rcv.inj_dev = st ? ctx->d_inj : nullptr;
    const int rmode = (p.flags & RTMB_FLAG_RCV_ADD) ? rtmb::kRecAdd : rtmb::kRecOverwrite;
    // FP32 forms: the source and receiver steps of one time step in one launch unless the autotuner
    // measured two launches faster (RBC: with the upper taper of HBC the two launches measured
    // faster, 1.83 against 2.99 ms at 592^3)
    const bool dual = !st && p.stencil_order == 8 && tma_ok(ctx) && !(p.flags & RTMB_FLAG_NO_DUAL) && p.nx > 1 &&
                      !hbc && ctx->use_dual != 0;
    // the merged dual step pairs its launches on the image: the first of a pair leaves its product
    // S_new R_new to the second, which adds both in the order two separate steps would (the image
    // is read and written every other step).  Only where every dual step of the loop is a merged
    // launch; an odd last step reads and writes the image itself.
    bool dual_geometry_ok = false;  // the dual step's conditions hold for every step of the loop
    if (dual && p.nt > 2) {
        rtmb::StepArgs s0 = src, r0 = rcv;
        s0.P = s_cur; s0.PP = s_prev;
        r0.P = rP; r0.PP = rPP; r0.ps = nullptr;
        set_receivers(r0, ctx, rmode, const_cast<float *>(rec), 0);
        r0.chunk = ctx->dual_chunk;
        r0.variant = ctx->dual_variant;
        dual_geometry_ok = rtmb::dual_step_supported(s0, r0, (int)p.stencil_order);
    }
    const bool pair_img = dual && ctx->dual_variant >= 4 && dual_geometry_ok;
    for (int it = (int)p.nt - 1; it >= 0; --it) {
        if (dual && it < (int)p.nt - 2) {
            src.P = s_cur; src.PP = s_prev; src.it = it;
            if (hbc) src.upb = ctx->d_upb + (size_t)it * upb_step;
            rcv.P = rP; rcv.PP = rPP; rcv.it = it;
            rcv.ps = nullptr;
            set_receivers(rcv, ctx, rmode, const_cast<float *>(rec), it);
            rcv.chunk = ctx->dual_chunk;
            rcv.variant = ctx->dual_variant;
            const int j = (int)p.nt - 3 - it;  // index of this dual step, from 0
            rcv.img_pair = !pair_img ? 0 : (j % 2 == 1 ? 2 : (it > 0 ? 1 : 0));
            if (rtmb::dual_step_supported(src, rcv, (int)p.stencil_order)) {
                LAUNCH_CAT(RTMB_PROF_BACKWARD_DUAL,
                           rtmb::launch_dual_step(src, rcv, (int)p.stencil_order, exact(ctx), ctx->stream));
                rcv.chunk = ctx->chunk;
                rcv.variant = ctx->variant;
                rcv.img_pair = 0;
                std::swap(s_cur, s_prev);
                std::swap(rP, rPP);
                continue;
            }
            if (pair_img) return fail(ctx, RTMB_EINVAL, "dual step no longer supported in a paired loop");
            rcv.chunk = ctx->chunk;
            rcv.variant = ctx->variant;
            rcv.img_pair = 0;
        }
        if (it == (int)p.nt - 2) {
            s_cur = sP;
            s_prev = sPP;
            std::swap(sc_cur, sc_prev);
        } else if (it < (int)p.nt - 2) {
            src.P = s_cur; src.PP = s_prev; src.it = it;
            if (hbc) src.upb = ctx->d_upb + (size_t)it * upb_step;
            rtmb::ScaleRec *lvl = nullptr;
            if (st) {
                if (!(lvl = new_scale(ctx))) return fail(ctx, RTMB_EINVAL, "scale record pool exhausted");
                src.sc_p = sc_cur; src.sc_pp = sc_prev; src.sc_out = lvl;
            }
            LAUNCH_CAT(RTMB_PROF_BACKWARD_SOURCE,
                       rtmb::launch_step(src, (int)p.stencil_order, exact(ctx), ctx->stream, tma_ok(ctx)));
            std::swap(s_cur, s_prev);
            sc_prev = sc_cur;
            sc_cur = lvl;
        }
        rcv.P = rP; rcv.PP = rPP; rcv.it = it;
        rcv.ps = s_cur;
        rtmb::ScaleRec *lvl = nullptr;
        if (st) {
            if (!(lvl = new_scale(ctx))) return fail(ctx, RTMB_EINVAL, "scale record pool exhausted");
            rcv.sc_p = sc_rP; rcv.sc_pp = sc_rPP; rcv.sc_out = lvl; rcv.sc_ps = sc_cur;
        }
        set_receivers(rcv, ctx, rmode, const_cast<float *>(rec), it);
        LAUNCH_CAT(RTMB_PROF_BACKWARD_RECEIVER,
                   rtmb::launch_step(rcv, (int)p.stencil_order, exact(ctx), ctx->stream, tma_ok(ctx)));
        std::swap(rP, rPP);
        sc_rPP = sc_rP;
        sc_rP = lvl;
    }
    if (img != img_out)
        LAUNCH_CAT(RTMB_PROF_OTHER, rtmb::launch_to_float(ctx->d_img64, static_cast<float *>(img_out), ctx->n,
                                                          ctx->stream));
    if ((rc = graph.end())) return rc;
    return check_err_flag(ctx);
}

}  // namespace

extern "C" {

int rtmb_migrate_shot(rtmb_ctx *ctx, uint32_t sx, uint32_t sy, uint32_t sz, const float *rec, float *img) {
    if (!ctx || !rec || !img) return fail(ctx, RTMB_EINVAL, "rtmb_migrate_shot: null pointer");
    return migrate_impl(ctx, sx, sy, sz, rec, img, false);
}

// ------------------------------------------------------------------ frequency-domain migration

int rtmb_fmig_nw(float dt, uint32_t nt, float fmin, float fmax) {
    // RTMFiniteDifferencesKernel_FreqDomain.cpp:133-137, in the reference's float / double mix
    const float df = (float)(1. / ((nt * 1.0) * dt));
    const float nf = ((fmax - fmin) / df);
    return nf > 0.f ? (int)(size_t)nf : 0;
}

namespace {
void fmig_tables(const rtmb_params &p, float fmin, int nw, std::vector<float> &w2, std::vector<float> &kre,
                 std::vector<float> &kim);
}  // namespace

int rtmb_fmig_tables(float dt, uint32_t nt, float fmin, float fmax, float *w2, float *kre, float *kim) {
    if (!w2 || !kre || !kim) return RTMB_EINVAL;
    rtmb_params p{};
    p.dt = dt;
    p.nt = nt;
    const int nw = rtmb_fmig_nw(dt, nt, fmin, fmax);
    std::vector<float> a, b, c;
    fmig_tables(p, fmin, nw, a, b, c);
    std::memcpy(w2, a.data(), a.size() * sizeof(float));
    std::memcpy(kre, b.data(), b.size() * sizeof(float));
    std::memcpy(kim, c.data(), c.size() * sizeof(float));
    return RTMB_OK;
}

namespace {

// The angular frequency per time step of frequency iw, w = 2 pi (iw df + fmin) dt, and the DFT
// kernels cos(w it), sin(w it) (..._FreqDomain.cpp:17-51, the same float / double mix, so the
// tables are the reference's bit for bit), with w2 = w^2 (wList->power2(), :151-152).
void fmig_tables(const rtmb_params &p, float fmin, int nw, std::vector<float> &w2, std::vector<float> &kre,
                 std::vector<float> &kim) {
    const float df = (float)(1. / ((p.nt * 1.0) * p.dt));
    const float pi = acosf(-1.);
    w2.assign(nw, 0.f);
    kre.assign((size_t)nw * p.nt, 0.f);
    kim.assign((size_t)nw * p.nt, 0.f);
    for (int iw = 0; iw < nw; ++iw) {
        const float lw = (float)iw * 1.0;
        const float w = (float)(2. * pi * ((lw * df) + fmin) * p.dt);
        for (uint32_t it = 0; it < p.nt; ++it) {
            kre[(size_t)iw * p.nt + it] = cosf((float)(w * (it * 1.0)));
            kim[(size_t)iw * p.nt + it] = sinf((float)(w * (it * 1.0)));
        }
        w2[iw] = w * w;
    }
}

}  // namespace

// RTMFiniteDifferencesKernel_FreqDomain.cpp:220-357 (rtmFreqDomainPropagation).  Both wavefields
// step forward in time st = nt-1-rt: the source one from the Ricker wavelet, the receiver one
// from the record read backwards.  Per step, as the reference orders it: the two steps (:358-369,
// rtmStepMultipleWave), the taper of the four fields, the source, the receivers, then the DFT and
// image update of every frequency of the group.  Each group of nwstep frequencies re-runs the
// time loop from zero fields; the image sums over the groups.
int rtmb_migrate_shot_fmig(rtmb_ctx *ctx, uint32_t sx, uint32_t sy, uint32_t sz, const float *rec, float fmin,
                           float fmax, uint32_t nwstep, float *img) {
    if (!ctx || !rec || !img) return fail(ctx, RTMB_EINVAL, "rtmb_migrate_shot_fmig: null pointer");
    int rc = check_shot(ctx, sx, sy, sz);
    if (rc) return rc;
    const rtmb_params &p = ctx->p;
    if (ctx->store != rtmb::kStoreF32) return fail(ctx, RTMB_EINVAL, "frequency-domain migration runs with FP32 storage");
    if (!(fmax > fmin)) return fail(ctx, RTMB_EINVAL, "fmig_max_freq must be above fmig_min_freq");  // RTMParam.cpp:246-251
    if (p.receiver_depth_z + p.blen >= (uint32_t)ctx->nze - ctx->h)
        return fail(ctx, RTMB_EINVAL, "receiver depth outside the computed region");
    const int nw = rtmb_fmig_nw(p.dt, p.nt, fmin, fmax);
    if (nw <= 0) return fail(ctx, RTMB_EINVAL, "no frequency in [fmig_min_freq, fmig_max_freq) at df = 1/(nt dt)");
    int nws = (nwstep == 0 || (int)nwstep > nw) ? nw : (int)nwstep;
    if (nws > rtmb::kFmigMaxGroup) return fail(ctx, RTMB_EINVAL, "at most %d frequencies per group (nwstep)", rtmb::kFmigMaxGroup);
    std::vector<float> w2, kre, kim;
    fmig_tables(p, fmin, nw, w2, kre, kim);
    if ((rc = alloc_driver(ctx))) return rc;
    const size_t ni = (size_t)p.nx * p.ny * p.nz, need = 4 * (size_t)nws * ni;
    if (ctx->fq_cap < need) {
        if (ctx->d_fq) CK(cudaFree(ctx->d_fq));
        ctx->d_fq = nullptr;
        ctx->fq_cap = 0;
        CK(cudaMalloc(&ctx->d_fq, need * sizeof(float)));
        ctx->fq_cap = need;
    }
    const rtmb::Geom g = geom(ctx);
    const rtmb::RcvGeom rg = rgeom(ctx);
    const size_t nb = wave_bytes(ctx), rchunk = (size_t)rg.rcx * rg.rcy * p.ntstep;
    const int rmode = (p.flags & RTMB_FLAG_RCV_ADD) ? 3 : 2;
    const int quirk = !(p.flags & RTMB_FLAG_NO_TAPER_QUIRK);
    rtmb::StepArgs a = base_args(ctx);
    a.V = ctx->d_v2dt2;
    a.taper_mode = rtmb::kTaperNone;
    a.sxe = -1;  // the source is a separate operator here (after the taper)
    // Where the TMA step kernel runs, the fields stay tapered in HBM (StepArgs::tw): each step
    // stores T(raw) of its new level and applies T to PP on load, which is the reference's
    // "step, then taper P and PP in place" (the source and the receivers still come after it, as
    // separate operators; no source or receiver lies in the quirk edge).  No taper launches.
    const bool tw = tma_ok(ctx) && p.stencil_order <= 8 && ctx->nze % 4 == 0 && p.blen > 0 &&
                    !(p.flags & RTMB_FLAG_NO_TAPER_STORE);
    const size_t qn = quirk && p.blen > 0 ? (size_t)p.blen * (ctx->nze - 2 * p.blen) : 1;
    if (tw) {
        a.taper_mode = rtmb::kTaperAll;
        a.tw = 1;
        a.quirk = quirk && p.blen > 0;
        for (float *&b : ctx->d_fquirk)
            if ((rc = ensure(ctx, &b, qn > 0 ? qn : 1, false))) return rc;
    }
    GraphScope graph(ctx, 3);
    if ((rc = graph.begin())) return rc;
    CK(cudaMemsetAsync(img, 0, ctx->n * sizeof(float), ctx->stream));
    rtmb::FmigStep fs;
    for (int gw = 0; gw < nw; gw += nws) {
        const int m = nw - gw < nws ? nw - gw : nws;
        float *Ps = ctx->d_w[0], *PPs = ctx->d_w[1], *Pr = ctx->d_w[2], *PPr = ctx->d_w[3];
        for (int k = 0; k < 4; ++k) CK(cudaMemsetAsync(ctx->d_w[k], 0, nb, ctx->stream));
        if (tw)
            for (float *b : ctx->d_fquirk) CK(cudaMemsetAsync(b, 0, (qn > 0 ? qn : 1) * sizeof(float), ctx->stream));
        CK(cudaMemsetAsync(ctx->d_fq, 0, 4 * (size_t)nws * ni * sizeof(float), ctx->stream));
        fs.nws = m;
        for (uint32_t st = 0; st < p.nt; ++st) {
            const uint32_t rt = p.nt - 1 - st;
            for (int k = 0; k < 2; ++k) {  // rtmStepMultipleWave: both wavefields, the same v2dt2
                a.P = k ? Pr : Ps;
                a.PP = k ? PPr : PPs;
                a.it = (int)st;
                if (tw && a.quirk) {  // side buffers of this wavefield, rotating over three levels
                    a.quirk_in = ctx->d_fquirk[3 * k + (st + 1) % 3];
                    a.quirk_out = ctx->d_fquirk[3 * k + st % 3];
                }
                LAUNCH_CAT(RTMB_PROF_FMIG_STEP, rtmb::launch_step(a, (int)p.stencil_order, exact(ctx), ctx->stream, tma_ok(ctx)));
            }
            if (!tw) {
                float *tap[4] = {Ps, PPs, Pr, PPr};
                LAUNCH_CAT(RTMB_PROF_OTHER, rtmb::launch_taper_fields(tap, 4, ctx->d_taper, g, 0, quirk, ctx->stream));
            }
            LAUNCH_CAT(RTMB_PROF_OTHER, rtmb::launch_source(PPs, ctx->d_wavelet, (int)st, (int)(sx + p.blen),
                                                            (int)(sy + p.blen), (int)(sz + p.blen), g, ctx->stream));
            LAUNCH_CAT(RTMB_PROF_OTHER, rtmb::launch_receivers(PPr, const_cast<float *>(rec) + (size_t)(rt / p.ntstep) * rchunk,
                                                               (int)(rt % p.ntstep), rmode, rg, g, ctx->stream));
            for (int lw = 0; lw < m; ++lw) {
                fs.kre[lw] = kre[(size_t)(gw + lw) * p.nt + st];
                fs.kim[lw] = kim[(size_t)(gw + lw) * p.nt + st];
                fs.w2[lw] = w2[gw + lw];
            }
            LAUNCH_CAT(RTMB_PROF_FMIG_FREQ, rtmb::launch_fmig_freq(PPs, PPr, img, ctx->d_fq, fs, g, (int)p.nx, (int)p.ny,
                                                                   (int)p.nz, exact(ctx), ctx->stream));
            std::swap(Ps, PPs);
            std::swap(Pr, PPr);
        }
    }
    if ((rc = graph.end())) return rc;
    return check_err_flag(ctx);
}

int rtmb_migrate_shot_acc64(rtmb_ctx *ctx, uint32_t sx, uint32_t sy, uint32_t sz, const float *rec,
                            double *stack) {
    if (!ctx || !rec || !stack) return fail(ctx, RTMB_EINVAL, "rtmb_migrate_shot_acc64: null pointer");
    return migrate_impl(ctx, sx, sy, sz, rec, stack, true);
}

int rtmb_model_shot_host(rtmb_ctx *ctx, uint32_t sx, uint32_t sy, uint32_t sz, float *rec_host) {
    if (!ctx || !rec_host) return fail(ctx, RTMB_EINVAL, "rtmb_model_shot_host: null pointer");
    const size_t nrec = (size_t)ctx->p.nt * ctx->p.receiver_count_x * ctx->p.receiver_count_y;
    int rc = ensure(ctx, &ctx->d_rec, nrec ? nrec : 1, false);
    if (rc) return rc;
    if ((rc = rtmb_model_shot(ctx, sx, sy, sz, ctx->d_rec))) return rc;
    CK(cudaMemcpyAsync(rec_host, ctx->d_rec, nrec * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return RTMB_OK;
}

int rtmb_migrate_shot_host(rtmb_ctx *ctx, uint32_t sx, uint32_t sy, uint32_t sz, const float *rec_host,
                           float *img_host) {
    if (!ctx || !rec_host || !img_host) return fail(ctx, RTMB_EINVAL, "rtmb_migrate_shot_host: null pointer");
    const size_t nrec = (size_t)ctx->p.nt * ctx->p.receiver_count_x * ctx->p.receiver_count_y;
    int rc = ensure(ctx, &ctx->d_rec, nrec ? nrec : 1, false);
    if (rc) return rc;
    if ((rc = ensure(ctx, &ctx->d_img, ctx->n, false))) return rc;
    CK(cudaMemcpyAsync(ctx->d_rec, rec_host, nrec * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
    if ((rc = rtmb_migrate_shot(ctx, sx, sy, sz, ctx->d_rec, ctx->d_img))) return rc;
    CK(cudaMemcpyAsync(img_host, ctx->d_img, ctx->n * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return RTMB_OK;
}

// ------------------------------------------------------------------ batched multi-shot migration

}  // extern "C"

namespace {

// One shot of a batch: its padded geometry, buffers and the bookkeeping of its wavefields.
struct BatchShot {
    rtmb_shot in;
    int nxe = 0, nye = 0, nze = 0, chunk = 1;
    size_t n = 0;
    float *w[4] = {};  // source pair, receiver pair (FP32 or 16-bit)
    void *img = nullptr;
    rtmb::ScaleRec *scale = nullptr;
    int sc_next = 0, sc_cap = 0;
    float *inj = nullptr;
    rtmb::ScaleRec *next_scale() { return sc_next < sc_cap ? scale + sc_next++ : nullptr; }
};

rtmb::StepArgs shot_args(const rtmb_ctx *ctx, const BatchShot &b) {
    rtmb::StepArgs a = base_args(ctx);
    a.nxe = b.nxe; a.nye = b.nye; a.nze = b.nze;
    a.chunk = b.chunk;
    a.V = b.in.v2dt2;
    a.store = ctx->store;
    return a;
}

void shot_receivers(rtmb::StepArgs &a, const rtmb_ctx *ctx, const BatchShot &b, int mode, int it) {
    const int bl = (int)ctx->p.blen;
    const rtmb_shot &s = b.in;
    a.rec_mode = mode;
    a.rec = const_cast<float *>(s.rec);
    a.rx0 = (int)s.receiver_start_x + bl; a.ry0 = (int)s.receiver_start_y + bl; a.rz = (int)s.receiver_depth_z + bl;
    a.rdx = s.receiver_distance_x ? (int)s.receiver_distance_x : 1;
    a.rdy = s.receiver_distance_y ? (int)s.receiver_distance_y : 1;
    a.rcx = (int)s.receiver_count_x; a.rcy = (int)s.receiver_count_y;
    const long long ntstep = ctx->p.ntstep;
    a.rec_si = (long long)a.rcy * ntstep;
    a.rec_sj = ntstep;
    a.rec_base = (long long)(it / ntstep) * a.rcx * a.rcy * ntstep + (it % ntstep);
}

}  // namespace

extern "C" {

}  // extern "C"

namespace {

// One group of at most kMaxBatch shots of rtmb_migrate_batch: their per-shot state is allocated
// here, their time loops advance together (one launch per step for the group, one CUDA graph with
// RTMB_FLAG_USE_GRAPH), and their images are added to the survey stack.  With forward_only, only
// `steps` forward steps run (the autotuner's measurement; nothing is stacked) and *ms receives
// their mean device time.
int migrate_group(rtmb_ctx *ctx, uint32_t nshots, const rtmb_shot *shots, double *stack, uint32_t snx,
                  uint32_t sny, uint32_t snz, int forward_only = 0, float *ms = nullptr) {
    const rtmb_params &p = ctx->p;
    const bool st = ctx->store != rtmb::kStoreF32;
    const size_t es = st ? 2 : 4;
    const bool img64 = st;  // the 16-bit forms stack through an FP64 shot image, FP32 through FP32
    const int bl = (int)p.blen;
    std::vector<BatchShot> sh(nshots);
    // allocation and checks
    size_t total_tiles = 0;
    for (uint32_t k = 0; k < nshots; ++k) {
        BatchShot &b = sh[k];
        b.in = shots[k];
        const rtmb_shot &s = b.in;
        if (!s.v2dt2 || !s.rec || !s.nx || !s.ny || !s.nz || s.sx >= s.nx || s.sy >= s.ny || s.sz >= s.nz ||
            s.receiver_count_x > s.nx || s.receiver_count_y > s.ny || s.receiver_depth_z + 2 * bl + ctx->h > s.nz + 2 * bl)
            return fail(ctx, RTMB_EINVAL, "rtmb_migrate_batch: shot %u: bad geometry", k);
        b.nxe = (int)s.nx + 2 * bl; b.nye = (int)s.ny + 2 * bl; b.nze = (int)s.nz + 2 * bl;
        if (b.nze % (st ? 8 : 4))
            return fail(ctx, RTMB_EINVAL, "rtmb_migrate_batch: shot %u: nz + 2*blen must be a multiple of %d", k,
                        st ? 8 : 4);
        b.n = (size_t)b.nxe * b.nye * b.nze;
        total_tiles += (size_t)((b.nze + rtmb::kTZ - 1) / rtmb::kTZ) * ((b.nye - 8 + rtmb::kTY - 1) / rtmb::kTY);
    }
    int rc = RTMB_OK;
    auto release = [&]() {
        for (BatchShot &b : sh) {
            for (float *w : b.w) if (w) cudaFree(w);
            if (b.img) cudaFree(b.img);
            if (b.scale) cudaFree(b.scale);
            if (b.inj) cudaFree(b.inj);
        }
    };
    for (BatchShot &b : sh) {
        // x planes per CTA: the batch shares the usual CTA budget of several waves on 148 SMs
        const int nxi = b.nxe - 8;
        const size_t target = 148 * 2 * 4;
        const size_t tiles = (size_t)((b.nze + rtmb::kTZ - 1) / rtmb::kTZ) * ((b.nye - 8 + rtmb::kTY - 1) / rtmb::kTY);
        size_t nch = (target * tiles / (total_tiles ? total_tiles : 1) + tiles - 1) / tiles;
        if (nch < 1) nch = 1;
        if (nch > (size_t)(nxi / 16 > 0 ? nxi / 16 : 1)) nch = nxi / 16 > 0 ? nxi / 16 : 1;
        b.chunk = (int)((nxi + nch - 1) / nch);
        bool ok = true;
        for (float *&w : b.w) ok = ok && cudaMalloc(&w, b.n * es) == cudaSuccess;
        ok = ok && cudaMalloc(&b.img, b.n * (img64 ? 8 : 4)) == cudaSuccess;
        if (st) {
            b.sc_cap = 3 * (int)p.nt + 8;
            ok = ok && cudaMalloc(&b.scale, b.sc_cap * sizeof(rtmb::ScaleRec)) == cudaSuccess &&
                 cudaMalloc(&b.inj, sizeof(float)) == cudaSuccess;
        }
        if (!ok) { release(); return fail(ctx, RTMB_ENOMEM, "rtmb_migrate_batch: device allocation failed"); }
        for (float *w : b.w) cudaMemsetAsync(w, 0, b.n * es, ctx->stream);
        cudaMemsetAsync(b.img, 0, b.n * (img64 ? 8 : 4), ctx->stream);
        if (st) {
            cudaMemsetAsync(b.scale, 0, b.sc_cap * sizeof(rtmb::ScaleRec), ctx->stream);
            const size_t nrec = (size_t)p.nt * b.in.receiver_count_x * b.in.receiver_count_y;
            if (rtmb::launch_absmax(b.in.rec, nrec, b.inj, ctx->stream) != cudaSuccess) {
                release();
                return fail(ctx, RTMB_ECUDA, "rtmb_migrate_batch: record scan failed");
            }
            ++ctx->launches;
        }
    }
    const int order = (int)p.stencil_order;
    std::vector<rtmb::StepArgs> args(nshots);
    // per shot: the source pair (P, PP) with scale records, the receiver pair likewise
    std::vector<float *> sP(nshots), sPP(nshots), rP(nshots), rPP(nshots);
    std::vector<rtmb::ScaleRec *> scP(nshots), scPP(nshots), srP(nshots), srPP(nshots);
    for (uint32_t k = 0; k < nshots; ++k) {
        sP[k] = sh[k].w[0]; sPP[k] = sh[k].w[1]; rP[k] = sh[k].w[2]; rPP[k] = sh[k].w[3];
        if (st) {
            scP[k] = sh[k].next_scale(); scPP[k] = sh[k].next_scale();
            srP[k] = sh[k].next_scale(); srPP[k] = sh[k].next_scale();
        }
    }
    if (forward_only) {  // the autotuner's measurement: forward steps of this group
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        bool ok = cudaEventCreate(&e0) == cudaSuccess && cudaEventCreate(&e1) == cudaSuccess;
        for (int it = 0; ok && it < forward_only + 2; ++it) {
            if (it == 2) ok = cudaEventRecord(e0, ctx->stream) == cudaSuccess;
            for (uint32_t k = 0; k < nshots; ++k) {
                rtmb::StepArgs &a = args[k];
                a = shot_args(ctx, sh[k]);
                a.P = sP[k]; a.PP = sPP[k]; a.it = 0;
                if (st) { a.sc_p = scP[k]; a.sc_pp = scPP[k]; a.sc_out = srP[k]; a.inj = ctx->wmax; }
            }
            ++ctx->launches;
            ok = ok && rtmb::launch_step_batch(args.data(), (int)nshots, order, exact(ctx), ctx->stream) == cudaSuccess;
        }
        ok = ok && cudaEventRecord(e1, ctx->stream) == cudaSuccess && cudaEventSynchronize(e1) == cudaSuccess &&
             cudaEventElapsedTime(ms, e0, e1) == cudaSuccess;
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
        if (ms) *ms /= forward_only;
        cudaStreamSynchronize(ctx->stream);
        release();
        return ok ? RTMB_OK : fail(ctx, RTMB_ECUDA, "rtmb_autotune_batch: measurement failed");
    }
    {
        GraphScope graph(ctx, 2);
        if ((rc = graph.begin())) { release(); return rc; }
        // forward (RBC.cpp:54-144), all shots per launch
        for (uint32_t it = 0; it < p.nt && !rc; ++it) {
            for (uint32_t k = 0; k < nshots; ++k) {
                std::swap(sP[k], sPP[k]);
                std::swap(scP[k], scPP[k]);
                rtmb::StepArgs &a = args[k];
                a = shot_args(ctx, sh[k]);
                a.P = sP[k]; a.PP = sPP[k]; a.it = (int)it;
                a.sxe = (int)sh[k].in.sx + bl; a.sye = (int)sh[k].in.sy + bl; a.sze = (int)sh[k].in.sz + bl;
                if (st) { a.sc_p = scP[k]; a.sc_pp = scPP[k]; a.sc_out = sh[k].next_scale(); a.inj = ctx->wmax; }
            }
            const size_t slot = prof_begin(ctx, RTMB_PROF_FORWARD);
            ++ctx->launches;
            if (rtmb::launch_step_batch(args.data(), (int)nshots, order, exact(ctx), ctx->stream) != cudaSuccess)
                rc = fail(ctx, RTMB_ECUDA, "rtmb_migrate_batch: forward launch failed");
            prof_end(ctx, slot);
            if (st) for (uint32_t k = 0; k < nshots; ++k) scPP[k] = args[k].sc_out;
        }
        // backward (RBC.cpp:146-274): s_cur images the receiver wavefield each step
        std::vector<float *> cur(nshots), prev(nshots);
        std::vector<rtmb::ScaleRec *> scur(nshots), sprev(nshots);
        for (uint32_t k = 0; k < nshots; ++k) { cur[k] = sPP[k]; prev[k] = sP[k]; scur[k] = scPP[k]; sprev[k] = scP[k]; }
        const int rmode = (p.flags & RTMB_FLAG_RCV_ADD) ? rtmb::kRecAdd : rtmb::kRecOverwrite;
        for (int it = (int)p.nt - 1; it >= 0 && !rc; --it) {
            if (it == (int)p.nt - 2) {
                for (uint32_t k = 0; k < nshots; ++k) {
                    std::swap(cur[k], prev[k]);
                    std::swap(scur[k], sprev[k]);
                }
            } else if (it < (int)p.nt - 2) {
                for (uint32_t k = 0; k < nshots; ++k) {
                    rtmb::StepArgs &a = args[k];
                    a = shot_args(ctx, sh[k]);
                    a.P = cur[k]; a.PP = prev[k]; a.it = it;
                    if (st) { a.sc_p = scur[k]; a.sc_pp = sprev[k]; a.sc_out = sh[k].next_scale(); }
                }
                const size_t slot = prof_begin(ctx, RTMB_PROF_BACKWARD_SOURCE);
                ++ctx->launches;
                if (rtmb::launch_step_batch(args.data(), (int)nshots, order, exact(ctx), ctx->stream) != cudaSuccess)
                    rc = fail(ctx, RTMB_ECUDA, "rtmb_migrate_batch: source launch failed");
                prof_end(ctx, slot);
                for (uint32_t k = 0; k < nshots; ++k) {
                    std::swap(cur[k], prev[k]);
                    if (st) { sprev[k] = scur[k]; scur[k] = args[k].sc_out; }
                }
            }
            for (uint32_t k = 0; k < nshots; ++k) {
                rtmb::StepArgs &a = args[k];
                a = shot_args(ctx, sh[k]);
                a.P = rP[k]; a.PP = rPP[k]; a.it = it;
                a.ps = cur[k];
                a.img = static_cast<float *>(sh[k].img);
                a.img64 = img64;
                a.img_z0 = bl; a.img_z1 = sh[k].nze - bl;
                shot_receivers(a, ctx, sh[k], rmode, it);
                if (st) {
                    a.sc_p = srP[k]; a.sc_pp = srPP[k]; a.sc_out = sh[k].next_scale(); a.sc_ps = scur[k];
                    a.inj_dev = sh[k].inj;
                }
            }
            const size_t slot = prof_begin(ctx, RTMB_PROF_BACKWARD_RECEIVER);
            ++ctx->launches;
            if (rtmb::launch_step_batch(args.data(), (int)nshots, order, exact(ctx), ctx->stream) != cudaSuccess)
                rc = fail(ctx, RTMB_ECUDA, "rtmb_migrate_batch: receiver launch failed");
            prof_end(ctx, slot);
            for (uint32_t k = 0; k < nshots; ++k) {
                std::swap(rP[k], rPP[k]);
                if (st) { srPP[k] = srP[k]; srP[k] = args[k].sc_out; }
            }
        }
        // each shot's image without its border into the survey stack (RTMGrid.cpp:168-223)
        for (uint32_t k = 0; k < nshots && !rc; ++k) {
            const rtmb::Geom g{sh[k].nxe, sh[k].nye, sh[k].nze, bl, ctx->h};
            ++ctx->launches;
            if (rtmb::launch_stack_region64(stack, (int)snx, (int)sny, (int)snz, sh[k].img, img64, g, (int)sh[k].in.ox,
                                            (int)sh[k].in.oy, (int)sh[k].in.oz, ctx->stream) != cudaSuccess)
                rc = fail(ctx, RTMB_ECUDA, "rtmb_migrate_batch: stacking failed");
        }
        if (!rc) rc = graph.end();
    }
    if (!rc) rc = check_err_flag(ctx);
    cudaStreamSynchronize(ctx->stream);
    release();
    return rc;
}

}  // namespace

extern "C" {

int rtmb_migrate_batch(rtmb_ctx *ctx, uint32_t nshots, const rtmb_shot *shots, double *stack, uint32_t snx,
                       uint32_t sny, uint32_t snz) {
    if (!ctx || !shots || !stack) return fail(ctx, RTMB_EINVAL, "rtmb_migrate_batch: null pointer");
    const rtmb_params &p = ctx->p;
    if (nshots == 0) return fail(ctx, RTMB_EINVAL, "rtmb_migrate_batch: no shots");
    if (ctx->diff) return fail(ctx, RTMB_EINVAL, "rtmb_migrate_batch: the increment storage form runs single shots");
    if (p.boundary != RTMB_BC_RBC || p.stencil_order != 8 || (int)p.blen < ctx->h || p.nx == 1)
        return fail(ctx, RTMB_EINVAL, "rtmb_migrate_batch: boundary RBC, stencil_order 8, blen >= 4, 3D (nx > 1)");
    // groups of batch_group shots, in order: each group's time loop runs with its shots together
    const uint32_t g = (uint32_t)ctx->batch_group;
    for (uint32_t k0 = 0; k0 < nshots; k0 += g) {
        const int rc = migrate_group(ctx, nshots - k0 < g ? nshots - k0 : g, shots + k0, stack, snx, sny, snz);
        if (rc) return rc;
    }
    return RTMB_OK;
}

int rtmb_set_batch_group(rtmb_ctx *ctx, uint32_t shots_per_launch) {
    if (!ctx || shots_per_launch == 0 || shots_per_launch > (uint32_t)rtmb::kMaxBatchShots)
        return fail(ctx, RTMB_EINVAL, "rtmb_set_batch_group: 1 to %d shots per launch", rtmb::kMaxBatchShots);
    ctx->batch_group = (int)shots_per_launch;
    return RTMB_OK;
}

int rtmb_autotune_batch(rtmb_ctx *ctx, uint32_t nshots, const rtmb_shot *shots, uint32_t *group_out, float *rate_out) {
    if (!ctx || !shots || nshots == 0) return fail(ctx, RTMB_EINVAL, "rtmb_autotune_batch: no shots");
    if (ctx->diff) return fail(ctx, RTMB_EINVAL, "rtmb_autotune_batch: the increment storage form runs single shots");
    const rtmb_params &p = ctx->p;
    if (p.boundary != RTMB_BC_RBC || p.stencil_order != 8 || (int)p.blen < ctx->h || p.nx == 1)
        return fail(ctx, RTMB_EINVAL, "rtmb_autotune_batch: boundary RBC, stencil_order 8, blen >= 4, 3D (nx > 1)");
    // the rate (padded points per ms) of the batched forward step for each group size, measured
    // on the first shots of the batch
    const uint32_t cand[] = {1, 2, 3, 4, 6, 8, 12, 16, 24};
    float best = 0.f;
    uint32_t best_g = (uint32_t)ctx->batch_group;
    for (uint32_t g : cand) {
        if (g > nshots || g > (uint32_t)rtmb::kMaxBatchShots) break;
        float ms = 0.f;
        const int rc = migrate_group(ctx, g, shots, nullptr, 0, 0, 0, 5, &ms);
        if (rc) return rc;
        double pts = 0;
        for (uint32_t k = 0; k < g; ++k)
            pts += (double)(shots[k].nx + 2 * p.blen) * (shots[k].ny + 2 * p.blen) * (shots[k].nz + 2 * p.blen);
        const float rate = ms > 0.f ? (float)(pts / ms) : 0.f;
        if (rate > best) { best = rate; best_g = g; }
    }
    ctx->batch_group = (int)best_g;
    if (group_out) *group_out = best_g;
    if (rate_out) *rate_out = best * 1e-6f;  // G point-updates per second
    return check_err_flag(ctx);
}


// ------------------------------------------------------------------ autotuner

}  // extern "C"

namespace {

// Mean time (ms) of `reps` launches of fn after `warm` untimed ones, on the context's stream.
template <typename F>
int time_launches(rtmb_ctx *ctx, cudaEvent_t e0, cudaEvent_t e1, F fn, float *ms, int warm = 2, int reps = 5) {
    for (int w = 0; w < warm; ++w) LAUNCH(fn());
    CK(cudaEventRecord(e0, ctx->stream));
    for (int r = 0; r < reps; ++r) LAUNCH(fn());
    CK(cudaEventRecord(e1, ctx->stream));
    CK(cudaEventSynchronize(e1));
    CK(cudaEventElapsedTime(ms, e0, e1));
    *ms /= reps;
    return RTMB_OK;
}

}  // namespace

extern "C" {

int rtmb_autotune_full(rtmb_ctx *ctx, rtmb_tuning *out) {
    if (!ctx) return RTMB_EINVAL;
    if (!ctx->d_v2dt2) return fail(ctx, RTMB_EINVAL, "rtmb_autotune: load v2dt2 first");
    int rc = alloc_driver(ctx);
    if (rc) return rc;
    const rtmb_params &p = ctx->p;
    const bool st = ctx->store != rtmb::kStoreF32;
    const int order = (int)p.stencil_order;
    // scratch of the measurement: scale records (16-bit forms) and an image volume
    rtmb::ScaleRec *rec5 = nullptr;
    if (st) {
        CK(cudaMalloc(&rec5, 5 * sizeof(rtmb::ScaleRec)));
        CK(cudaMemsetAsync(rec5, 0, 5 * sizeof(rtmb::ScaleRec), ctx->stream));
    }
    void *img = nullptr;
    const size_t img_bytes = ctx->n * (ctx->img64 ? sizeof(double) : sizeof(float));
    CK(cudaMalloc(&img, img_bytes));
    CK(cudaMemsetAsync(img, 0, img_bytes, ctx->stream));
    for (int k = 0; k < 4; ++k) CK(cudaMemsetAsync(ctx->d_w[k], 0, wave_bytes(ctx), ctx->stream));
    for (int k = 0; ctx->diff && k < 2; ++k) CK(cudaMemsetAsync(ctx->d_inc[k], 0, wave_bytes(ctx), ctx->stream));
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    auto release = [&]() {
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (rec5) cudaFree(rec5);
        cudaFree(img);
    };
    // the step forms of the context: forward (no image) and receiver (image of the source level)
    auto args = [&](bool with_img) {
        rtmb::StepArgs a = base_args(ctx);
        a.V = ctx->d_v2dt2;
        a.P = ctx->d_w[0];
        a.PP = ctx->d_w[1];
        a.store = ctx->store;
        if (st) { a.sc_p = rec5; a.sc_pp = rec5 + 1; a.sc_out = rec5 + 2; a.sc_out2 = rec5 + 3; a.inj = 1.f; }
        if (ctx->diff) { a.diff = 1; a.Pout = ctx->d_w[2]; a.PP = static_cast<float *>(ctx->d_inc[0]); }
        if (with_img) {
            a.img = static_cast<float *>(img);
            a.img64 = ctx->img64;
            a.ps = ctx->d_w[3];
            a.sc_ps = rec5 ? rec5 + 4 : nullptr;
            a.img_z0 = 0;
            a.img_z1 = ctx->nze;
        }
        return a;
    };
    const int nxi = ctx->nxe - 2 * ctx->h;
    const int cand[] = {8, 12, 16, 24, 32, 48, 64, 96, 128, 192, 256};
    // launch variants exist for the FP32 forms without taper at order 8 on the TMA kernel
    const bool variants = !st && order == 8 && tma_ok(ctx) && ctx->nze % 4 == 0;
    const int nv = variants ? rtmb::kStepVariants : 1;
    float best = 1e30f, best_fwd = 0.f;
    int best_v = 0, best_c = ctx->chunk;
    for (int v = 0; v < nv && !rc; ++v) {
        for (int c : cand) {
            if (c > nxi) break;
            ctx->variant = v;
            ctx->chunk = c;
            rtmb::StepArgs af = args(false), ai = args(true);
            float tf = 0.f, ti = 0.f;
            if ((rc = time_launches(ctx, e0, e1, [&] { return rtmb::launch_step(af, order, exact(ctx), ctx->stream, tma_ok(ctx)); }, &tf)))
                break;
            if ((rc = time_launches(ctx, e0, e1, [&] { return rtmb::launch_step(ai, order, exact(ctx), ctx->stream, tma_ok(ctx)); }, &ti)))
                break;
            if (tf + ti < best) { best = tf + ti; best_fwd = tf; best_v = v; best_c = c; }
        }
    }
    if (rc) { release(); return rc; }
    ctx->variant = best_v;
    ctx->chunk = best_c;
    // backward time step: the dual launch against the source and receiver steps as two launches
    float two = 0.f;
    {
        rtmb::StepArgs as = args(false), ai = args(true);
        rc = time_launches(ctx, e0, e1, [&] {
            cudaError_t e = rtmb::launch_step(as, order, exact(ctx), ctx->stream, tma_ok(ctx));
            return e != cudaSuccess ? e : rtmb::launch_step(ai, order, exact(ctx), ctx->stream, tma_ok(ctx));
        }, &two);
    }
    const bool dual_ok = !rc && !st && order == 8 && tma_ok(ctx) && !(p.flags & RTMB_FLAG_NO_DUAL) &&
                         p.nx > 1 && p.boundary == RTMB_BC_RBC;
    float best_dual = 1e30f;
    int best_dc = ctx->dual_chunk, best_dv = ctx->dual_variant;
    for (int dv = 0; dv < rtmb::kDualVariants && dual_ok && !rc; ++dv) {
        for (int c : cand) {
            if (rc || c > nxi) break;
            rtmb::StepArgs src = args(false), rcv = args(true);
            src.P = ctx->d_w[0]; src.PP = ctx->d_w[1];
            rcv.P = ctx->d_w[2]; rcv.PP = ctx->d_w[3]; rcv.ps = nullptr;
            rcv.chunk = c;
            rcv.variant = dv;
            if (!rtmb::dual_step_supported(src, rcv, order)) break;
            float t = 0.f;
            if ((rc = time_launches(ctx, e0, e1, [&] { return rtmb::launch_dual_step(src, rcv, order, exact(ctx), ctx->stream); },
                                    &t)))
                break;
            if (t < best_dual) { best_dual = t; best_dc = c; best_dv = dv; }
        }
    }
    release();
    if (rc) return rc;
    ctx->dual_chunk = best_dc;
    ctx->dual_variant = best_dv;
    ctx->use_dual = dual_ok ? (best_dual < two ? 1 : 0) : -1;
    if (out) {
        out->variant = (uint32_t)ctx->variant;
        out->chunk = (uint32_t)ctx->chunk;
        out->dual = ctx->use_dual == 1;
        out->dual_chunk = (uint32_t)ctx->dual_chunk;
        out->ms_step = best_fwd;
        out->ms_backward = ctx->use_dual == 1 ? best_dual : two;
        out->dual_variant = (uint32_t)ctx->dual_variant;
    }
    return check_err_flag(ctx);
}

int rtmb_set_tuning(rtmb_ctx *ctx, const rtmb_tuning *t) {
    if (!ctx || !t || !t->chunk || !t->dual_chunk || t->variant >= (uint32_t)rtmb::kStepVariants ||
        t->dual_variant >= (uint32_t)rtmb::kDualVariants)
        return fail(ctx, RTMB_EINVAL, "rtmb_set_tuning: bad tuning");
    ctx->variant = (int)t->variant;
    ctx->dual_variant = (int)t->dual_variant;
    ctx->chunk = (int)t->chunk;
    ctx->dual_chunk = (int)t->dual_chunk;
    ctx->use_dual = t->dual ? 1 : 0;
    return RTMB_OK;
}

int rtmb_autotune(rtmb_ctx *ctx, uint32_t *chunk_out, float *ms_out) {
    rtmb_tuning t{};
    const int rc = rtmb_autotune_full(ctx, &t);
    if (rc) return rc;
    if (chunk_out) *chunk_out = t.chunk;
    if (ms_out) *ms_out = t.ms_step;
    return RTMB_OK;
}

int rtmb_set_chunk(rtmb_ctx *ctx, uint32_t chunk) {
    if (!ctx || !chunk) return RTMB_EINVAL;
    ctx->chunk = (int)chunk;
    return RTMB_OK;
}

}  // extern "C"
