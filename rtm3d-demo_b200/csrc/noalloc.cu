// noalloc.cu -- rtmb_model_shot_noalloc: the modeling driver for callers that cannot allocate
// device memory.
//
// Some hosts cannot call cudaMalloc: a framework whose allocator has already reserved the GPU's
// memory and accounts for every byte, or a latency-sensitive loop where cudaMalloc's implicit device
// synchronisation is not acceptable.  This entry point runs the same modeling shot as
// rtmb_model_shot (same kernels, same results) without creating a context: the caller passes v2dt2
// and the record, and every other buffer the shot needs lives in g_scratch below, a file-scope
// device array that each GPU which loads the library holds until the process exits.
#include <cstring>
#include <mutex>

#include "ctx.hpp"
#include "host_math.hpp"

namespace {

// Capacity of the shared scratch: 64 MiB.  It holds two wavefields of the padded grid plus the
// taper side buffers and the taper and Ricker tables, so grids up to about 8.3 million padded
// points (for example 200^3) fit.
constexpr size_t kScratchFloats = size_t(16) << 20;
static __device__ __align__(256) float g_scratch[kScratchFloats];

constexpr int kMaxDevices = 64;
float *g_scratch_ptr[kMaxDevices] = {};
std::mutex g_setup_mutex;

// Device address of g_scratch on the current device, resolved once per device.  In host code the
// name g_scratch is a host-side stand-in, not a device address, so kernels only ever get this
// pointer.
int scratch_on(int dev, float **out) {
    if (dev < 0 || dev >= kMaxDevices)
        return rtmb::driver::fail_noctx(RTMB_EINVAL, "rtmb_model_shot_noalloc: device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_ptr[dev]) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
        if (e != cudaSuccess || !p)
            return rtmb::driver::fail_noctx(RTMB_ECUDA, "rtmb_model_shot_noalloc: cudaGetSymbolAddress failed");
        g_scratch_ptr[dev] = static_cast<float *>(p);
    }
    *out = g_scratch_ptr[dev];
    return RTMB_OK;
}

size_t align_floats(size_t n) { return (n + 63) & ~size_t(63); }  // 256-byte sections

// Longest taper table (blen) the entry point takes: the tables go up through a stack buffer of
// this many floats.
constexpr uint32_t kMaxBlen = 1024;

// Is p memory that kernels on device dev may read and write: device memory of dev, or managed
// memory?  cudaPointerGetAttributes allocates nothing.
bool device_buffer(const void *p, int dev) {
    cudaPointerAttributes at{};
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        (void)cudaGetLastError();
        return false;
    }
    if (at.type == cudaMemoryTypeManaged) return true;
    return at.type == cudaMemoryTypeDevice && at.device == dev;
}

}  // namespace

extern "C" int rtmb_model_shot_noalloc(const rtmb_params *params, const float *v2dt2, uint32_t sx, uint32_t sy,
                                       uint32_t sz, float *rec, void *cuda_stream) {
    using rtmb::driver::fail_noctx;
    if (!params || !v2dt2 || !rec) return fail_noctx(RTMB_EINVAL, "rtmb_model_shot_noalloc: null pointer");
    const rtmb_params &p = *params;
    if (!p.nx || !p.ny || !p.nz || p.stencil_order < 2 || p.stencil_order > 16 || (p.stencil_order & 1u) ||
        !p.ntstep || p.nt % p.ntstep)
        return fail_noctx(RTMB_EINVAL, "rtmb_model_shot_noalloc: invalid parameters");
    if (p.flags & (RTMB_FLAG_STORE_F16 | RTMB_FLAG_STORE_BF16 | RTMB_FLAG_IMG_F64))
        return fail_noctx(RTMB_EINVAL, "rtmb_model_shot_noalloc: the 16-bit storage forms need a context");
    // the learned closure needs its parameters and strip tables, which only a context holds
    if (p.boundary == RTMB_BC_LEARNED)
        return fail_noctx(RTMB_EINVAL, "rtmb_model_shot_noalloc: boundary RTMB_BC_LEARNED needs a context");
    // the taper table is uploaded through a 1024-float stack buffer
    if (p.blen > kMaxBlen)
        return fail_noctx(RTMB_EINVAL, "rtmb_model_shot_noalloc: blen above 1024");

    // a context on the stack: it owns nothing, every device pointer below points into g_scratch or
    // at the caller's buffers
    rtmb_ctx c;
    c.p = p;
    rtmb::driver::init_geometry(&c);
    const size_t qn = (size_t)p.blen * (size_t)(c.nze > 2 * (int)p.blen ? c.nze - 2 * (int)p.blen : 1);
    const size_t off_err = 0, off_taper = 64, off_wav = off_taper + align_floats(p.blen ? p.blen : 1);
    const size_t off_q = off_wav + align_floats(p.nt);
    const size_t off_w0 = off_q + 3 * align_floats(qn);
    const size_t off_w1 = off_w0 + align_floats(c.n);
    const size_t need = off_w1 + align_floats(c.n);
    if (need > kScratchFloats)
        return fail_noctx(RTMB_EINVAL,
                          "rtmb_model_shot_noalloc: the grid needs more than the 64 MiB scratch (two padded "
                          "wavefields of at most ~8.3 million points); use rtmb_model_shot");

    int dev = p.device;
    if (dev < 0) {
        if (cudaGetDevice(&dev) != cudaSuccess) return fail_noctx(RTMB_ECUDA, "cudaGetDevice failed");
    } else if (cudaSetDevice(dev) != cudaSuccess) {
        return fail_noctx(RTMB_ECUDA, "cudaSetDevice failed");
    }
    // v2dt2 and rec go straight to the kernels: accept only device (or managed) memory of this
    // device, so a host or stale pointer is an error here and not a fault on the GPU
    if (!device_buffer(v2dt2, dev) || !device_buffer(rec, dev))
        return fail_noctx(RTMB_EINVAL,
                          "rtmb_model_shot_noalloc: v2dt2 and rec must be device memory of the call's device");
    float *scr = nullptr;
    int rc = scratch_on(dev, &scr);
    if (rc) return rc;

    c.device = dev;
    c.stream = static_cast<cudaStream_t>(cuda_stream);  // NULL: the legacy default stream
    c.d_err = reinterpret_cast<unsigned *>(scr + off_err);
    c.d_taper = scr + off_taper;
    c.d_wavelet = scr + off_wav;
    for (int k = 0; k < 3; ++k) c.d_quirk[k] = scr + off_q + k * align_floats(qn);
    c.d_w[0] = scr + off_w0;
    c.d_w[1] = scr + off_w1;
    c.d_v2dt2 = const_cast<float *>(v2dt2);
    if ((rc = rtmb::driver::check_model_shot(&c, sx, sy, sz))) return fail_noctx(rc, c.err.c_str());

    // tables computed on the host (bit-identical to the reference) and copied into the scratch in
    // chunks through a stack buffer; each copy is complete before the buffer is refilled
    float buf[kMaxBlen];
    bool ok = true;
    if (p.blen) {
        ok = rtmb_taper_vector(p.blen, p.taper_factor, buf) == RTMB_OK &&
             cudaMemcpyAsync(c.d_taper, buf, p.blen * sizeof(float), cudaMemcpyHostToDevice, c.stream) == cudaSuccess &&
             cudaStreamSynchronize(c.stream) == cudaSuccess;
    }
    for (uint32_t i = 0; ok && i < p.nt; i += kMaxBlen) {
        const uint32_t m = p.nt - i < kMaxBlen ? p.nt - i : kMaxBlen;
        for (uint32_t k = 0; k < m; ++k) buf[k] = rtmb::ricker_sample(i + k, p.dt, p.fpeak);
        ok = cudaMemcpyAsync(c.d_wavelet + i, buf, m * sizeof(float), cudaMemcpyHostToDevice, c.stream) == cudaSuccess &&
             cudaStreamSynchronize(c.stream) == cudaSuccess;
    }
    if (!ok) return fail_noctx(RTMB_ECUDA, "rtmb_model_shot_noalloc: table upload failed");
    // the scratch keeps the previous call's contents: clear what must start at zero
    if (cudaMemsetAsync(c.d_err, 0, sizeof(unsigned), c.stream) != cudaSuccess)
        return fail_noctx(RTMB_ECUDA, "rtmb_model_shot_noalloc: memset failed");

    float *P = nullptr, *PP = nullptr;
    if ((rc = rtmb::driver::run_forward(&c, sx, sy, sz, rtmb::kTaperAll, rec, nullptr, &P, &PP, RTMB_PROF_MODEL)))
        return fail_noctx(rc, c.err.c_str());
    if ((rc = rtmb::driver::check_err_flag(&c))) return fail_noctx(rc, c.err.c_str());
    return RTMB_OK;
}
