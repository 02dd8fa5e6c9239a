// stencil.cuh -- the fused time-step kernel of librtm3d_b200 (sm_100a).
//
// One launch advances one wavefield one time step:
//     PP <- 2 T(P) - T(T(PP)) + v2dt2 * lap(T(P))        on [h, n-h)^3, h = order/2
// (RTMCPUPlatform::rtmStep3D, RTMCPUPlatform.cpp:325-395) where T is the reference's border taper
// (taper3D / taperUpper3D, RTMCPUPlatform.cpp:566-920) or the identity.  The reference tapers P
// and PP in place before every step, so a wavefield is tapered once as "P" and a second time as
// "PP" on the next step; here the wavefields stay RAW in HBM and the kernel applies T (and T o T)
// to the values it loads, which makes the taper free of HBM traffic.  The epilogue fuses what the
// reference runs as separate launches after the step: Ricker injection, receiver sampling or
// injection, upper-border (UPB) save/restore and the cross-correlation image.
//
// Data layout: x slowest, z fastest (RTMGrid.hpp:217-221).  A CTA owns a TZ x TY tile of the
// (y, z) plane and streams along x over a chunk of planes.  Each thread computes VZ consecutive
// z-points of one y row; the x-direction taps live in a per-thread register queue of 2H+1 planes,
// the y/z taps come from a double-buffered shared-memory copy of the current plane plus halo.
// Loads for plane x+1 are issued before the arithmetic of plane x.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace rtmb {

constexpr int kTZ = 64;      // tile extent along z (contiguous), floats
constexpr int kTY = 16;      // tile extent along y
constexpr int kVZ = 4;       // z-points per thread
constexpr int kThreads = (kTZ / kVZ) * kTY;  // 256
constexpr int kMaxOrder = 16;

enum TaperMode : int { kTaperNone = 0, kTaperUpper = 1, kTaperAll = 2 };
enum RecMode : int { kRecNone = 0, kRecSample = 1, kRecOverwrite = 2, kRecAdd = 3 };
enum UpbMode : int { kUpbNone = 0, kUpbSave = 1, kUpbRestore = 2 };

struct StepArgs {
    // geometry (padded sizes)
    int nxe, nye, nze, blen;
    int chunk;                  // x planes per CTA
    // stencil coefficients, [order+1] per axis
    float cx[kMaxOrder + 1], cy[kMaxOrder + 1], cz[kMaxOrder + 1];
    // wavefields
    const float *P;
    float *PP;
    const float *V;
    // taper
    const float *taper;         // blen factors (RTMTaperFunction)
    int taper_mode;             // TaperMode
    int quirk;                  // front-right x-y edge reads x = blen (taper3D, :901)
    const float *quirk_in;      // [blen][nze-2blen]: raw PP(blen, nye-blen+j, blen+k) of this PP
    float *quirk_out;           // same, receives PP_new(blen, ...)
    // source: PP[sxe,sye,sze] += wavelet[it]
    const float *wavelet;
    int it;
    int sxe, sye, sze;          // sxe < 0: no source
    // receivers
    int rec_mode;               // RecMode
    float *rec;
    long long rec_base;         // offset of (i=0, j=0) for this time step
    long long rec_si, rec_sj;   // strides of receiver index i (x) and j (y)
    int rx0, ry0, rz, rdx, rdy, rcx, rcy;  // padded receiver grid
    // upper border: planes z in [blen-h, blen), layout [nxe][nye][h] for this time step
    int upb_mode;               // UpbMode
    float *upb;
    // image: img += ps * PP_new on z in [img_z0, img_z1)
    float *img;
    const float *ps;
    int img_z0, img_z1;
    // error flags (bit 0: NaN)
    unsigned int *err;
};

// Launch one step.  Selects the instantiation for order/2 and the alignment of the arrays.
// allow_tma = false forces the plain-load form (used by tests to check both forms).
cudaError_t launch_step(const StepArgs &a, int order, bool exact, cudaStream_t s, bool allow_tma = true);

}  // namespace rtmb
