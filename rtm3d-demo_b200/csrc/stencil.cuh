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
#include <cmath>
#include <cstdint>
#include <cuda_runtime.h>

namespace rtmb {

constexpr int kTZ = 64;      // tile extent along z (contiguous), floats
constexpr int kTY = 16;      // tile extent along y
constexpr int kVZ = 4;       // z-points per thread
constexpr int kThreads = (kTZ / kVZ) * kTY;  // 256
constexpr int kMaxOrder = 16;

// kTaperAllStored / kTaperUpperStored: kTaperAll / kTaperUpper with the fields stored tapered
// (StepArgs::tw), kernel forms only.
enum TaperMode : int { kTaperNone = 0, kTaperUpper = 1, kTaperAll = 2, kTaperAllStored = 3, kTaperUpperStored = 4 };
// StepArgs::tw bits.  kTwStored: P and PP hold T(u) (the taper of the raw level u) instead of u,
// the launch applies T once more to PP and stores T(u_new); kTwRawOut: with kTwStored, store u_new
// raw (a driver's last levels); kTwPPOnce: without kTwStored (P raw, tapered on load), PP holds
// T(u) and takes T once.  The same products of the same factors in the same order as the taper
// on load, so the results are bit-identical.
enum TwBits : int { kTwStored = 1, kTwRawOut = 2, kTwPPOnce = 4 };
// How P, PP and ps are stored in HBM.  The 16-bit forms hold value * 2^-e in the 16-bit type, with
// one power-of-two exponent e per stored time level (ScaleRec); all arithmetic stays FP32.
enum StoreType : int { kStoreF32 = 0, kStoreF16 = 1, kStoreBF16 = 2 };

// Scale record of one stored time level of a 16-bit wavefield.  e: the level's exponent, written by
// the launch that produces the level; amax: bits of max |value| over the level (a non-negative float,
// so its bits order like the values), accumulated by that launch with atomicMax; zero beforehand.
struct ScaleRec {
    int e;
    unsigned amax;
};
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
    // TwBits (taper launches of the TMA kernel only; 0 elsewhere).  Taper-all: the quirk cells of
    // a stored level are written by the CTA of plane blen.
    int tw;
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
    // storage form.  store != kStoreF32: P, PP and ps point at 16-bit values (StoreType), with the
    // scale records below; img64: img points at doubles.
    int store;
    int img64;
    const ScaleRec *sc_p, *sc_pp, *sc_ps;
    ScaleRec *sc_out;           // record of the level this launch writes into PP
    float inj;                  // bound on |values| written by injection (source, receivers, border)
    const float *inj_dev;       // optional device scalar added to inj
    int iso;                    // cx == cy == cz, symmetric: the FMA form may use the packed symmetric sum
    // 2D models (nx == 1, the reference's rtmStep2D): computed planes restricted to [x_lo, x_hi)
    // when x_hi > 0, with the x coefficients zero (so lap = acmy + acmz exactly)
    int x_lo, x_hi;
    // increment storage (16-bit forms only): P holds p(t), PP the increment d(t) = p(t) - p(t-1),
    // updated in place to d(t+1); p(t+1) goes to Pout.  sc_pp is d(t)'s record, sc_out p(t+1)'s,
    // sc_out2 d(t+1)'s.
    int diff;
    void *Pout;
    ScaleRec *sc_out2;
    // launch variant of the TMA step kernel (tile shape and ring depths, 0 = default): taken by the
    // FP32 forms without taper at order 8, ignored elsewhere
    int variant;
    // image pairing of the merged dual step (receiver arguments): 0 the image is read and written
    // (img += S_new R_new); 1 this step's product is left to the next launch (no image traffic);
    // 2 the previous step's product, S R of this step's input levels, is added first:
    // img = (img + S R) + S_new R_new, the same FP32 sequence as two steps of mode 0
    int img_pair;
};

// In-plane tile (z, y) of a launch variant of the TMA step kernel (stencil_tma_impl.cuh: Variant).
void variant_tile(int variant, int *tz, int *ty);
constexpr int kStepVariants = 4;
// launch variants of the dual backward step (in-plane tile and ring depths, StepArgs::variant)
constexpr int kDualVariants = 8;
// Shots per launch of the batched step kernel (their arguments travel as kernel parameters).
constexpr int kMaxBatchShots = 24;

// Exponent of a produced level: the smallest e with bound * 2^-e < 2^15.  bound is
// 8 * max(amax(P), amax(PP)) + injection: a stable step (v^2 dt^2 * sum|coef| <= 4 over the three
// axes) keeps |2p - pp + v^2 dt^2 lap p| <= 7 max(amax(P), amax(PP)), so a 16-bit level never
// overflows (FP16 max 65504 > 2^15) and keeps at least 12 bits of headroom below it.
__host__ __device__ inline int storage_exponent(float bound) {
    if (!(bound > 0.f)) return 0;
    int k = 0;
    (void)frexpf(bound, &k);  // bound = m 2^k, 0.5 <= m < 1
    int e = k - 15;
    return e < -100 ? -100 : (e > 100 ? 100 : e);
}

// Launch one step.  Selects the instantiation for order/2 and the alignment of the arrays.
// allow_tma = false forces the plain-load form (used by tests to check both forms).
cudaError_t launch_step(const StepArgs &a, int order, bool exact, cudaStream_t s, bool allow_tma = true);

// One launch of the step kernel over several volumes (the batched multi-shot drivers): order 8, no
// taper, TMA-aligned volumes, the same form and the same stencil coefficients for every shot
// (args[0]'s are used).  At most kMaxBatchShots shots.
cudaError_t launch_step_batch(const StepArgs *args, int nshots, int order, bool exact, cudaStream_t s);

// The dual-wavefield backward step of RBC migration: src advances the reconstructed source
// wavefield, rcv the receiver wavefield with its receiver injection and the image of the new source
// values (rcv.ps is not read); neither is tapered.  One launch instead of two; FP32, order 8,
// TMA-aligned volumes, rcv.chunk x planes per CTA (64 x 8 tiles).
bool dual_step_supported(const StepArgs &src, const StepArgs &rcv, int order);
cudaError_t launch_dual_step(const StepArgs &src, const StepArgs &rcv, int order, bool exact, cudaStream_t s);

// Whether the 16-bit storage forms (and the FP64 image) can run on this geometry: order 8 and
// z rows whose 16-bit pitch is a multiple of 16 bytes (nze % 8 == 0).
bool storage_form_supported(int order, int nze);

}  // namespace rtmb
