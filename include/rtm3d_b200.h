/*
 * rtm3d_b200.h -- C ABI of librtm3d_b200.so, the B200 (sm_100a) time-stepping library for
 * 3D acoustic seismic modeling and reverse-time migration.
 *
 * The library replaces the GPU back-end of sc4ii-cimatec/rtm3d-demo (paths below are relative
 * to its source/rtm-3d/ directory):
 *   - the per-step operators of the platform interface RTMPlatform (include/RTMPlatform.hpp:28-102)
 *     and their CUDA wrappers (kernel/gpu/rtmgpu.hpp:8-65), and
 *   - the per-shot time loops of the kernel classes: RTMFiniteDifferencesKernel::rtmModel
 *     (src/kernel/RTMFiniteDifferencesKernel.cpp:103-246), RTMHBCKernel::rtmMigrate
 *     (src/kernel/RTMFiniteDifferencesKernel_HBC.cpp:64-364) and RTMRBCKernel::rtmMigrate
 *     (src/kernel/RTMFiniteDifferencesKernel_RBC.cpp:36-274).
 *
 * Conventions
 *   - Volumes are FP32, padded by blen cells on every face: (nx+2*blen, ny+2*blen, nz+2*blen),
 *     x slowest, z fastest, offset = (x*nye + y)*nze + z (include/RTMGrid.hpp:217-221).
 *   - Source and receiver coordinates are in the UNPADDED model, as in input.json.
 *   - A shot record is held in the reference's file layout: nt/ntstep chunks, each chunk
 *     [receiver_count_x][receiver_count_y][ntstep] with time fastest -- exactly the
 *     concatenation of the .seism files (include/RTMBase.hpp:131-138).
 *   - Per-operator entry points take caller-owned DEVICE pointers (the reference's
 *     GPUDeviceGrid ownership, src/grid/RTMGPUDeviceGrid.cpp:14-57) and are asynchronous on the
 *     context's stream; they never synchronise the device (the reference syncs after every
 *     launch, src/platform/gpu/RTMGPUPlatform.cpp:193-194).  *_host driver entry points take
 *     host pointers and return after the result is in host memory.
 *   - Every function returns an rtmb_status.  Nothing calls exit() or abort() (the reference's
 *     CUDACHECK exits, include/RTMGPU.hpp:18-33); rtmb_last_error() describes the last failure.
 *   - A context is bound to one device and is not thread-safe; separate contexts are.
 */
#ifndef RTM3D_B200_H
#define RTM3D_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RTMB_ABI_VERSION 2  /* 2: frequency-domain migration, two more profile categories */

typedef enum rtmb_status {
    RTMB_OK = 0,
    RTMB_EINVAL = 1,   /* bad argument or parameter combination */
    RTMB_ENOMEM = 2,   /* device or host allocation failed */
    RTMB_ECUDA = 3,    /* a CUDA runtime call failed */
    RTMB_ENAN = 4,     /* a NaN appeared in a wavefield ("Numerical Dispersion" in the reference) */
    RTMB_ETIMEOUT = 5, /* a bounded device-side wait ran out */
    RTMB_EIO = 6       /* a file could not be read or written */
} rtmb_status;

/* Boundary handling of a migration (getRTMBoundaryCondition, include/RTMGrid.hpp:27-57). */
typedef enum rtmb_boundary {
    RTMB_BC_ABC = 1,
    RTMB_BC_HBC = 2,
    RTMB_BC_RBC = 3,
    RTMB_BC_LEARNED = 4 /* modeling with the learned 8-cell closure (rtmb_closure_*); no reference value */
} rtmb_boundary;

/* Flags for rtmb_params.flags. */
#define RTMB_FLAG_FAST_FMA      0x1u  /* contract stencil arithmetic into FMA; not bit-exact with the
                                         reference CPU path (rel-L2 ~1e-7/step) */
#define RTMB_FLAG_RCV_ADD       0x2u  /* backward receiver injection ADDS (reference GPU kernel,
                                         kernel/gpu/rtmgpu_finitediff.cu:403) instead of overwriting
                                         (reference CPU path, RTMCPUPlatform.cpp:127) */
#define RTMB_FLAG_IMG_FULL_Z    0x4u  /* imaging covers every z (reference GPU kernel, .cu:440-458)
                                         instead of z in [blen, nze-blen) (CPU, RTMCPUPlatform.cpp:532) */
#define RTMB_FLAG_NO_TAPER_QUIRK 0x8u /* taper the front-right x-y edge from its own cells instead of
                                         from x = blen (RTMCPUPlatform.cpp:901) */
#define RTMB_FLAG_USE_GRAPH     0x10u /* per-shot drivers: capture the shot's launches in a CUDA
                                         graph on the context's stream and replay it with one launch;
                                         the executable graph is updated in place for the next shot.
                                         Not on the legacy or per-thread default streams, nor while
                                         rtmb_profile is on (launches then run one by one). */
#define RTMB_FLAG_NO_TMA        0x20u /* use the plain-load step kernel even when rows are 16-byte
                                         aligned (the TMA-pipelined kernel is the default then) */
/* Storage forms of the per-shot drivers (no reference counterpart; the reference stores FP32).
 * The wavefields the drivers own (source and receiver pairs) are stored as FP16 or BF16 holding
 * value * 2^-e, with one power-of-two exponent per stored time level chosen from the previous
 * levels' max |value| so that no level overflows; all stencil arithmetic stays FP32.  The record,
 * v2dt2 and the caller's image stay FP32.  Needs stencil_order 8 and nz + 2*blen a multiple of 8,
 * boundary RBC for migration (modeling tapers every face as usual); the per-operator entry
 * points ignore these flags. */
#define RTMB_FLAG_STORE_F16     0x40u
#define RTMB_FLAG_STORE_BF16    0x80u
/* With a storage flag: accumulate the image over the time steps in FP64 (the caller's FP32 image
 * is written from it at the end of the shot). */
#define RTMB_FLAG_IMG_F64       0x100u
/* FP32 RBC migration in the FMA form runs the backward source and receiver steps of each time step
 * as ONE launch (both wavefields and the image in one pass over the grid: 36 instead of 44 bytes per
 * point) when stencil_order is 8 and rows are 16-byte aligned; same results as two launches (no
 * reference counterpart: the reference runs them as separate operators).  This flag keeps the two
 * launches.  HBC migration (whose receiver steps taper the upper border) keeps two launches: there
 * one launch lost. */
#define RTMB_FLAG_NO_DUAL       0x200u
/* Modeling (every face tapered) and HBC migration (the upper border tapered) keep the wavefields
 * tapered in HBM between time steps: each step stores T(u) of its new level instead of u, so the
 * next step reads its input without a taper pass (T: the reference's taper3D / taperUpper3D,
 * RTMCPUPlatform.cpp:566-920; the same products of per-axis factors in the same order, so records
 * and images are bit-identical).  Taken when the TMA step kernel runs (stencil_order <= 8, rows
 * 16-byte aligned, no RTMB_FLAG_NO_TMA); this flag keeps the raw fields and tapers on load (no
 * reference counterpart). */
#define RTMB_FLAG_NO_TAPER_STORE 0x400u
/* With a 16-bit storage flag: store each wavefield as its current level p(t) and its increment
 * d(t) = p(t) - p(t-1) instead of the two levels p(t) and p(t-1), and step as
 * d(t+1) = d(t) + v2dt2 lap p(t), p(t+1) = p(t) + d(t+1): algebraically the same leapfrog.
 * In the two-level form 2p - p(t-1) cancels most of its digits, so the rounding of the stored
 * p(t-1) lands in full on the small difference that carries the wave's time derivative; stored as
 * its own 16-bit value with its own exponent, the increment keeps its relative precision.  Each
 * level and each increment has its own power-of-two exponent.  12 bytes per point and step instead
 * of 10 (both levels' increments are written), against 16 for FP32.  RBC migration only (no taper
 * in the steps); no reference counterpart. */
#define RTMB_FLAG_STORE_DIFF    0x800u

/* The input.json parameters on the path (include/RTMParam.hpp:188-249). */
typedef struct rtmb_params {
    uint32_t nx, ny, nz;          /* unpadded model size */
    uint32_t blen;                /* border cells on every face */
    uint32_t nt, ntstep;          /* time steps; record chunk length (nt % ntstep == 0) */
    uint32_t stencil_order;       /* even, 2..16 */
    float dx, dy, dz, dt;
    float fpeak;                  /* Ricker peak frequency */
    float taper_factor;
    uint32_t receiver_start_x, receiver_start_y, receiver_depth_z;
    uint32_t receiver_distance_x, receiver_distance_y;
    uint32_t receiver_count_x, receiver_count_y;
    int32_t boundary;             /* rtmb_boundary, used by the migration drivers */
    uint32_t flags;               /* RTMB_FLAG_* */
    int32_t device;               /* CUDA device ordinal; -1 = current device */
} rtmb_params;

typedef struct rtmb_ctx rtmb_ctx;

/* ------------------------------------------------------------------ context */
/* Replaces RTMGPUPlatform::initRTMPlatform (src/platform/gpu/RTMGPUPlatform.cpp:22-57) without its
 * cudaDeviceReset; allocates the stencil, taper and Ricker tables on the device. */
int rtmb_create(const rtmb_params *params, rtmb_ctx **out);
/* Replaces RTMGPUPlatform::destroyRTMPlatform (:16-21); frees every context-owned buffer. */
int rtmb_destroy(rtmb_ctx *ctx);
/* Description of the last failure of this context; with NULL, of the calling thread's last failed
 * call that takes no context (rtmb_model_shot_noalloc). */
const char *rtmb_last_error(const rtmb_ctx *ctx);
/* Run subsequent work on this cudaStream_t (NULL = the context's own stream). */
int rtmb_set_stream(rtmb_ctx *ctx, void *cuda_stream);
int rtmb_sync(rtmb_ctx *ctx);
int rtmb_abi_version(void);
/* Count of this library's kernel launches since the context was created. */
uint64_t rtmb_launch_count(const rtmb_ctx *ctx);
/* Per-kernel timing of the per-shot drivers (no counterpart in the reference, whose report keeps
 * millisecond wall times per phase, src/kernel/RTMKernel.cpp:11-80).  When enabled, every driver
 * launch is bracketed by CUDA events on the context's stream; the durations are summed per category
 * at the end of each driver call.  Enabling clears the totals. */
#define RTMB_PROF_CATEGORIES 8
#define RTMB_PROF_MODEL 0             /* modeling step (taper, source, receivers fused) */
#define RTMB_PROF_FORWARD 1           /* migration forward step */
#define RTMB_PROF_BACKWARD_SOURCE 2   /* backward source-wavefield reconstruction step */
#define RTMB_PROF_BACKWARD_RECEIVER 3 /* backward receiver step with receiver injection and imaging */
#define RTMB_PROF_OTHER 4
#define RTMB_PROF_BACKWARD_DUAL 5     /* source and receiver steps with imaging in one launch */
#define RTMB_PROF_FMIG_STEP 6         /* frequency-domain migration: wavefield steps */
#define RTMB_PROF_FMIG_FREQ 7         /* frequency-domain migration: DFT and image update */
int rtmb_profile(rtmb_ctx *ctx, int enable);
/* ms[RTMB_PROF_CATEGORIES]: summed kernel time; launches[RTMB_PROF_CATEGORIES]: launch counts. */
int rtmb_profile_read(const rtmb_ctx *ctx, double *ms, uint64_t *launches);

/* ------------------------------------------------------------------ host-side tables
 * Bit-identical to the reference's host computations; usable without a GPU. */
/* RTMStencil::setStencilCoefficients (include/RTMGrid.hpp:433-446) with laplacian_coefs / makeo2
 * (src/misc/Misc.cpp:106-176).  out: [3][order+1] for x, y, z. */
int rtmb_stencil_coefs(uint32_t order, float dx, float dy, float dz, float *out);
/* RTMTaperFunction::inittaper (include/RTMSeismic.hpp:294-305).  out: blen floats. */
int rtmb_taper_vector(uint32_t blen, float taper_factor, float *out);
/* RTMSeismicSource::loadSamples / ricker (include/RTMSeismic.hpp:135-144, 191-198). */
int rtmb_ricker(uint32_t nt, float dt, float fpeak, float *out);
/* RTMCube::extendBorders + initBorders (src/grid/RTMGrid.cpp:47-86, 371-714) on the host.
 * bc: 0 none (border left zero), RTMB_BC_ABC, RTMB_BC_HBC, RTMB_BC_RBC.  The random border uses
 * libc rand() in the reference's single-thread order after srand(seed); seed < 0 skips srand. */
int rtmb_prepare_velocity(const float *v, uint32_t nx, uint32_t ny, uint32_t nz, uint32_t blen,
                          int32_t bc, int64_t seed, float *ve);
/* Grid::power2 then multiplyBy(dt*dt) (src/controller/RTMController.cpp:110-111), in place. */
int rtmb_v2dt2_host(float *ve, size_t n, float dt);

/* ------------------------------------------------------------------ per-step operators
 * Device pointers, padded volumes sized by the context's parameters. */
/* RTMPlatform::rtmStep (include/RTMPlatform.hpp:50-51), RTMSTEP_WRAPPER (kernel/gpu/rtmgpu.hpp:8-11):
 * PP <- 2P - PP + v2dt2 * lap(P) on [h, n-h)^3, h = order/2; PP updated in place. */
int rtmb_step(rtmb_ctx *ctx, const float *P, float *PP, const float *v2dt2);
/* RTMPlatform::rtmStepMultipleWave (RTMCPUPlatform.cpp:397-472): rtmb_step on two wavefields
 * with the same v2dt2. */
int rtmb_step_multiwave(rtmb_ctx *ctx, const float *P0, float *PP0, const float *P1, float *PP1, const float *v2dt2);
/* RTMPlatform::rtmUpdateFreqContributions (RTMCPUPlatform.cpp:20-64): for frequency iw at time step
 * it, slot lw of the frequency grids += kre/kim[iw][it] * PS / PR over the model interior.
 * sre, sim, rre, rim: [nwstep][nx][ny][nz] (RTMGridCollection); kre, kim: [nw][nt] (RTMPlane);
 * PS, PR: padded wavefields.  All device pointers. */
int rtmb_fmig_update_freq(rtmb_ctx *ctx, uint32_t it, uint32_t iw, uint32_t lw, const float *PS, const float *PR,
                          float *sre, float *sim, float *rre, float *rim, const float *kre, const float *kim);
/* RTMPlatform::rtmFreqDomainImageCondition (RTMCPUPlatform.cpp:66-102): img += w2[iw] (sRe rRe -
 * sIm rIm) over the model interior from slot lw; w2: the squared frequencies [nw] (device). */
int rtmb_fmig_image_condition(rtmb_ctx *ctx, uint32_t iw, uint32_t lw, const float *w2, float *img, const float *sre,
                              const float *sim, const float *rre, const float *rim);
/* RTMPlatform::rtmTaperAllBorders / rtmTaperUpperBorders (RTMPlatform.hpp:35-42),
 * RTMTAPER_WRAPPER (rtmgpu.hpp:27-30); CPU taper semantics (RTMCPUPlatform.cpp:566-920). */
int rtmb_taper_all_borders(rtmb_ctx *ctx, float *P);
int rtmb_taper_upper_borders(rtmb_ctx *ctx, float *P);
/* RTMPlatform::rtmApplySource (RTMPlatform.hpp:70), RTMSOURCE_WRAPPER (rtmgpu.hpp:21-25):
 * PP[sx+b, sy+b, sz+b] += wavelet[it] (the context's Ricker table). */
int rtmb_apply_source(rtmb_ctx *ctx, float *PP, uint32_t sx, uint32_t sy, uint32_t sz, uint32_t it);
/* RTMPlatform::rtmSaveReceiverData / rtmRestoreReceiverData (RTMPlatform.hpp:75-80),
 * RTMSEISM_WRAPPER (rtmgpu.hpp:13-19).  rec: one chunk [rcx][rcy][ntstep]; lt < ntstep. */
int rtmb_save_receiver_data(rtmb_ctx *ctx, const float *PP, float *rec, uint32_t lt);
int rtmb_restore_receiver_data(rtmb_ctx *ctx, float *PP, const float *rec, uint32_t lt);
/* RTMPlatform::rtmSaveUpperBorder / rtmRestoreUpperBorder (RTMPlatform.hpp:85-90),
 * RTMWUPB_WRAPPER (rtmgpu.hpp:32-33).  upb: [ntstep][nxe][nye][order/2], 64-bit offsets. */
int rtmb_save_upper_border(rtmb_ctx *ctx, const float *P, float *upb, uint32_t lt);
int rtmb_restore_upper_border(rtmb_ctx *ctx, float *P, const float *upb, uint32_t lt);
/* RTMPlatform::rtmImageCondition (RTMPlatform.hpp:65), RTMIMG_WRAPPER (rtmgpu.hpp:35-37):
 * IMG += PS * PR. */
int rtmb_image_condition(rtmb_ctx *ctx, float *img, const float *ps, const float *pr);
/* Image finalisation of the controller (src/controller/RTMAcousticController.cpp:244-249):
 * order-2 Laplacian filter (src/grid/RTMGrid.cpp:226-300) then removeBorders (:129-166).
 * img: padded device volume; out: nx*ny*nz device volume. */
int rtmb_image_finalize(rtmb_ctx *ctx, const float *img, float *out);
/* RTMCube::stack / stackRegion over the whole cube (src/grid/RTMGrid.cpp:168-223): acc += img. */
int rtmb_image_stack(rtmb_ctx *ctx, float *acc, const float *img);

/* ------------------------------------------------------------------ per-shot drivers
 * The extended squared-slowness-times-dt^2 volume (v2dt2, padded) must be loaded first.
 * (sx, sy, sz) is the shot position in the unpadded model (RTMController.cpp:145-147). */
int rtmb_load_v2dt2(rtmb_ctx *ctx, const float *v2dt2, int from_host);
/* RTMFiniteDifferencesKernel::rtmModel: taper every face, step, inject, sample receivers.
 * rec: record in file layout (nt*rcx*rcy floats), device pointer. */
int rtmb_model_shot(rtmb_ctx *ctx, uint32_t sx, uint32_t sy, uint32_t sz, float *rec);
/* RTMHBCKernel::rtmMigrate / RTMRBCKernel::rtmMigrate (by params.boundary): forward pass, then the
 * backward pass rebuilding the source wavefield and cross-correlating it with the back-propagated
 * receiver wavefield.  rec: record in file layout (device); img: padded per-shot image (device),
 * overwritten (the reference's shotImage). */
int rtmb_migrate_shot(rtmb_ctx *ctx, uint32_t sx, uint32_t sy, uint32_t sz, const float *rec,
                      float *img);
/* Modeling without any device allocation.  This entry point has no counterpart in the reference.
 * It is for callers that cannot call cudaMalloc, for example a host framework whose allocator has
 * reserved the GPU's memory up front and must account for every byte, or a latency-sensitive loop
 * that cannot afford cudaMalloc's implicit device synchronisation.  It runs the same shot as
 * rtmb_model_shot, with the same kernels and results, but creates no context: the caller passes
 * v2dt2 (padded, device) and rec (device, file layout) and the stream (NULL: the legacy default
 * stream), and every other buffer lives in one 64 MiB device array inside the library that each GPU
 * loading the library holds until the process exits.  Grids up to about 8.3 million padded points
 * fit (two wavefields plus small tables); larger ones are rejected with RTMB_EINVAL, and so are
 * blen above 1024 (the taper table goes up through a stack buffer of 1024 floats), the 16-bit
 * storage flags and boundary RTMB_BC_LEARNED (both need a context), and v2dt2 or rec that are not
 * device (or managed) memory of the call's device (checked with cudaPointerGetAttributes).
 *   - The first call on a device looks up that array's address (once per device, with the device
 *     current); make that first call before any stream capture on the device.
 *   - All calls on a device share the array and it keeps the previous call's contents; the entry
 *     point clears what must start at zero.  Calls that overlap on the GPU (several host threads or
 *     streams) race on it and must be serialised by the caller.
 *   - It allocates no device memory and calls no allocating library routine.  On failure,
 *     rtmb_last_error(NULL) describes the error (per host thread). */
int rtmb_model_shot_noalloc(const rtmb_params *params, const float *v2dt2, uint32_t sx, uint32_t sy,
                            uint32_t sz, float *rec, void *cuda_stream);

/* Frequency-domain RTM of one shot (input.json "fmig": true; the reference's RTMFreqDomainKernel,
 * src/kernel/RTMFiniteDifferencesKernel_FreqDomain.cpp:220-357, with the CPU platform's operators
 * RTMCPUPlatform.cpp:20-102 and :397-472).  Both wavefields step forward in time together, the
 * source one from the Ricker wavelet and the receiver one from the record read backwards, every
 * field tapered on all faces after each step; for each of the nw frequencies
 * w = 2 pi (fmin + iw df) dt, df = 1 / (nt dt), nw = (fmax - fmin) / df (fmig_min_freq,
 * fmig_max_freq), a running DFT of both fields over the model interior feeds the image
 * img += w^2 (Re S Re R - Im S Im R) at every time step.
 *   rec:    device record in the file layout (as rtmb_migrate_shot);
 *   nwstep: frequencies per pass over time (fmig_nwstep; 0 = all nw in one pass, the reference CPU
 *           build's choice and its order of the image sums, so the exact form is bit-exact with it).
 *           The pass holds 4 nwstep nx ny nz floats of frequency grids; smaller groups cost a time
 *           loop each.  At most 256.
 *   img:    padded FP32 image, overwritten with this shot's image.  (The reference never clears
 *           its image between fmig shots, so its shot images accumulate; this call does not.)
 * RTMB_FLAG_FAST_FMA selects the FMA arithmetic for the steps and the DFT.  FP32 storage only. */
int rtmb_migrate_shot_fmig(rtmb_ctx *ctx, uint32_t sx, uint32_t sy, uint32_t sz, const float *rec, float fmin,
                           float fmax, uint32_t nwstep, float *img);
/* nw of a frequency-domain migration (..._FreqDomain.cpp:133-137); 0 when there is none. */
int rtmb_fmig_nw(float dt, uint32_t nt, float fmin, float fmax);
/* Its tables, host arrays (..._FreqDomain.cpp:17-51, :151-152): w2[nw] = w^2 and kre/kim[nw][nt]
 * = cos/sin(w it), w = 2 pi (fmin + iw df) dt; the inputs of rtmb_fmig_update_freq and
 * rtmb_fmig_image_condition once copied to the device. */
int rtmb_fmig_tables(float dt, uint32_t nt, float fmin, float fmax, float *w2, float *kre, float *kim);

/* rtmb_migrate_shot that ADDS the shot's image to a caller-owned FP64 stack (padded, device)
 * instead of writing an FP32 image: the shot stacking of RTMAcousticController.cpp:223-242 with an
 * FP64 accumulator.  With a storage flag the time accumulation runs in FP64 directly into the
 * stack; with FP32 storage the FP32 shot image is added to it.  No reference counterpart. */
int rtmb_migrate_shot_acc64(rtmb_ctx *ctx, uint32_t sx, uint32_t sy, uint32_t sz, const float *rec,
                            double *stack);

/* FP64 GPU oracle (no reference counterpart): the reference's operator sequence of
 * RTMFiniteDifferencesKernel::rtmModel and RTMHBCKernel/RTMRBCKernel::rtmMigrate, one launch per
 * operator, in double precision on the same discrete scheme (the FP32 stencil coefficients, taper
 * factors, Ricker samples and v2dt2, widened).  It is the yardstick for the error of the FP32 and
 * 16-bit forms, not a fast path.  rec (model): double record in file layout; img (migrate): padded
 * double image, overwritten; both device pointers.  Ignores the storage and FMA flags. */
int rtmb_model_shot_f64(rtmb_ctx *ctx, uint32_t sx, uint32_t sy, uint32_t sz, double *rec);
int rtmb_migrate_shot_f64(rtmb_ctx *ctx, uint32_t sx, uint32_t sy, uint32_t sz, const float *rec,
                          double *img);

/* ------------------------------------------------------------------ learned boundary closure
 * No reference counterpart (the reference absorbs with the taper of taper3D, RTMCPUPlatform.cpp:710-920).
 * A per-cell MLP (55 -> 32 -> 32 -> 1, tanh; BF16 tensor-core GEMMs with FP32 accumulation) closes
 * an 8-cell strip on every face, so modeling runs on nx+16 x ny+16 x nz+16 instead of nx+2*blen ...:
 * the network advances the strip's outer 4 cells, the stencil the inner 4.  Inputs per strip cell: the 3x3x3 neighbourhood of p(t) and p(t-1) in the frame of
 * its nearest face (inward normal first), divided by their max |value| s, and the Courant number
 * sqrt(v2dt2)/dx; 64 BF16 features per row (the last 9 zero).  Output r: the correction to the
 * first-order one-way (upwind) update of an outgoing wave, p(t+1) = p + C (p_in - p) + s*clamp(r, +-0.5),
 * p_in the inward neighbour, C the Courant number.
 * params: RTMB_CLOSURE_NPARAM floats, W1[32][64], b1[32], W2[32][32], b2[32], w3[32], b3.
 * Device pointers unless stated; on failure of the context-free calls rtmb_last_error(NULL) describes
 * the error. */
#define RTMB_CLOSURE_NPARAM 3169
#define RTMB_CLOSURE_NIN 64
int rtmb_closure_param_count(void);
/* Seeded Glorot-uniform initialisation of host params (biases zero). */
int rtmb_closure_init(float *params_host, uint64_t seed);
/* y[i] = network(X[i]) for n rows of BF16 features (X: n*64 bf16). */
int rtmb_closure_forward(const float *params, const void *X, uint64_t n, float *y, void *cuda_stream);
/* Gradient of loss = mean_i (network(X[i]) - R[i])^2 with respect to params, and the loss. */
int rtmb_closure_grad(const float *params, const void *X, const float *R, uint32_t n, float *grad, float *loss,
                      void *cuda_stream);
/* Adam training: steps mini-batches of batch rows drawn at random (seeded) from (X, R); params is
 * updated in place; loss_host (optional, host) receives each step's batch loss.  noise: standard
 * deviation of Gaussian noise added to the 54 normalised wavefield features of each drawn row. */
int rtmb_closure_train(float *params, const void *X, const float *R, uint64_t n, uint32_t steps, uint32_t batch,
                       float lr, float noise, uint64_t seed, float *loss_host, void *cuda_stream);
/* Training pairs from a modeling shot of the plain method on a wide context (blen >= 16, loaded
 * v2dt2): the strip of the 8-cell domain nx+16 x ny+16 x nz+16 centred in it, sampled at
 * per_step random strip cells on steps t0, t0+tstride, ... (cells whose neighbourhood max |p| is
 * below min_scale are skipped); X (capacity*64 bf16) and R (capacity floats) receive the rows,
 * *count (host) how many were written. */
int rtmb_closure_collect(rtmb_ctx *wide, uint32_t sx, uint32_t sy, uint32_t sz, uint32_t t0, uint32_t tstride,
                         uint32_t per_step, uint64_t seed, float min_scale, void *X, float *R, uint64_t capacity,
                         uint64_t *count);
/* Installs params (device or host) in a context with boundary RTMB_BC_LEARNED and blen 8; its
 * rtmb_model_shot then advances the strip with the network (the stencil runs inside it).  Strip
 * cells whose neighbourhood max |p| is below min_scale stay zero (the stencil's numerical tail ahead
 * of the wavefront, where the network is not trained); the others are multiplied by
 * 1 - damp * ((4 - depth) / 4)^2 each step, depth 0 at the outer face (0 <= damp < 1). */
int rtmb_closure_set(rtmb_ctx *ctx, const float *params, float min_scale, float damp);
/* The closure's judge and fallback.  Runs the same modeling shot on three contexts of the same
 * model, receivers, nt and device -- `learned` (RTMB_BC_LEARNED with its closure installed), `hbc`
 * (the plain taper border, 32 cells by design) and `wide` (a border so wide that no reflection
 * returns within nt) -- and measures each bordered run's reflected energy as the record rel-L2
 * against the wide run's record (on device, double accumulation).  The learned context passes when
 * it reflects no more than the taper border; otherwise it is marked fallen back.  Outputs: both
 * reflections. */
int rtmb_closure_judge(rtmb_ctx *learned, rtmb_ctx *hbc, rtmb_ctx *wide, uint32_t sx, uint32_t sy, uint32_t sz,
                       float *refl_learned, float *refl_hbc);
/* Modeling with the judged boundary: the learned context's shot when its closure passed its judge,
 * else the fallback (taper-border) context's shot; *ran (optional) receives RTMB_BC_LEARNED or the
 * fallback's boundary.  The learned context must have been judged. */
int rtmb_model_shot_judged(rtmb_ctx *learned, rtmb_ctx *fallback, uint32_t sx, uint32_t sy, uint32_t sz, float *rec,
                           int *ran);

/* ------------------------------------------------------------------ batched multi-shot migration
 * No reference counterpart (the reference migrates one shot per process, RTMAcousticController.cpp:
 * 193-242).  Any number of shots, each on its own aperture sub-volume of the survey (sizes may
 * differ), run in groups of batch_group shots (default 12, at most 24; rtmb_set_batch_group,
 * rtmb_autotune_batch): the shots of a group advance together, every time step of the group is one
 * launch of the step kernel over all its shots' volumes, and with RTMB_FLAG_USE_GRAPH the group's
 * whole time loop is one CUDA graph.  A group's wavefields and shot images are allocated for the
 * group and freed after it.  Each shot's image
 * is added, without its border, to the survey's FP64 stack at the aperture's origin.  The context
 * supplies what the shots share: blen, nt, ntstep, stencil_order (8), dx/dy/dz, dt, fpeak,
 * boundary (RBC) and the form flags (FP32 exact or FMA, or a 16-bit storage flag with or without
 * RTMB_FLAG_IMG_F64).  Shot volumes need nz + 2*blen a multiple of 4 (FP32) or 8 (16-bit). */
typedef struct rtmb_shot {
    uint32_t nx, ny, nz;          /* aperture (unpadded) size */
    uint32_t ox, oy, oz;          /* aperture origin in the survey model */
    uint32_t sx, sy, sz;          /* source, aperture coordinates */
    uint32_t receiver_start_x, receiver_start_y, receiver_depth_z;
    uint32_t receiver_distance_x, receiver_distance_y;
    uint32_t receiver_count_x, receiver_count_y;
    const float *v2dt2;           /* padded aperture v2dt2 (device) */
    const float *rec;             /* the shot's record, file layout (device) */
} rtmb_shot;
/* stack: survey image (snx * sny * snz doubles, device), added to. */
int rtmb_migrate_batch(rtmb_ctx *ctx, uint32_t nshots, const rtmb_shot *shots, double *stack, uint32_t snx,
                       uint32_t sny, uint32_t snz);
/* Shots per launch of rtmb_migrate_batch (1 .. 24). */
int rtmb_set_batch_group(rtmb_ctx *ctx, uint32_t shots_per_launch);
/* Times the batched forward step (2 warm-up and 5 timed launches, CUDA events) for 1, 2, 3, 4, 6, 8,
 * 12, 16 and 24 shots per launch on the first shots of the batch and keeps the group size with the
 * highest point-update rate for the context's later batches.  Optional outputs: the group size and
 * its rate (G point-updates/s). */
int rtmb_autotune_batch(rtmb_ctx *ctx, uint32_t nshots, const rtmb_shot *shots, uint32_t *group_out,
                        float *rate_out);

/* ------------------------------------------------------------------ autotuner (no reference counterpart)
 * The reference launches a fixed 10^3-thread block grid (RTMGPUPlatform.cpp:167-196); here the
 * launch shape of the step kernels is measured on the context's own geometry, form and v2dt2.
 *
 * rtmb_autotune_full times, with CUDA events on the context's stream (2 warm-up and 5 timed
 * launches per candidate):
 *   - the single-wavefield step (forward form plus imaging form) for every launch variant -- the
 *     in-plane tile (0: 64 z x 16 y, 1: 32 x 32, 2: 64 x 8 at three CTAs per SM, 3: 64 x 16 with
 *     shallower load rings) -- and every x-chunk length (x planes per CTA, 8 .. 256).  Variants 1-3
 *     exist for the FP32 forms without taper at stencil order 8; other forms tune the chunk only;
 *   - where the dual-wavefield backward step applies (FP32 RBC migration, order 8): its launch
 *     variant (0: 64 x 8 tiles, 1: 32 x 16, 2: 32 x 16 with two more P-ring slots and a fourth
 *     exchange slot, 3: 32 x 16 with one more P-ring slot, a fourth core slot and a fourth exchange
 *     slot; 4 to 7: 64 x 8, 32 x 16, 64 x 16 and 32 x 32 with every thread stepping both
 *     wavefields) and x-chunk, and the dual step against the source and receiver steps as two
 *     launches.
 * The fastest choices are kept for every later launch of the context (rtmb_tuning; results do not
 * change: every variant computes the same arithmetic per point).  The measurement runs the step
 * forms without taper (those of RBC migration); the chunk it picks serves every form of the
 * context.  rtmb_autotune is the same call reporting only the chunk and the step time. */
typedef struct rtmb_tuning {
    uint32_t variant;     /* launch variant of the single-wavefield step (see above) */
    uint32_t chunk;       /* x planes per CTA of that step */
    uint32_t dual;        /* 1: dual-wavefield backward step, 0: two launches per backward time step */
    uint32_t dual_chunk;  /* x planes per CTA of the dual step */
    float ms_step;        /* forward step (ms) with the chosen variant and chunk */
    float ms_backward;    /* one backward time step (ms): the dual launch, or source + receiver steps */
    uint32_t dual_variant;  /* launch variant of the dual step (0 .. 7, see above) */
} rtmb_tuning;
int rtmb_autotune_full(rtmb_ctx *ctx, rtmb_tuning *out);
/* Applies a tuning (for example one measured earlier on the same geometry). */
int rtmb_set_tuning(rtmb_ctx *ctx, const rtmb_tuning *t);
int rtmb_autotune(rtmb_ctx *ctx, uint32_t *chunk_out, float *ms_out);
/* Sets the x-chunk length directly (the default is chosen from the grid at rtmb_create). */
int rtmb_set_chunk(rtmb_ctx *ctx, uint32_t chunk);

/* Host-buffer forms: copy in, run, copy out, return when the result is on the host. */
int rtmb_model_shot_host(rtmb_ctx *ctx, uint32_t sx, uint32_t sy, uint32_t sz, float *rec_host);
int rtmb_migrate_shot_host(rtmb_ctx *ctx, uint32_t sx, uint32_t sy, uint32_t sz,
                           const float *rec_host, float *img_host);

#ifdef __cplusplus
}
#endif
#endif /* RTM3D_B200_H */
