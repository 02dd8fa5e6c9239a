// stencil_tma_impl.cuh -- the TMA-pipelined form of the fused time step (sm_100a).
//
// Same contract and arithmetic as stencil_impl.cuh (bit-identical results); used when rows are
// 16-byte aligned (nze % 4 == 0, 16-byte aligned base pointers).
//
// Pipeline.  A CTA owns a TZ x TY tile of the (y, z) plane and a chunk of x planes; eight consumer
// warps compute, and lane 0 of a ninth warp is the producer of two rings of shared-memory slots
// filled by cp.async.bulk.tensor (TMA) loads that complete on "full" mbarriers:
//   * the P ring (D slots): the P tile of one plane with a y halo of H rows and a z halo of ZH
//     columns.  A slot is needed from the plane's arrival (its centre values enter each thread's
//     register queue of x taps) until the plane is computed H planes later (y and z taps);
//   * the core ring (R slots): the PP and v2dt2 tiles (and PS and IMG for the imaging form) of the
//     plane being computed.
// The CTA has eight consumer warps and one producer warp.  Lane 0 of the producer warp issues the
// loads in order; each slot is refilled once its "empty" mbarrier shows that all eight consumer warps
// have released it, so loads run up to D-H-1 planes (P) and R-1 planes (core) ahead and no consumer
// ever waits at a block barrier (the taper-on-load forms add a consumer-only named barrier per
// tapered plane; the stored-taper forms taper on store and need none).  Each thread keeps the 2H+1
// x taps of its four points in a register queue that shifts by one plane per iteration.
//
// The rare per-cell work (source, receivers, upper border, taper side buffer) is found per plane by
// CTA-uniform tests: the kernel runs at the 96-register cap of two CTAs per SM, and per-thread
// state kept live through the plane loop costs instructions everywhere.
//
// Every wait is bounded (about two seconds): a wait that runs out sets error bit 2 and the warp
// stops; the producer waits, again bounded, for the copies it issued before it exits.
#pragma once
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "stencil_common.cuh"

// Unroll factors of the plane loops of the single-wavefield TMA step kernel and of the dual step
// kernel (compile-time tuning).  The x register queue shifts by one plane per iteration; an
// unrolled body lets the compiler rename part of it instead of moving it.  Measured on a 592^3
// shot: 3 took 4% off the exact and FP16 steps and 1.4% off the FMA forward step, but made the
// dual step spill and run 8% slower, where 2 took 2% off.
#ifndef RTMB_PLANE_UNROLL
#define RTMB_PLANE_UNROLL 3
#endif
#ifndef RTMB_DUAL_UNROLL
#define RTMB_DUAL_UNROLL 2
#endif
#define RTMB_DO_PRAGMA(x) _Pragma(#x)
#define RTMB_UNROLL_PRAGMA(n) RTMB_DO_PRAGMA(unroll n)

namespace rtmb {
namespace detail {

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait for the completion of the phase with the given parity: false after ~2^32 cycles.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
    if (mbar_try_wait(bar, parity)) return true;
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity))
        if (clock64() - t0 > (1ll << 32)) return false;
    return true;
}

// The producer's bounded wait for a free slot: the same limit as mbar_wait, with a sleep between
// polls (32 ns doubling to 512 ns).  The producer runs several planes ahead of the consumers and
// spends most of its time waiting for them; polling without a pause would take issue slots from the
// consumer warps of its SM sub-partition.
__device__ __forceinline__ bool mbar_wait_producer(uint64_t *bar, uint32_t parity) {
    if (mbar_try_wait(bar, parity)) return true;
    const long long t0 = clock64();
    unsigned ns = 32;
    while (!mbar_try_wait(bar, parity)) {
        if (clock64() - t0 > (1ll << 32)) return false;
        __nanosleep(ns);
        ns = ns < 512 ? 2 * ns : 512;
    }
    return true;
}

__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, uint64_t *bar, int c0, int c1,
                                            int c2) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
        ::"r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ float4 ld_f4(const float *p) { return *reinterpret_cast<const float4 *>(p); }

// The new level of one point in the two arithmetic forms of the FP32 step: exact (every product and
// sum rounded on its own, the reference CPU order) or one FMA.  Used by the merged dual step, which
// restates the step body for two wavefields.
template <bool EXACT>
__device__ __forceinline__ float step_update(float v, float lap, float p, float pp) {
    if (EXACT) {
        const float two_p = 2.f * p;
        const float d = two_p - pp;
        const float vl = v * lap;
        return d + vl;
    }
    return fmaf(v, lap, 2.f * p - pp);
}

// Barrier 1 over the NT consumer threads only (the producer warp never joins it).
template <int NT>
__device__ __forceinline__ void consumer_sync() { asm volatile("bar.sync 1, %0;" ::"n"(NT) : "memory"); }
template <int NT>
__device__ __forceinline__ bool consumer_sync_or(bool v) {
    uint32_t out;
    asm volatile("{\n .reg .pred p, q;\n setp.ne.u32 p, %1, 0;\n bar.red.or.pred q, 1, %2, p;\n selp.u32 %0, 1, 0, q;\n}\n"
                 : "=r"(out)
                 : "r"((uint32_t)v), "n"(NT)
                 : "memory");
    return out != 0;
}

constexpr int kTmaThreads = kThreads + 32;  // eight consumer warps and one producer warp

// Launch variants of the step kernel (StepArgs::variant, picked per context by rtmb_autotune):
// the in-plane tile (TZ along z, TY along y; four z points per consumer thread) and the depth of
// the P ring (slots beyond the centre plane: DX, DX_IMG for the imaging form) and of the core ring
// (R, R_IMG); MINB CTAs per SM.  Variant 0 is the default and the only one of the taper forms.
template <int V>
struct Variant;
template <>
struct Variant<0> {  // 64 x 16, deep rings
    static constexpr int TZ = 64, TY = 16, DX = 6, DX_IMG = 5, R = 4, R_IMG = 3, MINB = 2;
};
template <>
struct Variant<1> {  // 32 x 32: fewer halo rows per point (40 x 40 tile for 32 x 32 points)
    static constexpr int TZ = 32, TY = 32, DX = 6, DX_IMG = 5, R = 4, R_IMG = 3, MINB = 2;
};
template <>
struct Variant<2> {  // 64 x 8 with three CTAs per SM
    static constexpr int TZ = 64, TY = 8, DX = 6, DX_IMG = 5, R = 4, R_IMG = 3, MINB = 3;
};
template <>
struct Variant<3> {  // 64 x 16, shallow rings (less shared memory per CTA, shorter lookahead)
    static constexpr int TZ = 64, TY = 16, DX = 4, DX_IMG = 4, R = 3, R_IMG = 2, MINB = 2;
};
constexpr int kVariants = 4;
template <int V>
constexpr int variant_threads() { return (Variant<V>::TZ / kVZ) * Variant<V>::TY + 32; }

// Tensor maps of one launch.  p: box {TZ + 2ZH, TY + 2H, 1}; the others: box {TZ, TY, 1}.
struct TmaMaps {
    CUtensorMap p, pp, v, ps, img;
};

// Element access for the storage types.  ld4 reads four consecutive values from shared memory and
// widens them to FP32; st4 narrows four FP32 values and stores them to global memory.
template <typename T>
struct Stor;
template <>
struct Stor<float> {
    static constexpr bool kScaled = false;
    __device__ static float4 ld4(const float *p) { return *reinterpret_cast<const float4 *>(p); }
    __device__ static float to_f(float v) { return v; }
    __device__ static float from_f(float v) { return v; }
    __device__ static void st4(float *p, float4 v) { *reinterpret_cast<float4 *>(p) = v; }
    __device__ static void st1(float *p, float v) { *p = v; }
};
template <>
struct Stor<__half> {
    static constexpr bool kScaled = true;
    __device__ static float4 ld4(const __half *p) {
        const uint2 u = *reinterpret_cast<const uint2 *>(p);
        const float2 a = __half22float2(*reinterpret_cast<const __half2 *>(&u.x));
        const float2 b = __half22float2(*reinterpret_cast<const __half2 *>(&u.y));
        return make_float4(a.x, a.y, b.x, b.y);
    }
    __device__ static float to_f(__half v) { return __half2float(v); }
    __device__ static __half from_f(float v) { return __float2half_rn(v); }
    __device__ static void st4(__half *p, float4 v) {
        const __half2 a = __floats2half2_rn(v.x, v.y), b = __floats2half2_rn(v.z, v.w);
        uint2 u;
        u.x = *reinterpret_cast<const uint32_t *>(&a);
        u.y = *reinterpret_cast<const uint32_t *>(&b);
        *reinterpret_cast<uint2 *>(p) = u;
    }
    __device__ static void st1(__half *p, float v) { *p = from_f(v); }
};
template <>
struct Stor<__nv_bfloat16> {
    static constexpr bool kScaled = true;
    __device__ static float4 ld4(const __nv_bfloat16 *p) {
        const uint2 u = *reinterpret_cast<const uint2 *>(p);
        const float2 a = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162 *>(&u.x));
        const float2 b = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162 *>(&u.y));
        return make_float4(a.x, a.y, b.x, b.y);
    }
    __device__ static float to_f(__nv_bfloat16 v) { return __bfloat162float(v); }
    __device__ static __nv_bfloat16 from_f(float v) { return __float2bfloat16_rn(v); }
    __device__ static void st4(__nv_bfloat16 *p, float4 v) {
        const __nv_bfloat162 a = __floats2bfloat162_rn(v.x, v.y), b = __floats2bfloat162_rn(v.z, v.w);
        uint2 u;
        u.x = *reinterpret_cast<const uint32_t *>(&a);
        u.y = *reinterpret_cast<const uint32_t *>(&b);
        *reinterpret_cast<uint2 *>(p) = u;
    }
    __device__ static void st1(__nv_bfloat16 *p, float v) { *p = from_f(v); }
};

// 2^e as a float for -126 <= e <= 127 (exact).
__device__ __forceinline__ float exp2i(int e) { return __int_as_float((e + 127) << 23); }

// Packed FP32 pairs (sm_100 f32x2 arithmetic): two independent lanes per instruction, each rounded
// as its scalar counterpart.
typedef unsigned long long f32x2;
__device__ __forceinline__ f32x2 pk2(float a, float b) {
    f32x2 r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
    return r;
}
__device__ __forceinline__ void upk2(f32x2 r, float &a, float &b) { asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(r)); }
__device__ __forceinline__ f32x2 add2(f32x2 a, f32x2 b) {
    f32x2 r;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
__device__ __forceinline__ f32x2 mul2(f32x2 a, f32x2 b) {
    f32x2 r;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
__device__ __forceinline__ f32x2 fma2(f32x2 a, f32x2 b, f32x2 c) {
    f32x2 r;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c));
    return r;
}

// Shared-memory plan of one variant.  T: storage type of P/PP/ps; IT: image type; V: launch variant.
template <int H, bool IMG, typename T = float, typename IT = float, int V = 0>
struct TmaShape {
    static constexpr int TZ = Variant<V>::TZ, TY = Variant<V>::TY;
    static constexpr int NT = (TZ / kVZ) * TY;  // consumer threads
    static constexpr int EALIGN = 16 / (int)sizeof(T) > 4 ? 16 / (int)sizeof(T) : 4;
    static constexpr int ZH = ((H + EALIGN - 1) / EALIGN) * EALIGN;  // z halo: whole 16-byte units
    static constexpr int SROWS = TY + 2 * H;
    static constexpr int SPITCH = TZ + 2 * ZH;
    static constexpr int STAGE = SROWS * SPITCH;  // elements written by one P tile load
    static constexpr int SALIGN = 128 / (int)sizeof(T);
    static constexpr int STRIDE = ((STAGE + SALIGN - 1) / SALIGN) * SALIGN;  // P slot pitch: 128 B
    static constexpr int CORE = TZ * TY;  // elements of one core tile
    // core slot, in bytes: PP (T), V (float) [, PS (T), IMG (IT)]
    static constexpr int OFF_V = CORE * (int)sizeof(T);
    static constexpr int OFF_PS = OFF_V + CORE * 4;
    static constexpr int OFF_IMG = OFF_PS + CORE * (int)sizeof(T);
    static constexpr int CSLOT = IMG ? OFF_IMG + CORE * (int)sizeof(IT) : OFF_PS;
    static constexpr int D = H + (IMG ? Variant<V>::DX_IMG : Variant<V>::DX);  // P slots
    static constexpr int R = IMG ? Variant<V>::R_IMG : Variant<V>::R;           // core slots
    static_assert(2 * H <= D && D >= H + 2, "warm-up planes and the lookahead must fit in the P ring");
    static constexpr size_t PRING_BYTES = (size_t)D * STRIDE * sizeof(T);
    static constexpr size_t SMEM = PRING_BYTES + (size_t)R * CSLOT + 2 * (D + R) * sizeof(uint64_t);
    // batched launches: one shot's StepArgs copied past the rings
    static constexpr size_t ARGS_OFF = (SMEM + 15) / 16 * 16;
    static constexpr size_t SMEM_BATCH = ARGS_OFF + sizeof(StepArgs);
    // taper forms: the taper factors of the P tile's SROWS rows, then of its SPITCH columns, past
    // the rings; a factor is stored negated (sign bit set) where the row / column is in a tapered
    // border, so one load gives both
    static constexpr size_t TAB_OFF = (SMEM + 15) / 16 * 16;
    static constexpr size_t SMEM_TAPER = TAB_OFF + (size_t)(SROWS + SPITCH) * sizeof(float);
    static constexpr size_t smem(int taper) { return taper == kTaperNone ? SMEM : SMEM_TAPER; }
};

// Taper of one P tile in shared memory, in place and in stored units (kTaperUpper / kTaperAll):
// plane x, rows yt0 - H .., columns zt0 - ZH ..; tab holds the tile's row and column factors
// (TmaShape::TAB_OFF).  Every consumer thread tapers a share of the tile; the caller ends the pass
// with a consumer barrier.
template <int H, int TAPER, bool IMG, typename T, typename IT>
__device__ __forceinline__ void taper_tile(T *st, const float *tab, const StepArgs &a, int x, int yt0, int zt0, int tid) {
    using S = TmaShape<H, IMG, T, IT>;
    using ST = Stor<T>;
    constexpr int ZH = S::ZH, SPITCH = S::SPITCH;
    const T *Pg = reinterpret_cast<const T *>(a.P);
    const size_t plane = (size_t)a.nye * a.nze;
    bool xb;
    const float fx = taper_factor(a.taper, a.blen, a.nxe, x, xb);
    constexpr int U = SPITCH / 4;  // four cells per unit
    for (int w = tid; w < S::SROWS * U; w += S::NT) {
        const int r = w / U, u = w - r * U;
        const int yy = yt0 - H + r;
        if (yy >= a.nye) continue;
        const float tyv = tab[r];
        const float fy = fabsf(tyv);
        const bool yb = signbit(tyv);
        const float4 tz4 = *reinterpret_cast<const float4 *>(tab + S::SROWS + 4 * u);
        T *p4 = st + r * SPITCH + 4 * u;
        float4 v4 = ST::ld4(p4);
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const int zz = zt0 - ZH + 4 * u + e;
            if (zz < 0 || zz >= a.nze) continue;
            const float fz = fabsf(get(tz4, e));
            const bool zb = signbit(get(tz4, e));
            float v = get(v4, e);
            if (TAPER == kTaperAll && quirk_cell(x, yy, zz, a)) {
                v = ST::to_f(Pg[(size_t)a.blen * plane + (size_t)yy * a.nze + zz]);
                v = v * fy;
                v = v * fx;
                v = v * fy;
            } else {
                v = taper_by_factors<TAPER>(v, fx, fy, fz, xb, yb, zb);
            }
            put(v4, e, v);
        }
        ST::st4(p4, v4);
    }
    // the slot is refilled by TMA later: order these generic-proxy writes before that
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// TAPER: kTaperNone / kTaperUpper / kTaperAll (raw P, tapered on load) / kTaperUpperStored /
// kTaperAllStored (the fields stored tapered: no pass over the P tile, no consumer barrier).
// IMG: the epilogue accumulates the image.
// T: storage type of P, PP and ps (float: the FP32 form, bit-identical to the plain-load kernel;
// __half / __nv_bfloat16: scaled 16-bit storage).  IT: image type (float or double).
// DF: increment storage (16-bit forms, no taper): the core ring's first tile is the increment
// d(t) = p(t) - p(t-1) instead of p(t-1); the launch writes d(t+1) = d(t) + v2dt2 lap p(t) in place
// and p(t+1) = p(t) + d(t+1) to StepArgs::Pout, each with its own exponent.
// The body of one CTA: the tile (bx, by) of the (z, y) plane and x chunk bz of the volume that
// (maps, a) describe; the stencil coefficients come from coef (for the compiler, a kernel
// parameter at a fixed offset, so the FMAs take them straight from the constant bank).
template <int H, bool EXACT, int TAPER, bool IMG, typename T, typename IT, bool DF = false, int V = 0, int UNR = 1>
__device__ __forceinline__ void tma_step_body(const TmaMaps &maps, const StepArgs &a, const StepArgs &coef, int bx,
                                              int by, int bz) {
    using S = TmaShape<H, IMG, T, IT, V>;
    static_assert(V == 0 || TAPER == kTaperNone, "the taper forms run the default variant");
    constexpr int kTZ = S::TZ, kTY = S::TY, kThreads = S::NT;  // this variant's tile and consumer threads
    using ST = Stor<T>;
    constexpr bool SC = ST::kScaled;
    static_assert(!DF || (SC && TAPER == kTaperNone), "increment storage: 16-bit forms without taper");
    // ALL: every face tapered; UPPER: the upper border only; TWS: the fields are stored tapered
    constexpr bool ALL = TAPER == kTaperAll || TAPER == kTaperAllStored;
    constexpr bool UPPER = TAPER == kTaperUpper || TAPER == kTaperUpperStored;
    constexpr bool TWS = TAPER == kTaperAllStored || TAPER == kTaperUpperStored;
    // CB: the consumers meet at named barriers (taper passes), so a timed-out wait must be seen by
    // all of them at the next barrier instead of one warp leaving alone
    constexpr bool CB = TAPER == kTaperUpper || TAPER == kTaperAll;
    static_assert(!(SC && EXACT), "the 16-bit storage forms use the FMA arithmetic");
    constexpr int ZH = S::ZH, SPITCH = S::SPITCH, STAGE = S::STAGE, STRIDE = S::STRIDE, D = S::D, R = S::R;
    constexpr int CSLOT = S::CSLOT;
    constexpr int NQ = 2 * H + 1;
    constexpr int ZQ = kTZ / kVZ;
    extern __shared__ __align__(128) unsigned char smem[];
    T *pring = reinterpret_cast<T *>(smem);
    unsigned char *cring = smem + S::PRING_BYTES;
    uint64_t *pfull = reinterpret_cast<uint64_t *>(cring + R * CSLOT);
    uint64_t *cfull = pfull + D;
    uint64_t *pempty = cfull + R;
    uint64_t *cempty = pempty + D;
    constexpr int NCW = kThreads / 32;  // consumer warps

    const int tid = threadIdx.x;
    const int tz = tid % ZQ, ty = tid / ZQ;
    const int zt0 = bx * kTZ;
    const int yt0 = H + by * kTY;
    const int z0 = zt0 + tz * kVZ;
    const int y = yt0 + ty;
    int xc0 = H + bz * a.chunk;
    int xc1 = min(xc0 + a.chunk, a.nxe - H);
    if (a.x_hi > 0) {  // 2D models: the plane x = blen only
        xc0 = max(xc0, a.x_lo);
        xc1 = min(xc1, a.x_hi);
    }
    if (xc0 >= xc1) return;
    const int n = xc1 - xc0;        // output planes, local index i <-> x = xc0 + i
    const int nplanes = n + 2 * H;  // P planes, local index k <-> x = xc0 - H + k
    const size_t plane = (size_t)a.nye * a.nze;

    float *tab = reinterpret_cast<float *>(smem + S::TAB_OFF);  // taper forms only
    if (TAPER != kTaperNone && tid < S::SROWS + SPITCH) {
        const bool row = tid < S::SROWS;
        const int i = row ? yt0 - H + tid : zt0 - ZH + (tid - S::SROWS);
        const int n_ax = row ? a.nye : a.nze;
        float f = 1.f;
        if (i >= 0 && i < n_ax) {
            bool in;
            f = taper_factor(a.taper, a.blen, n_ax, i, in);
            if (UPPER && !row) in = i < a.blen;
            if (in) f = -f;
        }
        tab[tid] = f;
    }
    if (tid == 0) {
        for (int s = 0; s < D; ++s) { mbar_init(&pfull[s], 1); mbar_init(&pempty[s], NCW); }
        for (int s = 0; s < R; ++s) { mbar_init(&cfull[s], 1); mbar_init(&cempty[s], NCW); }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();  // the last block-wide barrier: the producer warp leaves below

    if (tid >= kThreads) {
        // ---- producer: P plane k into slot k % D once plane k - D has been released; the core
        // tiles of output plane i = k - 2H right after, once core plane i - R has been released
        if (tid != kThreads) return;
        bool ok = true;
        int p_issued = 0, c_issued = 0;
        for (int k = 0; k < nplanes && ok; ++k) {
            const int s = k % D;
            if (k >= D && !(ok = mbar_wait_producer(&pempty[s], ((k / D) + 1) & 1))) break;
            mbar_expect_tx(&pfull[s], STAGE * sizeof(T));
            tma_load_3d(pring + s * STRIDE, &maps.p, &pfull[s], zt0 - ZH, yt0 - H, xc0 - H + k);
            p_issued = k + 1;
            if (k >= 2 * H) {
                const int i = k - 2 * H, cs = i % R;
                if (i >= R && !(ok = mbar_wait_producer(&cempty[cs], ((i / R) + 1) & 1))) break;
                unsigned char *dst = cring + cs * CSLOT;
                mbar_expect_tx(&cfull[cs], CSLOT);
                tma_load_3d(dst, &maps.pp, &cfull[cs], zt0, yt0, xc0 + i);
                tma_load_3d(dst + S::OFF_V, &maps.v, &cfull[cs], zt0, yt0, xc0 + i);
                if (IMG) {
                    tma_load_3d(dst + S::OFF_PS, &maps.ps, &cfull[cs], zt0, yt0, xc0 + i);
                    tma_load_3d(dst + S::OFF_IMG, &maps.img, &cfull[cs], zt0, yt0, xc0 + i);
                }
                c_issued = i + 1;
            }
        }
        if (!ok && a.err) atomicOr(a.err, 2u);
        // stay until every copy this CTA issued has landed (bounded), so none outlives the CTA
        for (int k = p_issued > D ? p_issued - D : 0; k < p_issued; ++k)
            if (!mbar_wait_producer(&pfull[k % D], (k / D) & 1)) break;
        for (int i = c_issued > R ? c_issued - R : 0; i < c_issued; ++i)
            if (!mbar_wait_producer(&cfull[i % R], (i / R) & 1)) break;
        return;
    }
    const int lane = tid & 31;

    // ---- scales of the 16-bit forms: the stored levels hold value * 2^-e
    float sP = 1.f, sPP = 1.f, sPS = 1.f, sOutInv = 1.f, sPPinv = 1.f, sKeep = 1.f;
    float sDInv = 1.f, sKeepP = 1.f;  // increment storage: d(t+1)'s inverse scale, p re-store factor
    if constexpr (SC) {
        const ScaleRec rp = *a.sc_p, rpp = *a.sc_pp;
        sP = exp2i(rp.e);
        sPP = exp2i(rpp.e);
        sPPinv = exp2i(-rpp.e);
        if (IMG) sPS = exp2i(a.sc_ps->e);
        const float inj = a.inj + (a.inj_dev ? *a.inj_dev : 0.f);
        const float ap = __uint_as_float(rp.amax), app = __uint_as_float(rpp.amax);
        if constexpr (DF) {
            // |d(t+1)| <= |d(t)| + 4 max|p(t)| + injection (a stable step: v2dt2 sum|coef| <= 4),
            // |p(t+1)| <= |p(t)| + |d(t+1)|; a receiver overwrite gives |d| <= |p| + |record|
            const float bd = app + 4.f * ap + inj;
            const int eD = storage_exponent(bd), eP = storage_exponent(ap + bd);
            sOutInv = exp2i(-eP);
            sDInv = exp2i(-eD);
            sKeep = exp2i(max(-126, min(127, rpp.e - eD)));  // cells outside the computed region
            sKeepP = exp2i(max(-126, min(127, rp.e - eP)));
            if (tid == 0 && bx == 0 && by == 0 && bz == 0) {
                a.sc_out->e = eP;
                a.sc_out2->e = eD;
            }
        } else {
            const float bound = 8.f * fmaxf(ap, app) + inj;
            const int eN = storage_exponent(bound);
            sOutInv = exp2i(-eN);
            sKeep = exp2i(max(-126, min(127, rpp.e - eN)));  // re-stores cells outside the computed region
            if (tid == 0 && bx == 0 && by == 0 && bz == 0) a.sc_out->e = eN;
        }
    }

    // ---- per-thread constants, hoisted out of the plane loop.  The rare per-cell work (source,
    // receivers, upper border, taper side buffer) is found per plane by CTA-uniform tests and its
    // per-thread details are derived there, so that nothing of it stays live across the stencil.
    // REC: receivers in the kernel (image forms inject them, 16-bit forms sample them); the FP32
    // forward forms have none (their drivers sample the stored level with a gather kernel).
    constexpr bool REC = IMG || SC;
    const bool row_ok = y < a.nye && z0 < a.nze;
    const bool y_ok = y < a.nye - H;
    unsigned vmask = 0, imask = 0;
#pragma unroll
    for (int e = 0; e < kVZ; ++e) {
        const int z = z0 + e;
        const bool v = y_ok && z >= H && z < a.nze - H;
        if (v) vmask |= 1u << e;
        if (v && IMG && z >= a.img_z0 && z < a.img_z1) imask |= 1u << e;
    }
    // CTA-uniform: which kinds of rare work can fall in this tile
    const bool src_cta = a.sye >= yt0 && a.sye < yt0 + kTY && a.sze >= zt0 && a.sze < zt0 + kTZ;
    const bool rec_cta = REC && a.rec_mode != kRecNone && a.rz >= zt0 && a.rz < zt0 + kTZ;
    const bool upb_cta = a.upb_mode != kUpbNone && zt0 < a.blen && zt0 + kTZ > a.blen - H;
    const bool q_cta = ALL && a.quirk_out && yt0 + kTY > a.nye - a.blen;
    bool tile_taper_yz = false;  // does this CTA's tile touch the taper region (x border aside)?
    if (ALL)
        tile_taper_yz = (yt0 - H < a.blen) || (yt0 + kTY + H > a.nye - a.blen) || (zt0 - ZH < a.blen) ||
                        (zt0 + kTZ + ZH > a.nze - a.blen);
    if (UPPER) tile_taper_yz = (zt0 - ZH < a.blen);
    bool pp_taper_yz = false;    // are this thread's own cells in the y or z taper region?
    if (ALL)
        pp_taper_yz = (y < a.blen) || (y >= a.nye - a.blen) || (z0 < a.blen) || (z0 + kVZ > a.nze - a.blen);
    if (UPPER) pp_taper_yz = z0 < a.blen;
    const size_t row_off = (size_t)y * a.nze + z0;
    T *PPp = reinterpret_cast<T *>(a.PP) + row_off;
    const int col = ZH + tz * kVZ;
    const int ccol = ty * kTZ + tz * kVZ;  // this thread's offset in a core tile

    bool bad_wait = false;
    // P slot k % D holds plane k; its "full" phase for plane k has parity (k / D) & 1.  The plane
    // loop keeps these as running counters instead of dividing.
    auto wait_p = [&](int slot, int parity) {  // warp-uniform outcome, so a warp never splits at a timeout
        // after a timeout (taper forms) the warp runs on without waiting, on undefined data, until
        // the next consumer barrier tells every warp to stop: so no warp leaves a barrier short
        if (CB && bad_wait) return;
        bad_wait |= !__all_sync(0xffffffffu, mbar_wait(&pfull[slot], parity));
    };
    auto release_p = [&](int slot) {  // this warp no longer reads the plane in this slot
        __syncwarp();
        if (lane == 0) mbar_arrive(&pempty[slot]);
    };
    // does the tile of P plane k need a pass before the stencil reads it?  Uniform across the CTA.
    auto plane_needs_taper = [&](int k) {
        const int x = xc0 - H + k;
        if (TAPER == kTaperAll) return tile_taper_yz || x < a.blen || x >= a.nxe - a.blen;
        return tile_taper_yz;
    };
    // taper of the tile of P plane k (kTaperUpper / kTaperAll)
    auto taper_stage = [&](int k, int slot) {
        taper_tile<H, TAPER, IMG, T, IT>(pring + slot * STRIDE, tab, a, xc0 - H + k, yt0, zt0, tid);
    };

    float4 q[NQ];
    float nanacc = 0.f;  // stays 0 unless a NaN or an infinity is written
    float amax = 0.f;    // max |value| written (16-bit forms)
    float amaxd = 0.f;   // max |increment| written (increment storage)
    // running ring positions: plane kin = i + 2H (slot, parity), the centre plane i + H (slot), the
    // core plane i (slot, parity)
    int s_in = (2 * H) % D, ph_in = ((2 * H) / D) & 1, s_mid = H % D, s_core = 0, ph_core = 0;
    // isotropic grids (dx = dy = dz) in the FP32 FMA form: packed pairs over the symmetric stencil
    // (14% fewer instructions; for the 16-bit forms the packing of the widened taps cost more than
    // it saved, measured 4% slower, so they keep the scalar chains)
    const bool iso = !EXACT && !SC && a.iso;
    f32x2 cpk[H + 1];
    cpk[0] = pk2(coef.cx[H] + coef.cy[H] + coef.cz[H], coef.cx[H] + coef.cy[H] + coef.cz[H]);
#pragma unroll
    for (int k = 1; k <= H; ++k) cpk[k] = pk2(coef.cx[H + k], coef.cx[H + k]);
    // warm-up: P planes 0 .. 2H-1 into the queue; planes 0 .. H-1 are not computed here
    for (int k = 0; k < 2 * H; ++k) {  // 2H <= D: slots 0 .. 2H-1, first phase
        wait_p(k, 0);
        if (CB && plane_needs_taper(k)) taper_stage(k, k);
    }
    if (CB ? consumer_sync_or<kThreads>(bad_wait) : bad_wait) goto drain;
#pragma unroll
    for (int k = 0; k < 2 * H; ++k) q[k + 1] = ST::ld4(pring + k * STRIDE + (ty + H) * SPITCH + col);
#pragma unroll
    for (int k = 0; k < H; ++k) release_p(k);  // planes 0 .. H-1 were only needed for the queue

RTMB_UNROLL_PRAGMA(UNR)
    for (int i = 0; i < n; ++i, s_in = s_in + 1 == D ? (ph_in ^= 1, 0) : s_in + 1, s_mid = s_mid + 1 == D ? 0 : s_mid + 1,
                           s_core = s_core + 1 == R ? (ph_core ^= 1, 0) : s_core + 1) {
        {
            const int x = xc0 + i;
            const int kin = i + 2 * H;
            // receivers in this plane (REC forms): the record value the receiver step injects is
            // loaded now so that its latency (a strided gather) overlaps the stencil instead of
            // stalling the warp at the end of the plane
            int rec_e = -1;
            float rec_v = 0.f;
            const float *rec_p = nullptr;
            if (REC && rec_cta) {
                const int dxr = x - a.rx0, dyr = y - a.ry0, e = a.rz - z0;
                if (dxr >= 0 && dxr % a.rdx == 0 && dxr / a.rdx < a.rcx && e >= 0 && e < kVZ && ((vmask >> e) & 1u) &&
                    dyr >= 0 && dyr % a.rdy == 0 && dyr / a.rdy < a.rcy) {
                    rec_e = e;
                    rec_p = a.rec + a.rec_base + (dxr / a.rdx) * a.rec_si + (dyr / a.rdy) * a.rec_sj;
                    if (IMG && a.rec_mode != kRecSample) rec_v = __ldg(rec_p);  // read-only in this launch
                }
            }
            wait_p(s_in, ph_in);
            const T *s = pring + s_mid * STRIDE;  // the centre plane's tile
            if constexpr (CB) {
                if (plane_needs_taper(kin)) {  // the pass is collective: all warps take this branch
                    taper_stage(kin, s_in);
                    if (consumer_sync_or<kThreads>(bad_wait)) goto drain;
                }
            } else if (bad_wait) {
                goto drain;  // a timed-out wait leaves the data undefined; stop without computing
            }
#pragma unroll
            for (int k = 0; k < NQ - 1; ++k) q[k] = q[k + 1];  // advance the x queue
            q[NQ - 1] = ST::ld4(pring + s_in * STRIDE + (ty + H) * SPITCH + col);

            float lap[kVZ] = {0.f, 0.f, 0.f, 0.f};
            if (row_ok) {
                float zr[kVZ + 2 * ZH];
#pragma unroll
                for (int k = 0; k < (kVZ + 2 * ZH) / 4; ++k) {
                    const float4 t4 =
                        (k == ZH / 4) ? q[H] : ST::ld4(s + (ty + H) * SPITCH + col - ZH + 4 * k);
                    zr[4 * k + 0] = t4.x; zr[4 * k + 1] = t4.y; zr[4 * k + 2] = t4.z; zr[4 * k + 3] = t4.w;
                }
                if (EXACT) {
                    float ax[kVZ], ay[kVZ], az[kVZ];
#pragma unroll
                    for (int e = 0; e < kVZ; ++e) { ax[e] = 0.f; ay[e] = 0.f; az[e] = 0.f; }
#pragma unroll
                    for (int io = 0; io < NQ; ++io) {
                        const float4 qx = q[io];
                        const float4 ry = (io == H) ? q[H] : ST::ld4(s + (ty + io) * SPITCH + col);
#pragma unroll
                        for (int e = 0; e < kVZ; ++e) {
                            ax[e] = ax[e] + get(qx, e) * coef.cx[io];
                            ay[e] = ay[e] + get(ry, e) * coef.cy[io];
                            az[e] = az[e] + zr[ZH - H + e + io] * coef.cz[io];
                        }
                    }
#pragma unroll
                    for (int e = 0; e < kVZ; ++e) lap[e] = ax[e] + ay[e] + az[e];
                } else if (iso) {
                    // lap = c0 p + sum_k c_k (x+-k, y+-k, z+-k neighbours), on the point pairs (0, 1)
                    // and (2, 3): 5 packed operations per k and pair instead of 6 scalar FMAs per k
                    // and point
                    const float4 qc = q[H];
                    f32x2 l0 = mul2(pk2(qc.x, qc.y), cpk[0]), l1 = mul2(pk2(qc.z, qc.w), cpk[0]);
#pragma unroll
                    for (int k = 1; k <= H; ++k) {
                        const float4 xa = q[H + k], xb = q[H - k];
                        const float4 ya = ST::ld4(s + (ty + H + k) * SPITCH + col);
                        const float4 yb = ST::ld4(s + (ty + H - k) * SPITCH + col);
                        const f32x2 t0 = add2(add2(add2(pk2(xa.x, xa.y), pk2(xb.x, xb.y)), add2(pk2(ya.x, ya.y), pk2(yb.x, yb.y))),
                                              add2(pk2(zr[ZH + k], zr[ZH + k + 1]), pk2(zr[ZH - k], zr[ZH - k + 1])));
                        const f32x2 t1 = add2(add2(add2(pk2(xa.z, xa.w), pk2(xb.z, xb.w)), add2(pk2(ya.z, ya.w), pk2(yb.z, yb.w))),
                                              add2(pk2(zr[ZH + 2 + k], zr[ZH + 3 + k]), pk2(zr[ZH + 2 - k], zr[ZH + 3 - k])));
                        l0 = fma2(t0, cpk[k], l0);
                        l1 = fma2(t1, cpk[k], l1);
                    }
                    upk2(l0, lap[0], lap[1]);
                    upk2(l1, lap[2], lap[3]);
                } else {
                    const float cc = coef.cx[H] + coef.cy[H] + coef.cz[H];
                    const float4 qc = q[H];
#pragma unroll
                    for (int e = 0; e < kVZ; ++e) lap[e] = get(qc, e) * cc;
#pragma unroll
                    for (int io = 0; io < NQ; ++io) {
                        if (io == H) continue;
                        const float4 qx = q[io];
                        const float4 ry = ST::ld4(s + (ty + io) * SPITCH + col);
#pragma unroll
                        for (int e = 0; e < kVZ; ++e) {
                            lap[e] = fmaf(get(qx, e), coef.cx[io], lap[e]);
                            lap[e] = fmaf(get(ry, e), coef.cy[io], lap[e]);
                            lap[e] = fmaf(zr[ZH - H + e + io], coef.cz[io], lap[e]);
                        }
                    }
                }
            }
            release_p(s_mid);  // the tile of plane x is no longer read
            // core tiles of plane x
            const int cs = s_core;
            if (CB && bad_wait) continue;  // run on to the next barrier (see wait_p)
            if (!__all_sync(0xffffffffu, mbar_wait(&cfull[cs], ph_core))) {
                bad_wait = true;
                if (CB) continue;  // the other warps learn of it at the next barrier
                goto drain;
            }
            const unsigned char *ct = cring + cs * CSLOT;
            const float4 pp_raw = ST::ld4(reinterpret_cast<const T *>(ct) + ccol);
            const float4 vv = ld_f4(reinterpret_cast<const float *>(ct + S::OFF_V) + ccol);
            float4 ps4 = pp_raw;
            IT im[kVZ];
            if (IMG) {
                ps4 = ST::ld4(reinterpret_cast<const T *>(ct + S::OFF_PS) + ccol);
                const IT *imt = reinterpret_cast<const IT *>(ct + S::OFF_IMG) + ccol;
                if constexpr (sizeof(IT) == 4) {
                    const float4 t4 = ld_f4(reinterpret_cast<const float *>(imt));
                    im[0] = t4.x; im[1] = t4.y; im[2] = t4.z; im[3] = t4.w;
                } else {
                    const double2 d0 = reinterpret_cast<const double2 *>(imt)[0];
                    const double2 d1 = reinterpret_cast<const double2 *>(imt)[1];
                    im[0] = d0.x; im[1] = d0.y; im[2] = d1.x; im[3] = d1.y;
                }
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(&cempty[cs]);
            if (!row_ok) continue;

            const float4 qc = q[H];
            float ppv[kVZ] = {pp_raw.x, pp_raw.y, pp_raw.z, pp_raw.w};  // stored units
            // the taper of this thread's cells of plane x: T(v) = ((v f1) f2) f3 (the factor order of
            // taper_by_factors; a factor of 1 is exact).  PP holds T(u) (TWS: one more T) or the raw
            // u (T o T); the factors are re-derived where they are needed, not kept live.
            bool tap = false, xb = false;
            if (TAPER != kTaperNone) {
                xb = x < a.blen || x >= a.nxe - a.blen;  // uniform over the CTA
                tap = pp_taper_yz || (ALL && xb);
            }
            if (TAPER != kTaperNone && tap) {
                const float fx = xb ? taper_factor_in(a.taper, a.blen, a.nxe, x) : 1.f;
                const float tyv = tab[H + ty];  // this thread's row
                const float fy = fabsf(tyv);
                const bool yb = signbit(tyv);
                const float4 tz4 = *reinterpret_cast<const float4 *>(tab + S::SROWS + ZH + tz * kVZ);
                const bool qx = ALL && a.quirk && x < a.blen && y >= a.nye - a.blen;
                const bool once = TWS || (a.tw & kTwPPOnce);  // PP holds T(u): one more T
                // the cases are uniform per thread, so each runs its own unrolled loop; cells
                // outside the computed region are tapered too (harmless: they keep their stored
                // value on output)
                if (qx) {  // rare: planes x < blen, rows on the right y border
#pragma unroll
                    for (int e = 0; e < kVZ; ++e) {
                        const int z = z0 + e;
                        float pp = ppv[e];
                        if (((vmask >> e) & 1u) && z >= a.blen && z < a.nze - a.blen) {
                            // the x = blen redirect, twice: from the raw u(blen, y, z) of PP's level
                            pp = a.quirk_in[(size_t)(y - (a.nye - a.blen)) * (a.nze - 2 * a.blen) + (z - a.blen)];
                            if (SC) pp = pp * sPPinv;  // the side buffer holds values, not stored units
                            pp = pp * fy;
                            pp = pp * fy;
                            pp = pp * fx;
                            pp = pp * fy;
                        } else {
                            float f1, f2, f3;
                            taper_factors3<ALL>(fx, fy, fabsf(get(tz4, e)), xb, yb, signbit(get(tz4, e)), f1, f2, f3);
                            pp = ((pp * f1) * f2) * f3;
                            if (!once) pp = ((pp * f1) * f2) * f3;
                        }
                        ppv[e] = pp;
                    }
                } else if (ALL && !xb) {  // fx = 1: T(v) = (v fy) fz
#pragma unroll
                    for (int e = 0; e < kVZ; ++e) {
                        const float fz = fabsf(get(tz4, e));
                        float pp = (ppv[e] * fy) * fz;
                        if (!once) pp = (pp * fy) * fz;
                        ppv[e] = pp;
                    }
                } else {
#pragma unroll
                    for (int e = 0; e < kVZ; ++e) {
                        float f1, f2, f3;
                        taper_factors3<ALL>(fx, fy, fabsf(get(tz4, e)), xb, yb, signbit(get(tz4, e)), f1, f2, f3);
                        float pp = ((ppv[e] * f1) * f2) * f3;
                        if (!once) pp = ((pp * f1) * f2) * f3;
                        ppv[e] = pp;
                    }
                }
            }
            float npp[kVZ];
            float dn[kVZ];  // increment storage: d(t+1)
#pragma unroll
            for (int e = 0; e < kVZ; ++e) {
                if (DF) {  // d(t+1) = d(t) + v2dt2 lap p(t), p(t+1) = p(t) + d(t+1)
                    dn[e] = fmaf(get(vv, e), lap[e] * sP, ppv[e] * sPP);
                    npp[e] = fmaf(get(qc, e), sP, dn[e]);
                } else if (EXACT) {
                    const float two_p = 2.f * get(qc, e);
                    const float d = two_p - ppv[e];
                    const float vl = get(vv, e) * lap[e];
                    npp[e] = d + vl;
                } else if (SC) {  // exact power-of-two rescaling of the stored units
                    npp[e] = fmaf(get(vv, e), lap[e] * sP, (2.f * sP) * get(qc, e) - ppv[e] * sPP);
                } else {
                    npp[e] = fmaf(get(vv, e), lap[e], 2.f * get(qc, e) - ppv[e]);
                }
            }
            // source, receivers, upper border, taper side buffer: CTA-uniform tests first
            if ((src_cta && x == a.sxe) || rec_e >= 0 || upb_cta || (q_cta && x == a.blen)) {
#pragma unroll
                for (int e = 0; e < kVZ; ++e) {
                    const int z = z0 + e;
                    const bool v = (vmask >> e) & 1u;
                    if (x == a.sxe && y == a.sye && z == a.sze && v) {
                        const float w = __ldg(a.wavelet + a.it);
                        npp[e] = npp[e] + w;
                        if (DF) dn[e] = dn[e] + w;
                    }
                    if (REC && e == rec_e) {
                        float *rp = const_cast<float *>(rec_p);
                        const float rv = IMG ? rec_v : *rp;
                        if (a.rec_mode == kRecSample) {
                            *rp = npp[e];
                        } else if (a.rec_mode == kRecOverwrite) {
                            if (DF) dn[e] = rv - get(qc, e) * sP;  // p(t+1) = record, d(t+1) = record - p(t)
                            npp[e] = rv;
                        } else {
                            npp[e] = npp[e] + rv;
                            if (DF) dn[e] = dn[e] + rv;
                        }
                    }
                    if (upb_cta && v && z >= a.blen - H && z < a.blen) {
                        float *up = a.upb + ((size_t)x * a.nye + y) * H + (z - (a.blen - H));
                        if (a.upb_mode == kUpbSave) *up = npp[e];
                        else npp[e] = *up;
                    }
                    if (q_cta && x == a.blen && v && y >= a.nye - a.blen && z >= a.blen && z < a.nze - a.blen)
                        a.quirk_out[(size_t)(y - (a.nye - a.blen)) * (a.nze - 2 * a.blen) + (z - a.blen)] = npp[e];
                }
                if (TWS && q_cta && x == a.blen && y >= a.nye - a.blen) {
                    // stored tapered, the quirk cells (x' < blen) of the new level hold
                    // ((u(blen, y, z) fy) fx') fy: written here, where u(blen, y, z) is known, and
                    // skipped by the CTAs that compute plane x'
                    unsigned qm = 0;
#pragma unroll
                    for (int e = 0; e < kVZ; ++e)
                        if (((vmask >> e) & 1u) && z0 + e >= a.blen && z0 + e < a.nze - a.blen) qm |= 1u << e;
                    const float fy = fabsf(tab[H + ty]);
                    T *qp = PPp;
                    for (int xq = 0; qm && xq < a.blen; ++xq, qp += plane) {
                        const float fxq = __ldg(a.taper + (a.blen - 1 - xq));
                        float4 o4;
#pragma unroll
                        for (int e = 0; e < kVZ; ++e) {
                            float v = ((npp[e] * fy) * fxq) * fy;
                            if (SC) v = v * sOutInv;
                            put(o4, e, v);
                        }
                        if (qm == 0xFu) {
                            ST::st4(qp, o4);
                        } else {
#pragma unroll
                            for (int e = 0; e < kVZ; ++e)
                                if ((qm >> e) & 1u) ST::st1(qp + e, get(o4, e));
                        }
                    }
                }
            }
            // the stored level: T(u_new) in the stored-taper forms; the receivers, the side buffer and
            // the image take u_new itself
            float nst[kVZ];
#pragma unroll
            for (int e = 0; e < kVZ; ++e) nst[e] = npp[e];
            if (TWS && tap && !(a.tw & kTwRawOut)) {
                const float tyv = tab[H + ty];
                const float4 tz4 = *reinterpret_cast<const float4 *>(tab + S::SROWS + ZH + tz * kVZ);
                if (ALL && !xb) {  // fx = 1: T(v) = (v fy) fz
#pragma unroll
                    for (int e = 0; e < kVZ; ++e) nst[e] = (npp[e] * fabsf(tyv)) * fabsf(get(tz4, e));
                } else {
                    const float fx = xb ? taper_factor_in(a.taper, a.blen, a.nxe, x) : 1.f;
#pragma unroll
                    for (int e = 0; e < kVZ; ++e) {
                        float f1, f2, f3;
                        taper_factors3<ALL>(fx, fabsf(tyv), fabsf(get(tz4, e)), xb, signbit(tyv), signbit(get(tz4, e)),
                                            f1, f2, f3);
                        nst[e] = ((npp[e] * f1) * f2) * f3;
                    }
                }
            }
            float4 out;
            if constexpr (DF) {  // d(t+1) in place, p(t+1) to Pout
                float4 od;
#pragma unroll
                for (int e = 0; e < kVZ; ++e) {
                    const bool v = (vmask >> e) & 1u;
                    put(od, e, v ? dn[e] * sDInv : get(pp_raw, e) * sKeep);
                    put(out, e, v ? npp[e] * sOutInv : get(qc, e) * sKeepP);
                    if (v) {
                        amax = fmaxf(amax, fabsf(npp[e]));
                        amaxd = fmaxf(amaxd, fabsf(dn[e]));
                    }
                    nanacc = fmaf(0.f, npp[e], nanacc);
                    nanacc = fmaf(0.f, dn[e], nanacc);
                }
                ST::st4(PPp + (size_t)x * plane, od);
                ST::st4(reinterpret_cast<T *>(a.Pout) + row_off + (size_t)x * plane, out);
            }
#pragma unroll
            for (int e = 0; e < kVZ && !DF; ++e) {
                const bool v = (vmask >> e) & 1u;
                float o;
                if (SC) {
                    o = v ? nst[e] * sOutInv : get(pp_raw, e) * sKeep;
                    if (v) amax = fmaxf(amax, fabsf(nst[e]));
                    nanacc = fmaf(0.f, nst[e], nanacc);
                } else {
                    o = v ? nst[e] : get(pp_raw, e);
                    nanacc = fmaf(0.f, o, nanacc);  // stays 0 unless a NaN or an infinity appears
                }
                put(out, e, o);
            }
            if (DF) {
                // stored above
            } else if (TWS && q_cta && x < a.blen && y >= a.nye - a.blen) {  // quirk cells: plane blen's CTA writes them
#pragma unroll
                for (int e = 0; e < kVZ; ++e) {
                    const int z = z0 + e;
                    if (!(((vmask >> e) & 1u) && z >= a.blen && z < a.nze - a.blen))
                        ST::st1(PPp + (size_t)x * plane + e, get(out, e));
                }
            } else {
                ST::st4(PPp + (size_t)x * plane, out);
            }
            if (IMG && imask) {
                IT *ig = reinterpret_cast<IT *>(a.img) + row_off + (size_t)x * plane;
                IT res[kVZ];
#pragma unroll
                for (int e = 0; e < kVZ; ++e) {
                    IT acc;
                    if (SC) acc = im[e] + (IT)(get(ps4, e) * sPS) * (IT)npp[e];
                    else acc = im[e] + (IT)get(ps4, e) * (IT)npp[e];  // valid cells: the new level
                    res[e] = ((imask >> e) & 1u) ? acc : im[e];
                }
                if constexpr (sizeof(IT) == 4) {
                    *reinterpret_cast<float4 *>(ig) = make_float4((float)res[0], (float)res[1], (float)res[2],
                                                                  (float)res[3]);
                } else {
                    reinterpret_cast<double2 *>(ig)[0] = make_double2((double)res[0], (double)res[1]);
                    reinterpret_cast<double2 *>(ig)[1] = make_double2((double)res[2], (double)res[3]);
                }
            }
        }
    }
    if (nanacc != nanacc && a.err) atomicOr(a.err, 1u);
    if (bad_wait && a.err) atomicOr(a.err, 2u);  // a core-tile wait ran out in the last plane
    if constexpr (SC) {
        const unsigned m = __reduce_max_sync(0xffffffffu, __float_as_uint(amax));
        if (lane == 0 && m) atomicMax(&a.sc_out->amax, m);
        if constexpr (DF) {
            const unsigned md = __reduce_max_sync(0xffffffffu, __float_as_uint(amaxd));
            if (lane == 0 && md) atomicMax(&a.sc_out2->amax, md);
        }
    }
    return;

drain:
    // A wait ran out: record it and stop this warp (the producer outlives the copies it issued).
    if (a.err) atomicOr(a.err, 2u);
}

// Plane-loop unroll of a step kernel: RTMB_PLANE_UNROLL for order 8 without taper and without
// increment storage (the forms it was measured on); the taper and increment forms and the batched
// kernel, which spill registers when unrolled, keep the plain loop.
template <int H, int TAPER, bool DF>
struct StepUnroll {
    static constexpr int value = (H == 4 && TAPER == kTaperNone && !DF) ? RTMB_PLANE_UNROLL : 1;
};

template <int H, bool EXACT, int TAPER, bool IMG, typename T = float, typename IT = float, bool DF = false, int V = 0>
__global__ void __launch_bounds__(variant_threads<V>(), Variant<V>::MINB)
    tma_step_kernel(const __grid_constant__ TmaMaps maps, const __grid_constant__ StepArgs a) {
    tma_step_body<H, EXACT, TAPER, IMG, T, IT, DF, V, StepUnroll<H, TAPER, DF>::value>(maps, a, a, blockIdx.x,
                                                                                       blockIdx.y, blockIdx.z);
}

// Several volumes in one launch (the batched multi-shot drivers): shot s owns the linear blocks
// [start[s], start[s+1]), laid out as its own (gx, gy, gz) grid.  All shots share the stencil
// coefficients (coef) and the kernel variant; everything else is per shot.
constexpr int kMaxBatch = kMaxBatchShots;
struct BatchArgs {
    int nshots;
    int start[kMaxBatch + 1];
    int gx[kMaxBatch], gy[kMaxBatch];
    StepArgs coef;
    TmaMaps maps[kMaxBatch];
    StepArgs args[kMaxBatch];
};

template <int H, bool EXACT, int TAPER, bool IMG, typename T = float, typename IT = float>
__global__ void __launch_bounds__(kTmaThreads, 2) tma_batch_kernel(const __grid_constant__ BatchArgs b) {
    int lin = blockIdx.x, s = 0;
    while (s + 1 < b.nshots && lin >= b.start[s + 1]) ++s;
    lin -= b.start[s];
    const int bx = lin % b.gx[s];
    lin /= b.gx[s];
    const int by = lin % b.gy[s], bz = lin / b.gy[s];
    // this shot's arguments in shared memory: read through a dynamic index the parameter space
    // would be reloaded after every global store of the plane loop; shared memory cannot alias them.
    // The copy sits in the dynamic region past the body's rings (a static __shared__ variable would
    // move the dynamic base off the 128-byte alignment the TMA destinations need).
    using S = TmaShape<H, IMG, T, IT>;
    extern __shared__ __align__(128) unsigned char smem_b[];
    StepArgs *sa = reinterpret_cast<StepArgs *>(smem_b + S::ARGS_OFF);
    static_assert(sizeof(StepArgs) % 4 == 0, "copied as words");
    const uint32_t *src = reinterpret_cast<const uint32_t *>(&b.args[s]);
    for (int i = threadIdx.x; i < (int)(sizeof(StepArgs) / 4); i += blockDim.x) reinterpret_cast<uint32_t *>(sa)[i] = src[i];
    __syncthreads();
    tma_step_body<H, EXACT, TAPER, IMG, T, IT>(b.maps[s], *sa, b.coef, bx, by, bz);
}

template <int H>
cudaError_t launch_tma_h(const TmaMaps &maps, const StepArgs &a, bool exact, int taper, bool img, dim3 grid,
                         cudaStream_t s) {
    // the dynamic shared-memory opt-in, once per (variant, device)
    static unsigned long long attr_done[20 * kVariants] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (a.tw & kTwStored) taper = taper == kTaperAll ? kTaperAllStored : (taper == kTaperUpper ? kTaperUpperStored : -1);
    if (taper < 0) return cudaErrorInvalidValue;
    const int lv = (taper == kTaperNone && H == 4) ? a.variant : 0;  // launch variant: RBC forms of order 8
    if (lv < 0 || lv >= kVariants) return cudaErrorInvalidValue;
    const int variant = 20 * lv + (exact ? 10 : 0) + (img ? 5 : 0) + taper;
    auto run = [&](void (*kern)(TmaMaps, StepArgs), size_t smem, int threads) -> cudaError_t {
        const unsigned long long bit = 1ull << (dev & 63);
        if (!(attr_done[variant] & bit)) {
            cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (e != cudaSuccess) return e;
            attr_done[variant] |= bit;
        }
        kern<<<grid, threads, smem, s>>>(maps, a);
        return cudaGetLastError();
    };
#define RTMB_TMA_CASE(EX, TP, IM) \
    if (lv == 0 && exact == EX && taper == TP && img == IM) \
        return run(tma_step_kernel<H, EX, TP, IM>, TmaShape<H, IM>::smem(TP), kTmaThreads);
    RTMB_TMA_CASE(true, kTaperNone, false)
    RTMB_TMA_CASE(true, kTaperUpper, false)
    RTMB_TMA_CASE(true, kTaperAll, false)
    RTMB_TMA_CASE(true, kTaperAllStored, false)
    RTMB_TMA_CASE(true, kTaperUpperStored, false)
    RTMB_TMA_CASE(true, kTaperNone, true)
    RTMB_TMA_CASE(true, kTaperUpper, true)
    RTMB_TMA_CASE(true, kTaperUpperStored, true)
    RTMB_TMA_CASE(false, kTaperNone, false)
    RTMB_TMA_CASE(false, kTaperUpper, false)
    RTMB_TMA_CASE(false, kTaperAll, false)
    RTMB_TMA_CASE(false, kTaperAllStored, false)
    RTMB_TMA_CASE(false, kTaperUpperStored, false)
    RTMB_TMA_CASE(false, kTaperNone, true)
    RTMB_TMA_CASE(false, kTaperUpper, true)
    RTMB_TMA_CASE(false, kTaperUpperStored, true)
#undef RTMB_TMA_CASE
    if constexpr (H == 4) {
#define RTMB_TMA_VCASE(VV, EX, IM)                                                                         \
    if (lv == VV && exact == EX && img == IM)                                                              \
        return run(tma_step_kernel<H, EX, kTaperNone, IM, float, float, false, VV>,                          \
                   TmaShape<H, IM, float, float, VV>::smem(kTaperNone), variant_threads<VV>());
        RTMB_TMA_VCASE(1, true, false) RTMB_TMA_VCASE(1, true, true) RTMB_TMA_VCASE(1, false, false) RTMB_TMA_VCASE(1, false, true)
        RTMB_TMA_VCASE(2, true, false) RTMB_TMA_VCASE(2, true, true) RTMB_TMA_VCASE(2, false, false) RTMB_TMA_VCASE(2, false, true)
        RTMB_TMA_VCASE(3, true, false) RTMB_TMA_VCASE(3, true, true) RTMB_TMA_VCASE(3, false, false) RTMB_TMA_VCASE(3, false, true)
#undef RTMB_TMA_VCASE
    }
    return cudaErrorInvalidValue;
}

// The 16-bit storage forms (order 8, FMA arithmetic): T = __half or __nv_bfloat16; img64 selects a
// double image.
template <typename T>
cudaError_t launch_tma_store(const TmaMaps &maps, const StepArgs &a, int taper, bool img, bool img64, dim3 grid,
                             cudaStream_t s) {
    static unsigned long long attr_done[16] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (a.tw & kTwStored) taper = taper == kTaperAll ? kTaperAllStored : -1;  // 16-bit forms: modeling only
    if (taper < 0) return cudaErrorInvalidValue;
    if (a.diff && (taper != kTaperNone || !a.Pout || !a.sc_out2)) return cudaErrorInvalidValue;
    const int variant = a.diff ? 12 + (img ? (img64 ? 2 : 1) : 0) : (img ? (img64 ? 8 : 4) : 0) + taper;
    auto run = [&](void (*kern)(TmaMaps, StepArgs), size_t smem) -> cudaError_t {
        const unsigned long long bit = 1ull << (dev & 63);
        if (!(attr_done[variant] & bit)) {
            cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (e != cudaSuccess) return e;
            attr_done[variant] |= bit;
        }
        kern<<<grid, kTmaThreads, smem, s>>>(maps, a);
        return cudaGetLastError();
    };
#define RTMB_TMA_STORE_CASE(TP, IM, IT)                                                          \
    if (!a.diff && taper == TP && img == IM && (!IM || img64 == (sizeof(IT) == 8)))              \
        return run(tma_step_kernel<4, false, TP, IM, T, IT>, TmaShape<4, IM, T, IT>::smem(TP));
#define RTMB_TMA_DIFF_CASE(IM, IT)                                                               \
    if (a.diff && img == IM && (!IM || img64 == (sizeof(IT) == 8)))                              \
        return run(tma_step_kernel<4, false, kTaperNone, IM, T, IT, true>, TmaShape<4, IM, T, IT>::smem(kTaperNone));
    RTMB_TMA_DIFF_CASE(false, float)
    RTMB_TMA_DIFF_CASE(true, float)
    RTMB_TMA_DIFF_CASE(true, double)
#undef RTMB_TMA_DIFF_CASE
    RTMB_TMA_STORE_CASE(kTaperNone, false, float)
    RTMB_TMA_STORE_CASE(kTaperUpper, false, float)
    RTMB_TMA_STORE_CASE(kTaperAll, false, float)
    RTMB_TMA_STORE_CASE(kTaperAllStored, false, float)
    RTMB_TMA_STORE_CASE(kTaperNone, true, float)
    RTMB_TMA_STORE_CASE(kTaperUpper, true, float)
    RTMB_TMA_STORE_CASE(kTaperNone, true, double)
    RTMB_TMA_STORE_CASE(kTaperUpper, true, double)
#undef RTMB_TMA_STORE_CASE
    return cudaErrorInvalidValue;
}

// The batched multi-shot kernels: the RBC migration variants (no taper), FP32 (exact or FMA) and the
// 16-bit storage forms (FMA), with or without the image.
template <typename T>
cudaError_t launch_tma_batch(const BatchArgs &b, bool exact, bool img, bool img64, int blocks, cudaStream_t s) {
    static unsigned long long attr_done[6] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    const int variant = (exact ? 3 : 0) + (img ? (img64 ? 2 : 1) : 0);
    auto run = [&](void (*kern)(BatchArgs), size_t smem) -> cudaError_t {
        const unsigned long long bit = 1ull << (dev & 63);
        if (!(attr_done[variant] & bit)) {
            cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (e != cudaSuccess) return e;
            attr_done[variant] |= bit;
        }
        kern<<<blocks, kTmaThreads, smem, s>>>(b);
        return cudaGetLastError();
    };
    if constexpr (sizeof(T) == 4) {
        if (img64) return cudaErrorInvalidValue;
        if (exact)
            return img ? run(tma_batch_kernel<4, true, kTaperNone, true>, TmaShape<4, true>::SMEM_BATCH)
                       : run(tma_batch_kernel<4, true, kTaperNone, false>, TmaShape<4, false>::SMEM_BATCH);
        return img ? run(tma_batch_kernel<4, false, kTaperNone, true>, TmaShape<4, true>::SMEM_BATCH)
                   : run(tma_batch_kernel<4, false, kTaperNone, false>, TmaShape<4, false>::SMEM_BATCH);
    } else {
        if (exact) return cudaErrorInvalidValue;
        if (!img) return run(tma_batch_kernel<4, false, kTaperNone, false, T, float>, TmaShape<4, false, T, float>::SMEM_BATCH);
        if (img64)
            return run(tma_batch_kernel<4, false, kTaperNone, true, T, double>, TmaShape<4, true, T, double>::SMEM_BATCH);
        return run(tma_batch_kernel<4, false, kTaperNone, true, T, float>, TmaShape<4, true, T, float>::SMEM_BATCH);
    }
}

}  // namespace detail
}  // namespace rtmb
