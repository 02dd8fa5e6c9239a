// stencil_dual_impl.cuh -- the dual-wavefield backward step (sm_100a, FP32): one launch advances the
// reconstructed source wavefield S and the back-propagated receiver wavefield R one step and adds
// S_new * R_new to the image, which the separate launches do in two passes (the source step, then
// the receiver step reading S_new back from HBM).  Per point it moves 36 bytes instead of 16 + 28:
// v2dt2 is read once and S_new never leaves the chip for the image.  The merged form can also pair
// consecutive launches on the image (StepArgs::img_pair): 28 + 36 bytes per point for two steps.
//
// Same arithmetic per point as the single-wavefield kernel (stencil_tma_impl.cuh), so results are
// bit-identical to the two launches, in both arithmetic forms.
//
// Two forms.  Split (dual_step_kernel, launch variants 0-3): eight consumer warps and one producer
// warp, two CTAs per SM; warps 0-3 step S, warps 4-7 step R, on the same tile and x chunk.  The
// producer fills two P rings (S and R halo tiles) and one core ring (S_prev, R_prev, v2dt2, IMG) with
// TMA; the source warps hand S_new of each plane to the receiver warps through a shared-memory
// exchange ring with its own full/empty mbarriers.  Merged (dual_merged_kernel, variants 4-7, the
// default): every consumer thread steps both wavefields at its four points, so S_new stays in its
// registers.  Every wait is bounded, as in the single-wavefield kernel.
#pragma once
#include "stencil_tma_impl.cuh"

namespace rtmb {
namespace detail {

constexpr int kDTY = 8;                        // tile rows (y) of the default variant
constexpr int kGThreads = (kTZ / kVZ) * kDTY;  // consumer threads per wavefield: 128
constexpr int kDualThreads = 2 * kGThreads + 32;

// Launch variants of the dual step (StepArgs::variant of the receiver arguments, picked by
// rtmb_autotune_full): the in-plane tile, 128 consumer threads per wavefield in all, and the ring
// depths (DX: P slots beyond H; R: core slots; E: exchange slots).
//   0: 64 (z) x 8 (y); 1: 32 x 16 (a 40 x 24 halo tile for 512 points instead of 72 x 16, and
//   z tiles of 32 cells, which waste less of a row whose length is not a multiple of 64);
//   2: 32 x 16 with P rings two planes deeper and a fourth exchange slot; 3: 32 x 16 with P rings
//   one plane deeper, a fourth core slot and a fourth exchange slot (2 and 3: 108 KB of shared
//   memory, still two CTAs per SM); 4 to 7: the merged form (below)
template <int DV>
struct DualTile;
template <>
struct DualTile<0> {
    static constexpr int TZ = 64, TY = 8, DX = 4, R = 3, E = 3;
};
template <>
struct DualTile<1> {
    static constexpr int TZ = 32, TY = 16, DX = 4, R = 3, E = 3;
};
template <>
struct DualTile<2> {
    static constexpr int TZ = 32, TY = 16, DX = 6, R = 3, E = 4;
};
template <>
struct DualTile<3> {
    static constexpr int TZ = 32, TY = 16, DX = 5, R = 4, E = 4;
};
// 4 and 5: the merged form (dual_merged_kernel): every consumer thread steps both wavefields at its
// four points, so S_new stays in registers for the image (no exchange ring); 64 x 8 and 32 x 16
template <>
struct DualTile<4> {
    static constexpr int TZ = 64, TY = 8, DX = 4, R = 3, E = 0;
};
template <>
struct DualTile<5> {
    static constexpr int TZ = 32, TY = 16, DX = 4, R = 3, E = 0;
};
// 6 and 7: the merged form on 64 x 16 and 32 x 32 tiles, 256 consumer threads, one CTA per SM
// (fewer halo cells per point: 72 x 24 and 40 x 40 tiles for 1024 points)
template <>
struct DualTile<6> {
    static constexpr int TZ = 64, TY = 16, DX = 4, R = 3, E = 0;
};
template <>
struct DualTile<7> {
    static constexpr int TZ = 32, TY = 32, DX = 4, R = 3, E = 0;
};

struct DualMaps {
    CUtensorMap ps, pr;            // halo boxes of S and R
    CUtensorMap pps, ppr, v, img;  // core boxes
};

struct DualArgs {
    StepArgs s;  // the source step (no taper)
    StepArgs r;  // the receiver step (receiver injection, image; no taper)
};

template <int H, int DV = 0>
struct DualShape {
    static constexpr int TZ = DualTile<DV>::TZ, TY = DualTile<DV>::TY;
    static_assert((TZ / kVZ) * TY == kGThreads || DV >= 6, "128 consumer threads per wavefield");
    static constexpr int MT = (TZ / kVZ) * TY;  // consumer threads of the merged form
    static constexpr int ZH = ((H + 3) / 4) * 4;
    static constexpr int SROWS = TY + 2 * H;
    static constexpr int SPITCH = TZ + 2 * ZH;
    static constexpr int STAGE = SROWS * SPITCH;
    static constexpr int STRIDE = ((STAGE + 31) / 32) * 32;  // 128-byte slots
    static constexpr int CORE = TZ * TY;
    static constexpr int OFF_PPR = CORE * 4, OFF_V = 2 * CORE * 4, OFF_IMG = 3 * CORE * 4, CSLOT = 4 * CORE * 4;
    static constexpr int D = H + DualTile<DV>::DX, R = DualTile<DV>::R, E = DualTile<DV>::E;
    static_assert(2 * H <= D, "warm-up planes must fit in the P rings");
    static constexpr size_t RING_BYTES = (size_t)D * STRIDE * 4;
    static constexpr size_t XOFF = 2 * RING_BYTES + (size_t)R * CSLOT;  // exchange slots
    static constexpr size_t BOFF = XOFF + (size_t)E * CORE * 4;         // barriers
    static constexpr size_t SMEM = BOFF + (size_t)(4 * D + 2 * R + 2 * E) * sizeof(uint64_t);
    static_assert(SMEM <= (DV >= 6 ? 227 : 113) * 1024, "two CTAs per SM (one for variants 6 and 7)");
};

// One wavefield's consumer warps.  ROLE 0: source (S), ROLE 1: receiver (R) with the image.
template <int H, bool EXACT, int TAPER, int ROLE, int DV = 0>
__device__ __forceinline__ void dual_consumer(const StepArgs &a, const StepArgs &coef, const float *pring,
                                              const unsigned char *cring, float *xring, uint64_t *pfull,
                                              uint64_t *pempty, uint64_t *cfull, uint64_t *cempty, uint64_t *xfull,
                                              uint64_t *xempty, int tid, int zt0, int yt0, int xc0, int n) {
    using S = DualShape<H, DV>;
    constexpr int kTZ = S::TZ;  // this variant's tile width (z)
    constexpr int ZH = S::ZH, SPITCH = S::SPITCH, STRIDE = S::STRIDE, D = S::D, R = S::R,
                  E = S::E, CSLOT = S::CSLOT, CORE = S::CORE;
    constexpr int NQ = 2 * H + 1;
    constexpr int ZQ = kTZ / kVZ;
    constexpr bool RCV = ROLE == 1;
    static_assert(TAPER == kTaperNone, "the dual step has no taper form (HBC runs two launches)");
    const int lane = tid & 31;
    const int tz = tid % ZQ, ty = tid / ZQ;
    const int z0 = zt0 + tz * kVZ;
    const int y = yt0 + ty;
    const size_t plane = (size_t)a.nye * a.nze;

    const bool row_ok = y < a.nye && z0 < a.nze;
    const bool y_ok = y < a.nye - H;
    unsigned vmask = 0, imask = 0, umask = 0;
#pragma unroll
    for (int e = 0; e < kVZ; ++e) {
        const int z = z0 + e;
        const bool v = y_ok && z >= H && z < a.nze - H;
        if (v) vmask |= 1u << e;
        if (v && RCV && z >= a.img_z0 && z < a.img_z1) imask |= 1u << e;
        if (v && a.upb_mode != kUpbNone && z >= a.blen - H && z < a.blen) umask |= 1u << e;
    }
    int rec_e = -1, rec_j = 0;
    if (RCV && a.rec_mode != kRecNone && a.rz >= z0 && a.rz < z0 + kVZ && ((vmask >> (a.rz - z0)) & 1u)) {
        const int dyr = y - a.ry0;
        if (dyr >= 0 && dyr % a.rdy == 0 && dyr / a.rdy < a.rcy) {
            rec_e = a.rz - z0;
            rec_j = dyr / a.rdy;
        }
    }
    const bool special = rec_e >= 0 || umask != 0;
    const size_t row_off = (size_t)y * a.nze + z0;
    float *PPp = a.PP + row_off;
    const int col = ZH + tz * kVZ;
    const int ccol = ty * kTZ + tz * kVZ;

    bool bad_wait = false;
    auto wait_p = [&](int slot, int parity) {
        bad_wait |= !__all_sync(0xffffffffu, mbar_wait(&pfull[slot], parity));
    };
    auto release = [&](uint64_t *bar) {
        __syncwarp();
        if (lane == 0) mbar_arrive(bar);
    };

    float4 q[NQ];
    float nanacc = 0.f;
    // the single-wavefield kernel's packed symmetric form for isotropic grids (same rounding)
    const bool iso = !EXACT && a.iso;
    f32x2 cpk[H + 1];
    cpk[0] = pk2(coef.cx[H] + coef.cy[H] + coef.cz[H], coef.cx[H] + coef.cy[H] + coef.cz[H]);
#pragma unroll
    for (int k = 1; k <= H; ++k) cpk[k] = pk2(coef.cx[H + k], coef.cx[H + k]);
    int s_in = (2 * H) % D, ph_in = ((2 * H) / D) & 1, s_mid = H % D, s_core = 0, ph_core = 0, s_x = 0, ph_x = 0;
    for (int k = 0; k < 2 * H; ++k) {
        wait_p(k, 0);
    }
    if (bad_wait) goto drain;
#pragma unroll
    for (int k = 0; k < 2 * H; ++k) q[k + 1] = ld_f4(pring + k * STRIDE + (ty + H) * SPITCH + col);
#pragma unroll
    for (int k = 0; k < H; ++k) release(&pempty[k]);

RTMB_UNROLL_PRAGMA(RTMB_DUAL_UNROLL)
    for (int i = 0; i < n; ++i, s_in = s_in + 1 == D ? (ph_in ^= 1, 0) : s_in + 1, s_mid = s_mid + 1 == D ? 0 : s_mid + 1,
                           s_core = s_core + 1 == R ? (ph_core ^= 1, 0) : s_core + 1,
                           s_x = s_x + 1 == E ? (ph_x ^= 1, 0) : s_x + 1) {
        const int x = xc0 + i;
        // the record value this plane injects, loaded now so that its latency overlaps the stencil
        const float *rec_p = nullptr;
        float rec_v = 0.f;
        if (RCV && rec_e >= 0) {
            const int dxr = x - a.rx0;
            if (dxr >= 0 && dxr % a.rdx == 0 && dxr / a.rdx < a.rcx) {
                rec_p = a.rec + a.rec_base + (dxr / a.rdx) * a.rec_si + rec_j * a.rec_sj;
                rec_v = __ldg(rec_p);
            }
        }
        wait_p(s_in, ph_in);
        const float *s = pring + s_mid * STRIDE;
        if (bad_wait) goto drain;
#pragma unroll
        for (int k = 0; k < NQ - 1; ++k) q[k] = q[k + 1];
        q[NQ - 1] = ld_f4(pring + s_in * STRIDE + (ty + H) * SPITCH + col);

        float lap[kVZ] = {0.f, 0.f, 0.f, 0.f};
        if (row_ok) {
            float zr[kVZ + 2 * ZH];
#pragma unroll
            for (int k = 0; k < (kVZ + 2 * ZH) / 4; ++k) {
                const float4 t4 = (k == ZH / 4) ? q[H] : ld_f4(s + (ty + H) * SPITCH + col - ZH + 4 * k);
                zr[4 * k + 0] = t4.x; zr[4 * k + 1] = t4.y; zr[4 * k + 2] = t4.z; zr[4 * k + 3] = t4.w;
            }
            if (EXACT) {
                float ax[kVZ], ay[kVZ], az[kVZ];
#pragma unroll
                for (int e = 0; e < kVZ; ++e) { ax[e] = 0.f; ay[e] = 0.f; az[e] = 0.f; }
#pragma unroll
                for (int io = 0; io < NQ; ++io) {
                    const float4 qx = q[io];
                    const float4 ry = (io == H) ? q[H] : ld_f4(s + (ty + io) * SPITCH + col);
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
                const float4 qc = q[H];
                f32x2 l0 = mul2(pk2(qc.x, qc.y), cpk[0]), l1 = mul2(pk2(qc.z, qc.w), cpk[0]);
#pragma unroll
                for (int k = 1; k <= H; ++k) {
                    const float4 xa = q[H + k], xb = q[H - k];
                    const float4 ya = ld_f4(s + (ty + H + k) * SPITCH + col);
                    const float4 yb = ld_f4(s + (ty + H - k) * SPITCH + col);
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
                    const float4 ry = ld_f4(s + (ty + io) * SPITCH + col);
#pragma unroll
                    for (int e = 0; e < kVZ; ++e) {
                        lap[e] = fmaf(get(qx, e), coef.cx[io], lap[e]);
                        lap[e] = fmaf(get(ry, e), coef.cy[io], lap[e]);
                        lap[e] = fmaf(zr[ZH - H + e + io], coef.cz[io], lap[e]);
                    }
                }
            }
        }
        release(&pempty[s_mid]);
        // core tiles of plane x
        if (!__all_sync(0xffffffffu, mbar_wait(&cfull[s_core], ph_core))) {
            bad_wait = true;
            goto drain;
        }
        const unsigned char *ct = cring + s_core * CSLOT;
        const float4 pp_raw = ld_f4(reinterpret_cast<const float *>(ct + (RCV ? S::OFF_PPR : 0)) + ccol);
        const float4 vv = ld_f4(reinterpret_cast<const float *>(ct + S::OFF_V) + ccol);
        float4 im4 = pp_raw;
        if (RCV) im4 = ld_f4(reinterpret_cast<const float *>(ct + S::OFF_IMG) + ccol);
        release(&cempty[s_core]);
        // the exchange slot of plane x: the source warps fill it, the receiver warps read it
        if (!__all_sync(0xffffffffu, mbar_wait(RCV ? &xfull[s_x] : &xempty[s_x], RCV ? ph_x : (ph_x ^ 1)))) {
            bad_wait = true;
            goto drain;
        }
        float4 ps4 = pp_raw;
        if (RCV) ps4 = ld_f4(xring + s_x * CORE + ccol);
        if (RCV) release(&xempty[s_x]);
        float4 out = pp_raw;
        if (row_ok) {
            const float4 qc = q[H];
            float ppv[kVZ] = {pp_raw.x, pp_raw.y, pp_raw.z, pp_raw.w};
            float npp[kVZ];
#pragma unroll
            for (int e = 0; e < kVZ; ++e) {
                if (EXACT) {
                    const float two_p = 2.f * get(qc, e);
                    const float d = two_p - ppv[e];
                    const float vl = get(vv, e) * lap[e];
                    npp[e] = d + vl;
                } else {
                    npp[e] = fmaf(get(vv, e), lap[e], 2.f * get(qc, e) - ppv[e]);
                }
            }
            if (special) {
#pragma unroll
                for (int e = 0; e < kVZ; ++e) {
                    const int z = z0 + e;
                    if (RCV && e == rec_e && rec_p) {
                        if (a.rec_mode == kRecOverwrite) npp[e] = rec_v;
                        else npp[e] = npp[e] + rec_v;
                    }
                    if (!RCV && ((umask >> e) & 1u) && a.upb_mode == kUpbRestore)
                        npp[e] = a.upb[((size_t)x * a.nye + y) * H + (z - (a.blen - H))];
                }
            }
#pragma unroll
            for (int e = 0; e < kVZ; ++e) {
                const float o = ((vmask >> e) & 1u) ? npp[e] : get(pp_raw, e);
                put(out, e, o);
                nanacc = fmaf(0.f, o, nanacc);
            }
            *reinterpret_cast<float4 *>(PPp + (size_t)x * plane) = out;
            if (RCV && imask) {
                float4 im;
#pragma unroll
                for (int e = 0; e < kVZ; ++e) {
                    const float acc = get(im4, e) + get(ps4, e) * get(out, e);
                    put(im, e, ((imask >> e) & 1u) ? acc : get(im4, e));
                }
                *reinterpret_cast<float4 *>(a.img + row_off + (size_t)x * plane) = im;
            }
        }
        if (!RCV) {
            // S_new of this plane for the receiver warps (cells outside the computed region carry
            // S_prev, which the image never reads)
            *reinterpret_cast<float4 *>(xring + s_x * CORE + ccol) = out;
            release(&xfull[s_x]);
        }
    }
    if (nanacc != nanacc && a.err) atomicOr(a.err, 1u);
    if (bad_wait && a.err) atomicOr(a.err, 2u);
    return;
drain:
    if (a.err) atomicOr(a.err, 2u);
}

template <int H, bool EXACT, int TAPER, int DV = 0>
__global__ void __launch_bounds__(kDualThreads, 2)
    dual_step_kernel(const __grid_constant__ DualMaps maps, const __grid_constant__ DualArgs d) {
    using S = DualShape<H, DV>;
    constexpr int kTZ = S::TZ, kDTY = S::TY;
    constexpr int ZH = S::ZH, STAGE = S::STAGE, STRIDE = S::STRIDE, D = S::D, R = S::R, E = S::E, CSLOT = S::CSLOT;
    extern __shared__ __align__(128) unsigned char smem[];
    float *ring_s = reinterpret_cast<float *>(smem);
    float *ring_r = ring_s + D * STRIDE;
    unsigned char *cring = smem + 2 * S::RING_BYTES;
    float *xring = reinterpret_cast<float *>(smem + S::XOFF);
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem + S::BOFF);
    uint64_t *pfull_s = bars, *pfull_r = pfull_s + D, *pempty_s = pfull_r + D, *pempty_r = pempty_s + D;
    uint64_t *cfull = pempty_r + D, *cempty = cfull + R, *xfull = cempty + R, *xempty = xfull + E;
    const StepArgs &a = d.r;  // geometry (both wavefields share it)

    const int tid = threadIdx.x;
    const int zt0 = blockIdx.x * kTZ;
    const int yt0 = H + blockIdx.y * kDTY;
    const int xc0 = H + blockIdx.z * a.chunk;
    const int xc1 = min(xc0 + a.chunk, a.nxe - H);
    if (xc0 >= xc1) return;
    const int n = xc1 - xc0;
    const int nplanes = n + 2 * H;
    if (tid == 0) {
        for (int s = 0; s < D; ++s) {
            mbar_init(&pfull_s[s], 1); mbar_init(&pfull_r[s], 1);
            mbar_init(&pempty_s[s], kGThreads / 32); mbar_init(&pempty_r[s], kGThreads / 32);
        }
        for (int s = 0; s < R; ++s) { mbar_init(&cfull[s], 1); mbar_init(&cempty[s], 2 * kGThreads / 32); }
        for (int s = 0; s < E; ++s) { mbar_init(&xfull[s], kGThreads / 32); mbar_init(&xempty[s], kGThreads / 32); }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    if (tid >= 2 * kGThreads) {
        // producer: S and R planes k, then the core tiles of output plane k - 2H
        if (tid != 2 * kGThreads) return;
        bool ok = true;
        int p_issued = 0, c_issued = 0;
        for (int k = 0; k < nplanes && ok; ++k) {
            const int s = k % D;
            if (k >= D && (!(ok = mbar_wait_producer(&pempty_s[s], ((k / D) + 1) & 1)) ||
                           !(ok = mbar_wait_producer(&pempty_r[s], ((k / D) + 1) & 1))))
                break;
            mbar_expect_tx(&pfull_s[s], STAGE * 4);
            tma_load_3d(ring_s + s * STRIDE, &maps.ps, &pfull_s[s], zt0 - ZH, yt0 - H, xc0 - H + k);
            mbar_expect_tx(&pfull_r[s], STAGE * 4);
            tma_load_3d(ring_r + s * STRIDE, &maps.pr, &pfull_r[s], zt0 - ZH, yt0 - H, xc0 - H + k);
            p_issued = k + 1;
            if (k >= 2 * H) {
                const int i = k - 2 * H, cs = i % R;
                if (i >= R && !(ok = mbar_wait_producer(&cempty[cs], ((i / R) + 1) & 1))) break;
                unsigned char *dst = cring + cs * CSLOT;
                mbar_expect_tx(&cfull[cs], CSLOT);
                tma_load_3d(dst, &maps.pps, &cfull[cs], zt0, yt0, xc0 + i);
                tma_load_3d(dst + S::OFF_PPR, &maps.ppr, &cfull[cs], zt0, yt0, xc0 + i);
                tma_load_3d(dst + S::OFF_V, &maps.v, &cfull[cs], zt0, yt0, xc0 + i);
                tma_load_3d(dst + S::OFF_IMG, &maps.img, &cfull[cs], zt0, yt0, xc0 + i);
                c_issued = i + 1;
            }
        }
        if (!ok && a.err) atomicOr(a.err, 2u);
        // stay until every copy this CTA issued has landed (bounded), so none outlives the CTA
        for (int k = p_issued > D ? p_issued - D : 0; k < p_issued; ++k) {
            if (!mbar_wait_producer(&pfull_s[k % D], (k / D) & 1)) break;
            if (!mbar_wait_producer(&pfull_r[k % D], (k / D) & 1)) break;
        }
        for (int i = c_issued > R ? c_issued - R : 0; i < c_issued; ++i)
            if (!mbar_wait_producer(&cfull[i % R], (i / R) & 1)) break;
        return;
    }
    if (tid < kGThreads)
        dual_consumer<H, EXACT, TAPER, 0, DV>(d.s, d.r, ring_s, cring, xring, pfull_s, pempty_s, cfull, cempty, xfull,
                                              xempty, tid, zt0, yt0, xc0, n);
    else
        dual_consumer<H, EXACT, TAPER, 1, DV>(d.r, d.r, ring_r, cring, xring, pfull_r, pempty_r, cfull, cempty, xfull,
                                              xempty, tid - kGThreads, zt0, yt0, xc0, n);
}

// ---- merged form (variants 4 to 7): one consumer thread per four points of BOTH wavefields.
// Four consumer warps and a producer warp per CTA (160 threads, two CTAs per SM) on 64 x 8 and
// 32 x 16 tiles; eight consumer warps (288 threads, one CTA per SM) on 64 x 16 and 32 x 32 tiles.  The producer loads
// the S and R halo tiles of a plane onto one "full" barrier and the core tiles (S_prev, R_prev,
// v2dt2, IMG) as in the split form.  Per point the arithmetic is the split form's, operation for
// operation, so the results are bit-identical to it and to the two single-wavefield launches; what
// goes away is the exchange ring (S_new stays in the thread's registers for the image), the second
// set of ring waits, loop and address work per plane, and the second read of v2dt2 from shared memory.
template <int DV>
constexpr int merged_threads() { return (DualTile<DV>::TZ / kVZ) * DualTile<DV>::TY + 32; }
// unroll factor of the merged form's plane loop (compile-time tuning; 2 and 3 measured within noise
// of 1 on the 512^3 shot, at 150 registers either way)
#ifndef RTMB_MERGED_UNROLL
#define RTMB_MERGED_UNROLL 1
#endif

// lap of this thread's four points from the centre tile s and the x queue q (the split form's
// arithmetic: exact, packed symmetric for isotropic FMA grids, or the FMA chain).
template <int H, bool EXACT, int ZH, int SPITCH>
__device__ __forceinline__ void dual_lap(const float *s, const float4 *q, int ty, int col, bool iso, const f32x2 *cpk,
                                         const StepArgs &coef, float lap[kVZ]) {
    constexpr int NQ = 2 * H + 1;
    float zr[kVZ + 2 * ZH];
#pragma unroll
    for (int k = 0; k < (kVZ + 2 * ZH) / 4; ++k) {
        const float4 t4 = (k == ZH / 4) ? q[H] : ld_f4(s + (ty + H) * SPITCH + col - ZH + 4 * k);
        zr[4 * k + 0] = t4.x; zr[4 * k + 1] = t4.y; zr[4 * k + 2] = t4.z; zr[4 * k + 3] = t4.w;
    }
    if (EXACT) {
        float ax[kVZ], ay[kVZ], az[kVZ];
#pragma unroll
        for (int e = 0; e < kVZ; ++e) { ax[e] = 0.f; ay[e] = 0.f; az[e] = 0.f; }
#pragma unroll
        for (int io = 0; io < NQ; ++io) {
            const float4 qx = q[io];
            const float4 ry = (io == H) ? q[H] : ld_f4(s + (ty + io) * SPITCH + col);
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
        const float4 qc = q[H];
        f32x2 l0 = mul2(pk2(qc.x, qc.y), cpk[0]), l1 = mul2(pk2(qc.z, qc.w), cpk[0]);
#pragma unroll
        for (int k = 1; k <= H; ++k) {
            const float4 xa = q[H + k], xb = q[H - k];
            const float4 ya = ld_f4(s + (ty + H + k) * SPITCH + col);
            const float4 yb = ld_f4(s + (ty + H - k) * SPITCH + col);
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
            const float4 ry = ld_f4(s + (ty + io) * SPITCH + col);
#pragma unroll
            for (int e = 0; e < kVZ; ++e) {
                lap[e] = fmaf(get(qx, e), coef.cx[io], lap[e]);
                lap[e] = fmaf(get(ry, e), coef.cy[io], lap[e]);
                lap[e] = fmaf(zr[ZH - H + e + io], coef.cz[io], lap[e]);
            }
        }
    }
}

template <int H, bool EXACT, int DV>
__device__ __forceinline__ void dual_merged_consumer(const StepArgs &as, const StepArgs &a, const float *ring_s,
                                                     const float *ring_r, const unsigned char *cring, uint64_t *pfull,
                                                     uint64_t *pempty, uint64_t *cfull, uint64_t *cempty, int tid,
                                                     int zt0, int yt0, int xc0, int n) {
    using S = DualShape<H, DV>;
    constexpr int kTZ = S::TZ;
    constexpr int ZH = S::ZH, SPITCH = S::SPITCH, STRIDE = S::STRIDE, D = S::D, R = S::R, CSLOT = S::CSLOT;
    constexpr int NQ = 2 * H + 1;
    constexpr int ZQ = kTZ / kVZ;
    const int lane = tid & 31;
    const int tz = tid % ZQ, ty = tid / ZQ;
    const int z0 = zt0 + tz * kVZ;
    const int y = yt0 + ty;
    const size_t plane = (size_t)a.nye * a.nze;

    const bool row_ok = y < a.nye && z0 < a.nze;
    const bool y_ok = y < a.nye - H;
    unsigned vmask = 0, imask = 0;
#pragma unroll
    for (int e = 0; e < kVZ; ++e) {
        const int z = z0 + e;
        const bool v = y_ok && z >= H && z < a.nze - H;
        if (v) vmask |= 1u << e;
        if (v && z >= a.img_z0 && z < a.img_z1) imask |= 1u << e;
    }
    int rec_e = -1, rec_j = 0;
    if (a.rec_mode != kRecNone && a.rz >= z0 && a.rz < z0 + kVZ && ((vmask >> (a.rz - z0)) & 1u)) {
        const int dyr = y - a.ry0;
        if (dyr >= 0 && dyr % a.rdy == 0 && dyr / a.rdy < a.rcy) {
            rec_e = a.rz - z0;
            rec_j = dyr / a.rdy;
        }
    }
    const size_t row_off = (size_t)y * a.nze + z0;
    const bool img_io = a.img_pair != 1;  // this launch reads and writes the image
    float *PPs = as.PP + row_off;
    float *PPr = a.PP + row_off;
    const int col = ZH + tz * kVZ;
    const int ccol = ty * kTZ + tz * kVZ;

    bool bad_wait = false;
    auto wait_p = [&](int slot, int parity) {
        bad_wait |= !__all_sync(0xffffffffu, mbar_wait(&pfull[slot], parity));
    };
    auto release = [&](uint64_t *bar) {
        __syncwarp();
        if (lane == 0) mbar_arrive(bar);
    };

    float4 qs[NQ], qr[NQ];
    float nanacc = 0.f;
    const bool iso = !EXACT && a.iso;
    f32x2 cpk[H + 1];
    cpk[0] = pk2(a.cx[H] + a.cy[H] + a.cz[H], a.cx[H] + a.cy[H] + a.cz[H]);
#pragma unroll
    for (int k = 1; k <= H; ++k) cpk[k] = pk2(a.cx[H + k], a.cx[H + k]);
    int s_in = (2 * H) % D, ph_in = ((2 * H) / D) & 1, s_mid = H % D, s_core = 0, ph_core = 0;
    for (int k = 0; k < 2 * H; ++k) wait_p(k, 0);
    if (bad_wait) goto drain;
#pragma unroll
    for (int k = 0; k < 2 * H; ++k) {
        qs[k + 1] = ld_f4(ring_s + k * STRIDE + (ty + H) * SPITCH + col);
        qr[k + 1] = ld_f4(ring_r + k * STRIDE + (ty + H) * SPITCH + col);
    }
#pragma unroll
    for (int k = 0; k < H; ++k) release(&pempty[k]);

RTMB_UNROLL_PRAGMA(RTMB_MERGED_UNROLL)
    for (int i = 0; i < n; ++i, s_in = s_in + 1 == D ? (ph_in ^= 1, 0) : s_in + 1, s_mid = s_mid + 1 == D ? 0 : s_mid + 1,
                           s_core = s_core + 1 == R ? (ph_core ^= 1, 0) : s_core + 1) {
        const int x = xc0 + i;
        // the record value this plane injects, loaded now so that its latency overlaps the stencils
        const float *rec_p = nullptr;
        float rec_v = 0.f;
        if (rec_e >= 0) {
            const int dxr = x - a.rx0;
            if (dxr >= 0 && dxr % a.rdx == 0 && dxr / a.rdx < a.rcx) {
                rec_p = a.rec + a.rec_base + (dxr / a.rdx) * a.rec_si + rec_j * a.rec_sj;
                rec_v = __ldg(rec_p);
            }
        }
        wait_p(s_in, ph_in);
        if (bad_wait) goto drain;
#pragma unroll
        for (int k = 0; k < NQ - 1; ++k) { qs[k] = qs[k + 1]; qr[k] = qr[k + 1]; }
        qs[NQ - 1] = ld_f4(ring_s + s_in * STRIDE + (ty + H) * SPITCH + col);
        qr[NQ - 1] = ld_f4(ring_r + s_in * STRIDE + (ty + H) * SPITCH + col);

        float lap_s[kVZ] = {0.f, 0.f, 0.f, 0.f}, lap_r[kVZ] = {0.f, 0.f, 0.f, 0.f};
        if (row_ok) {
            dual_lap<H, EXACT, ZH, SPITCH>(ring_s + s_mid * STRIDE, qs, ty, col, iso, cpk, a, lap_s);
            dual_lap<H, EXACT, ZH, SPITCH>(ring_r + s_mid * STRIDE, qr, ty, col, iso, cpk, a, lap_r);
        }
        release(&pempty[s_mid]);
        if (!__all_sync(0xffffffffu, mbar_wait(&cfull[s_core], ph_core))) {
            bad_wait = true;
            goto drain;
        }
        const unsigned char *ct = cring + s_core * CSLOT;
        const float4 pps = ld_f4(reinterpret_cast<const float *>(ct) + ccol);
        const float4 ppr = ld_f4(reinterpret_cast<const float *>(ct + S::OFF_PPR) + ccol);
        const float4 vv = ld_f4(reinterpret_cast<const float *>(ct + S::OFF_V) + ccol);
        float4 im4 = vv;
        if (img_io) im4 = ld_f4(reinterpret_cast<const float *>(ct + S::OFF_IMG) + ccol);
        release(&cempty[s_core]);
        if (row_ok) {
            const float4 qcs = qs[H], qcr = qr[H];
            float4 outs, outr;
#pragma unroll
            for (int e = 0; e < kVZ; ++e) {
                const bool v = (vmask >> e) & 1u;
                const float ns = step_update<EXACT>(get(vv, e), lap_s[e], get(qcs, e), get(pps, e));
                float nr = step_update<EXACT>(get(vv, e), lap_r[e], get(qcr, e), get(ppr, e));
                if (e == rec_e && rec_p) nr = a.rec_mode == kRecOverwrite ? rec_v : nr + rec_v;
                const float os = v ? ns : get(pps, e);
                const float orr = v ? nr : get(ppr, e);
                put(outs, e, os);
                put(outr, e, orr);
                nanacc = fmaf(0.f, os, nanacc);
                nanacc = fmaf(0.f, orr, nanacc);
            }
            *reinterpret_cast<float4 *>(PPs + (size_t)x * plane) = outs;
            *reinterpret_cast<float4 *>(PPr + (size_t)x * plane) = outr;
            if (imask && img_io) {
                float4 im;
                const float4 pcs = qs[H], pcr = qr[H];  // this step's input levels: the previous step's output
#pragma unroll
                for (int e = 0; e < kVZ; ++e) {
                    float acc = get(im4, e);
                    if (a.img_pair == 2) acc = acc + get(pcs, e) * get(pcr, e);
                    acc = acc + get(outs, e) * get(outr, e);
                    put(im, e, ((imask >> e) & 1u) ? acc : get(im4, e));
                }
                *reinterpret_cast<float4 *>(a.img + row_off + (size_t)x * plane) = im;
            }
        }
    }
    if (nanacc != nanacc && a.err) atomicOr(a.err, 1u);
    if (bad_wait && a.err) atomicOr(a.err, 2u);
    return;
drain:
    if (a.err) atomicOr(a.err, 2u);
}

template <int H, bool EXACT, int DV>
__global__ void __launch_bounds__((DualTile<DV>::TZ / kVZ) * DualTile<DV>::TY + 32, DV >= 6 ? 1 : 2)
    dual_merged_kernel(const __grid_constant__ DualMaps maps, const __grid_constant__ DualArgs d) {
    using S = DualShape<H, DV>;
    static_assert(DV >= 4, "merged variants only");
    constexpr int kTZ = S::TZ, kDTY2 = S::TY;
    constexpr int ZH = S::ZH, STAGE = S::STAGE, STRIDE = S::STRIDE, D = S::D, R = S::R, CSLOT = S::CSLOT;
    constexpr int MT = S::MT;
    extern __shared__ __align__(128) unsigned char smem[];
    float *ring_s = reinterpret_cast<float *>(smem);
    float *ring_r = ring_s + D * STRIDE;
    unsigned char *cring = smem + 2 * S::RING_BYTES;
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem + S::BOFF);
    uint64_t *pfull = bars, *pempty = pfull + D, *cfull = pempty + D, *cempty = cfull + R;
    const StepArgs &a = d.r;  // geometry (both wavefields share it)

    const int tid = threadIdx.x;
    const int zt0 = blockIdx.x * kTZ;
    const int yt0 = H + blockIdx.y * kDTY2;
    const int xc0 = H + blockIdx.z * a.chunk;
    const int xc1 = min(xc0 + a.chunk, a.nxe - H);
    if (xc0 >= xc1) return;
    const int n = xc1 - xc0;
    const int nplanes = n + 2 * H;
    if (tid == 0) {
        for (int s = 0; s < D; ++s) { mbar_init(&pfull[s], 1); mbar_init(&pempty[s], MT / 32); }
        for (int s = 0; s < R; ++s) { mbar_init(&cfull[s], 1); mbar_init(&cempty[s], MT / 32); }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    const bool img_io = a.img_pair != 1;  // this launch reads and writes the image
    if (tid >= MT) {
        // producer: the S and R planes k onto one barrier, then the core tiles of output plane k - 2H
        if (tid != MT) return;
        bool ok = true;
        int p_issued = 0, c_issued = 0;
        for (int k = 0; k < nplanes && ok; ++k) {
            const int s = k % D;
            if (k >= D && !(ok = mbar_wait_producer(&pempty[s], ((k / D) + 1) & 1))) break;
            mbar_expect_tx(&pfull[s], 2 * STAGE * 4);
            tma_load_3d(ring_s + s * STRIDE, &maps.ps, &pfull[s], zt0 - ZH, yt0 - H, xc0 - H + k);
            tma_load_3d(ring_r + s * STRIDE, &maps.pr, &pfull[s], zt0 - ZH, yt0 - H, xc0 - H + k);
            p_issued = k + 1;
            if (k >= 2 * H) {
                const int i = k - 2 * H, cs = i % R;
                if (i >= R && !(ok = mbar_wait_producer(&cempty[cs], ((i / R) + 1) & 1))) break;
                unsigned char *dst = cring + cs * CSLOT;
                mbar_expect_tx(&cfull[cs], img_io ? CSLOT : S::OFF_IMG);
                tma_load_3d(dst, &maps.pps, &cfull[cs], zt0, yt0, xc0 + i);
                tma_load_3d(dst + S::OFF_PPR, &maps.ppr, &cfull[cs], zt0, yt0, xc0 + i);
                tma_load_3d(dst + S::OFF_V, &maps.v, &cfull[cs], zt0, yt0, xc0 + i);
                if (img_io) tma_load_3d(dst + S::OFF_IMG, &maps.img, &cfull[cs], zt0, yt0, xc0 + i);
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
    dual_merged_consumer<H, EXACT, DV>(d.s, d.r, ring_s, ring_r, cring, pfull, pempty, cfull, cempty, tid, zt0, yt0,
                                       xc0, n);
}

template <int H>
cudaError_t launch_dual_h(const DualMaps &maps, const DualArgs &d, bool exact, int taper, int dv, dim3 grid,
                          cudaStream_t s) {
    static unsigned long long attr_done[2 * kDualVariants] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dv < 0 || dv >= kDualVariants) return cudaErrorInvalidValue;
    const int variant = 2 * dv + (exact ? 1 : 0);
    auto run = [&](void (*kern)(DualMaps, DualArgs), size_t smem) -> cudaError_t {
        const unsigned long long bit = 1ull << (dev & 63);
        if (!(attr_done[variant] & bit)) {
            cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (e != cudaSuccess) return e;
            attr_done[variant] |= bit;
        }
        kern<<<grid, kDualThreads, smem, s>>>(maps, d);
        return cudaGetLastError();
    };
    if (taper != kTaperNone) return cudaErrorInvalidValue;
    auto run_merged = [&](void (*kern)(DualMaps, DualArgs), size_t smem, int threads) -> cudaError_t {
        const unsigned long long bit = 1ull << (dev & 63);
        if (!(attr_done[variant] & bit)) {
            cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (e != cudaSuccess) return e;
            attr_done[variant] |= bit;
        }
        kern<<<grid, threads, smem, s>>>(maps, d);
        return cudaGetLastError();
    };
    switch (dv) {
    case 4:
        return exact ? run_merged(dual_merged_kernel<H, true, 4>, DualShape<H, 4>::SMEM, merged_threads<4>())
                     : run_merged(dual_merged_kernel<H, false, 4>, DualShape<H, 4>::SMEM, merged_threads<4>());
    case 5:
        return exact ? run_merged(dual_merged_kernel<H, true, 5>, DualShape<H, 5>::SMEM, merged_threads<5>())
                     : run_merged(dual_merged_kernel<H, false, 5>, DualShape<H, 5>::SMEM, merged_threads<5>());
    case 6:
        return exact ? run_merged(dual_merged_kernel<H, true, 6>, DualShape<H, 6>::SMEM, merged_threads<6>())
                     : run_merged(dual_merged_kernel<H, false, 6>, DualShape<H, 6>::SMEM, merged_threads<6>());
    case 7:
        return exact ? run_merged(dual_merged_kernel<H, true, 7>, DualShape<H, 7>::SMEM, merged_threads<7>())
                     : run_merged(dual_merged_kernel<H, false, 7>, DualShape<H, 7>::SMEM, merged_threads<7>());
    case 1:
        return exact ? run(dual_step_kernel<H, true, kTaperNone, 1>, DualShape<H, 1>::SMEM)
                     : run(dual_step_kernel<H, false, kTaperNone, 1>, DualShape<H, 1>::SMEM);
    case 2:
        return exact ? run(dual_step_kernel<H, true, kTaperNone, 2>, DualShape<H, 2>::SMEM)
                     : run(dual_step_kernel<H, false, kTaperNone, 2>, DualShape<H, 2>::SMEM);
    case 3:
        return exact ? run(dual_step_kernel<H, true, kTaperNone, 3>, DualShape<H, 3>::SMEM)
                     : run(dual_step_kernel<H, false, kTaperNone, 3>, DualShape<H, 3>::SMEM);
    default:
        return exact ? run(dual_step_kernel<H, true, kTaperNone>, DualShape<H>::SMEM)
                     : run(dual_step_kernel<H, false, kTaperNone>, DualShape<H>::SMEM);
    }
}

}  // namespace detail
}  // namespace rtmb
