// stencil_rows_impl.cuh -- launch variant 4 of the single-wavefield step (sm_100a, FP32, order 8):
// every consumer thread computes four z points in each of TWO adjacent y rows.
//
// The forward and backward-source steps of RBC migration (no taper, no image, no receivers, no
// upper-border save) spend most of their instructions outside the arithmetic: ring waits, the x
// queue, addressing and the epilogue checks run once per thread and plane whatever the number of
// points behind them, and the y taps of neighbouring rows are the same shared-memory rows.  Two rows
// per thread share the per-plane work and eight of the sixteen y-tap row loads (rows y-4 .. y+5
// serve both rows; the two centre rows come from the x queues).  The arithmetic per point is the
// one-row kernel's (stencil_tma_impl.cuh), operation for operation, so the results are bit-identical.
//
// CTA: four consumer warps (128 threads: 16 along z x 8 row pairs) and one producer warp on a
// 64 (z) x 16 (y) tile, two CTAs per SM; the producer fills a P ring (8 slots of the halo'd plane
// tile) and a core ring (PP and v2dt2) with TMA.  Every wait is bounded, as in the one-row kernel.
#pragma once
#include "stencil_tma_impl.cuh"

namespace rtmb {
namespace detail {

struct RowsShape {
    static constexpr int H = 4, TZ = 64, TY = 16, RY = 2;
    static constexpr int ZQ = TZ / kVZ;          // threads along z
    static constexpr int NT = ZQ * (TY / RY);    // consumer threads: 128
    static constexpr int ZH = 4;
    static constexpr int SROWS = TY + 2 * H, SPITCH = TZ + 2 * ZH;
    static constexpr int STAGE = SROWS * SPITCH;
    static constexpr int STRIDE = ((STAGE + 31) / 32) * 32;  // 128-byte slots
    static constexpr int CORE = TZ * TY;
    static constexpr int OFF_V = CORE * 4, CSLOT = 2 * CORE * 4;
    static constexpr int D = H + 4, R = 3;
    static constexpr size_t PRING_BYTES = (size_t)D * STRIDE * 4;
    static constexpr size_t SMEM = PRING_BYTES + (size_t)R * CSLOT + 2 * (D + R) * sizeof(uint64_t);
    static_assert(2 * H <= D, "warm-up planes must fit in the P ring");
    static_assert(SMEM <= 113 * 1024, "two CTAs per SM");
};
constexpr int kRowsThreads = RowsShape::NT + 32;

// lap of four z points of one row: q = the row's x queue, Y[io] = the row's y neighbours y - H + io
// (Y[H] = q[H]), zr = the row's z window.  The one-row kernel's three arithmetic forms.
template <bool EXACT>
__device__ __forceinline__ void rows_lap(const float4 (&q)[9], const float4 (&Y)[9], const float (&zr)[12], bool iso,
                                         const f32x2 *cpk, const StepArgs &coef, float lap[kVZ]) {
    constexpr int H = 4, NQ = 9, ZH = 4;
    if (EXACT) {
        float ax[kVZ], ay[kVZ], az[kVZ];
#pragma unroll
        for (int e = 0; e < kVZ; ++e) { ax[e] = 0.f; ay[e] = 0.f; az[e] = 0.f; }
#pragma unroll
        for (int io = 0; io < NQ; ++io) {
            const float4 qx = q[io];
            const float4 ry = Y[io];
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
            const float4 ya = Y[H + k], yb = Y[H - k];
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
            const float4 ry = Y[io];
#pragma unroll
            for (int e = 0; e < kVZ; ++e) {
                lap[e] = fmaf(get(qx, e), coef.cx[io], lap[e]);
                lap[e] = fmaf(get(ry, e), coef.cy[io], lap[e]);
                lap[e] = fmaf(zr[ZH - H + e + io], coef.cz[io], lap[e]);
            }
        }
    }
}

// The z window of one row (12 values around the thread's four points; the centre four are q[H]).
__device__ __forceinline__ void rows_zwin(const float *row, int col, const float4 &qc, float (&zr)[12]) {
    const float4 lo = ld_f4(row + col - 4), hi = ld_f4(row + col + 4);
    zr[0] = lo.x; zr[1] = lo.y; zr[2] = lo.z; zr[3] = lo.w;
    zr[4] = qc.x; zr[5] = qc.y; zr[6] = qc.z; zr[7] = qc.w;
    zr[8] = hi.x; zr[9] = hi.y; zr[10] = hi.z; zr[11] = hi.w;
}

// The new level of one row's four points: update, source injection, the computed-region select, the
// NaN check and the store (the one-row kernel's epilogue for the FP32 forms without taper).
template <bool EXACT>
__device__ __forceinline__ void rows_store(const StepArgs &a, const float lap[kVZ], const float4 &qc, const float4 &pp,
                                           const float4 &vv, unsigned vmask, bool src_row, int x, int z0, float *dst,
                                           float &nanacc) {
    float npp[kVZ];
#pragma unroll
    for (int e = 0; e < kVZ; ++e) npp[e] = step_update<EXACT>(get(vv, e), lap[e], get(qc, e), get(pp, e));
    if (src_row && x == a.sxe) {
#pragma unroll
        for (int e = 0; e < kVZ; ++e)
            if (z0 + e == a.sze && ((vmask >> e) & 1u)) npp[e] = npp[e] + __ldg(a.wavelet + a.it);
    }
    float4 out;
#pragma unroll
    for (int e = 0; e < kVZ; ++e) {
        const float o = ((vmask >> e) & 1u) ? npp[e] : get(pp, e);
        nanacc = fmaf(0.f, o, nanacc);
        put(out, e, o);
    }
    *reinterpret_cast<float4 *>(dst) = out;
}

template <bool EXACT>
__global__ void __launch_bounds__(kRowsThreads, 2)
    tma_rows_kernel(const __grid_constant__ TmaMaps maps, const __grid_constant__ StepArgs a) {
    using S = RowsShape;
    constexpr int H = S::H, ZH = S::ZH, SPITCH = S::SPITCH, STAGE = S::STAGE, STRIDE = S::STRIDE, D = S::D,
                  R = S::R, CSLOT = S::CSLOT, NQ = 2 * H + 1, ZQ = S::ZQ, NCW = S::NT / 32;
    extern __shared__ __align__(128) unsigned char smem[];
    float *pring = reinterpret_cast<float *>(smem);
    unsigned char *cring = smem + S::PRING_BYTES;
    uint64_t *pfull = reinterpret_cast<uint64_t *>(cring + R * CSLOT);
    uint64_t *cfull = pfull + D;
    uint64_t *pempty = cfull + R;
    uint64_t *cempty = pempty + D;

    const int tid = threadIdx.x;
    const int zt0 = blockIdx.x * S::TZ;
    const int yt0 = H + blockIdx.y * S::TY;
    int xc0 = H + blockIdx.z * a.chunk;
    int xc1 = min(xc0 + a.chunk, a.nxe - H);
    if (a.x_hi > 0) {  // 2D models: the plane x = blen only
        xc0 = max(xc0, a.x_lo);
        xc1 = min(xc1, a.x_hi);
    }
    if (xc0 >= xc1) return;
    const int n = xc1 - xc0;
    const int nplanes = n + 2 * H;
    const size_t plane = (size_t)a.nye * a.nze;
    if (tid == 0) {
        for (int s = 0; s < D; ++s) { mbar_init(&pfull[s], 1); mbar_init(&pempty[s], NCW); }
        for (int s = 0; s < R; ++s) { mbar_init(&cfull[s], 1); mbar_init(&cempty[s], NCW); }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    if (tid >= S::NT) {
        // producer: P plane k into slot k % D, then the core tiles of output plane k - 2H
        if (tid != S::NT) return;
        bool ok = true;
        int p_issued = 0, c_issued = 0;
        for (int k = 0; k < nplanes && ok; ++k) {
            const int s = k % D;
            if (k >= D && !(ok = mbar_wait_producer(&pempty[s], ((k / D) + 1) & 1))) break;
            mbar_expect_tx(&pfull[s], STAGE * 4);
            tma_load_3d(pring + s * STRIDE, &maps.p, &pfull[s], zt0 - ZH, yt0 - H, xc0 - H + k);
            p_issued = k + 1;
            if (k >= 2 * H) {
                const int i = k - 2 * H, cs = i % R;
                if (i >= R && !(ok = mbar_wait_producer(&cempty[cs], ((i / R) + 1) & 1))) break;
                unsigned char *dst = cring + cs * CSLOT;
                mbar_expect_tx(&cfull[cs], CSLOT);
                tma_load_3d(dst, &maps.pp, &cfull[cs], zt0, yt0, xc0 + i);
                tma_load_3d(dst + S::OFF_V, &maps.v, &cfull[cs], zt0, yt0, xc0 + i);
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

    // ---- consumers: rows ya = yt0 + 2 t and yb = ya + 1, z points z0 .. z0 + 3
    const int lane = tid & 31;
    const int tz = tid % ZQ, t2 = tid / ZQ;
    const int z0 = zt0 + tz * kVZ;
    const int ya = yt0 + 2 * t2, yb = ya + 1;
    const int ra = 2 * t2 + H;  // tile row of ya (yb: ra + 1)
    const bool za_ok = z0 < a.nze;
    const bool rowa_ok = ya < a.nye && za_ok, rowb_ok = yb < a.nye && za_ok;
    unsigned vma = 0, vmb = 0;
#pragma unroll
    for (int e = 0; e < kVZ; ++e) {
        const int z = z0 + e;
        const bool zv = z >= H && z < a.nze - H;
        if (zv && ya < a.nye - H) vma |= 1u << e;
        if (zv && yb < a.nye - H) vmb |= 1u << e;
    }
    const bool src_cta = a.sye >= yt0 && a.sye < yt0 + S::TY && a.sze >= zt0 && a.sze < zt0 + S::TZ;
    const bool src_a = src_cta && ya == a.sye, src_b = src_cta && yb == a.sye;
    float *PPa = a.PP + (size_t)ya * a.nze + z0;
    float *PPb = PPa + a.nze;
    const int col = ZH + tz * kVZ;
    const int ccol = 2 * t2 * S::TZ + tz * kVZ;  // row ya of a core tile (yb: + TZ)

    bool bad_wait = false;
    auto wait_p = [&](int slot, int parity) {
        bad_wait |= !__all_sync(0xffffffffu, mbar_wait(&pfull[slot], parity));
    };
    auto release = [&](uint64_t *bar) {
        __syncwarp();
        if (lane == 0) mbar_arrive(bar);
    };

    float4 qa[NQ], qb[NQ];
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
        qa[k + 1] = ld_f4(pring + k * STRIDE + ra * SPITCH + col);
        qb[k + 1] = ld_f4(pring + k * STRIDE + (ra + 1) * SPITCH + col);
    }
#pragma unroll
    for (int k = 0; k < H; ++k) release(&pempty[k]);

#pragma unroll 1
    for (int i = 0; i < n; ++i, s_in = s_in + 1 == D ? (ph_in ^= 1, 0) : s_in + 1, s_mid = s_mid + 1 == D ? 0 : s_mid + 1,
                           s_core = s_core + 1 == R ? (ph_core ^= 1, 0) : s_core + 1) {
        const int x = xc0 + i;
        wait_p(s_in, ph_in);
        if (bad_wait) goto drain;
#pragma unroll
        for (int k = 0; k < NQ - 1; ++k) { qa[k] = qa[k + 1]; qb[k] = qb[k + 1]; }
        qa[NQ - 1] = ld_f4(pring + s_in * STRIDE + ra * SPITCH + col);
        qb[NQ - 1] = ld_f4(pring + s_in * STRIDE + (ra + 1) * SPITCH + col);

        float lapa[kVZ] = {0.f, 0.f, 0.f, 0.f}, lapb[kVZ] = {0.f, 0.f, 0.f, 0.f};
        if (rowa_ok) {
            const float *s = pring + s_mid * STRIDE;
            // the y neighbours of both rows: tile rows ra - 4 .. ra + 5; ra and ra + 1 are the queues'
            // centres
            float4 L[8];
#pragma unroll
            for (int j = 0; j < 4; ++j) L[j] = ld_f4(s + (ra - 4 + j) * SPITCH + col);
#pragma unroll
            for (int j = 0; j < 4; ++j) L[4 + j] = ld_f4(s + (ra + 2 + j) * SPITCH + col);
            const float4 Ya[NQ] = {L[0], L[1], L[2], L[3], qa[H], qb[H], L[4], L[5], L[6]};
            const float4 Yb[NQ] = {L[1], L[2], L[3], qa[H], qb[H], L[4], L[5], L[6], L[7]};
            float zr[12];
            rows_zwin(s + ra * SPITCH, col, qa[H], zr);
            rows_lap<EXACT>(qa, Ya, zr, iso, cpk, a, lapa);
            if (rowb_ok) {
                rows_zwin(s + (ra + 1) * SPITCH, col, qb[H], zr);
                rows_lap<EXACT>(qb, Yb, zr, iso, cpk, a, lapb);
            }
        }
        release(&pempty[s_mid]);
        if (!__all_sync(0xffffffffu, mbar_wait(&cfull[s_core], ph_core))) {
            bad_wait = true;
            goto drain;
        }
        const unsigned char *ct = cring + s_core * CSLOT;
        const float4 ppa = ld_f4(reinterpret_cast<const float *>(ct) + ccol);
        const float4 ppb = ld_f4(reinterpret_cast<const float *>(ct) + ccol + S::TZ);
        const float4 va = ld_f4(reinterpret_cast<const float *>(ct + S::OFF_V) + ccol);
        const float4 vb = ld_f4(reinterpret_cast<const float *>(ct + S::OFF_V) + ccol + S::TZ);
        release(&cempty[s_core]);
        if (rowa_ok) rows_store<EXACT>(a, lapa, qa[H], ppa, va, vma, src_a, x, z0, PPa + (size_t)x * plane, nanacc);
        if (rowb_ok) rows_store<EXACT>(a, lapb, qb[H], ppb, vb, vmb, src_b, x, z0, PPb + (size_t)x * plane, nanacc);
    }
    if (nanacc != nanacc && a.err) atomicOr(a.err, 1u);
    if (bad_wait && a.err) atomicOr(a.err, 2u);
    return;
drain:
    if (a.err) atomicOr(a.err, 2u);
}

}  // namespace detail
}  // namespace rtmb
