// stencil_impl.cuh -- kernel template of the fused time step; instantiated once per stencil
// half-order by stencil_h<N>.cu so the instantiations compile in parallel.
//
// Built with --fmad=false: in the exact (default) form every product and sum is rounded on its
// own, in the reference CPU order (acmx, acmy, acmz each summed from 0 in tap order, then
// (acmx + acmy) + acmz, then (2p - pp) + v*lapl), so results are bit-identical to
// RTMCPUPlatform::rtmStep3D.  The fast form uses explicit fmaf().
#pragma once
#include "stencil_common.cuh"

namespace rtmb {
namespace detail {

template <int H, bool EXACT, bool ALIGNED>
__global__ void __launch_bounds__(kThreads, 2) step_kernel(const __grid_constant__ StepArgs a) {
    constexpr int ZH = ((H + 3) / 4) * 4;          // z halo rounded up to a float4
    constexpr int SROWS = kTY + 2 * H;
    constexpr int SPITCH = kTZ + 2 * ZH;
    constexpr int NQ = 2 * H + 1;
    constexpr int ZQ = kTZ / kVZ;                   // threads along z
    constexpr int NYH = 2 * H * ZQ;                 // y-halo float4 slots
    constexpr int NZH = kTY * 2 * (ZH / kVZ);       // z-halo float4 slots
    constexpr int NHALO = NYH + NZH;
    constexpr int NHT = (NHALO + kThreads - 1) / kThreads;
    __shared__ __align__(16) float sm[2][SROWS * SPITCH];

    const int tid = threadIdx.x;
    const int tz = tid % ZQ, ty = tid / ZQ;
    const int zt0 = blockIdx.x * kTZ;
    const int yt0 = H + blockIdx.y * kTY;
    const int z0 = zt0 + tz * kVZ;
    const int y = yt0 + ty;
    int xc0 = H + blockIdx.z * a.chunk;
    int xc1 = min(xc0 + a.chunk, a.nxe - H);
    if (a.x_hi > 0) {  // 2D models: the plane x = blen only
        xc0 = max(xc0, a.x_lo);
        xc1 = min(xc1, a.x_hi);
    }
    if (xc0 >= xc1) return;
    const size_t plane = (size_t)a.nye * a.nze;
    const bool row_ok = y < a.nye;

    // halo slot -> (tile row, tile col) of its float4
    int hrow[NHT], hcol[NHT];
#pragma unroll
    for (int k = 0; k < NHT; ++k) {
        const int s = tid + k * kThreads;
        if (s < NYH) {
            const int r = s / ZQ, c = s % ZQ;
            hrow[k] = r < H ? r : kTY + r;           // rows [0,H) and [TY+H, TY+2H)
            hcol[k] = ZH + c * kVZ;
        } else if (s < NHALO) {
            const int u = s - NYH;
            const int per_row = 2 * (ZH / kVZ);
            const int r = u / per_row, c = u % per_row;
            hrow[k] = H + r;
            hcol[k] = c < ZH / kVZ ? c * kVZ : kTZ + ZH + (c - ZH / kVZ) * kVZ;
        } else {
            hrow[k] = -1;
            hcol[k] = 0;
        }
    }

    float4 q[NQ];
    // warm-up: planes xc0-H .. xc0+H-1 into q[1..2H]
#pragma unroll
    for (int k = 0; k < 2 * H; ++k) q[k + 1] = load_tapered_p<ALIGNED>(xc0 - H + k, y, z0, a, plane);

    float4 c_next = load_tapered_p<ALIGNED>(xc0 + H, y, z0, a, plane);
    float4 h_next[NHT];
#pragma unroll
    for (int k = 0; k < NHT; ++k)
        h_next[k] = hrow[k] >= 0 ? load_tapered_p<ALIGNED>(xc0, yt0 - H + hrow[k], zt0 - ZH + hcol[k], a, plane)
                                 : make_float4(0.f, 0.f, 0.f, 0.f);
    float4 pp_next = load4<ALIGNED, false>(a.PP, (size_t)xc0 * plane, y, z0, a);
    float4 v_next = load4<ALIGNED, true>(a.V, (size_t)xc0 * plane, y, z0, a);

    unsigned bad = 0;
    const int col = ZH + tz * kVZ;

    for (int x = xc0; x < xc1; ++x) {
        // advance the x queue
#pragma unroll
        for (int k = 0; k < NQ - 1; ++k) q[k] = q[k + 1];
        q[NQ - 1] = c_next;
        float4 h_cur[NHT];
#pragma unroll
        for (int k = 0; k < NHT; ++k) h_cur[k] = h_next[k];
        const float4 pp_raw = pp_next;
        const float4 vv = v_next;

        float *s = sm[x & 1];
        *reinterpret_cast<float4 *>(&s[(ty + H) * SPITCH + col]) = q[H];
#pragma unroll
        for (int k = 0; k < NHT; ++k)
            if (hrow[k] >= 0) *reinterpret_cast<float4 *>(&s[hrow[k] * SPITCH + hcol[k]]) = h_cur[k];
        __syncthreads();

        // prefetch plane x+1
        if (x + 1 < xc1) {
            c_next = load_tapered_p<ALIGNED>(x + 1 + H, y, z0, a, plane);
#pragma unroll
            for (int k = 0; k < NHT; ++k)
                if (hrow[k] >= 0)
                    h_next[k] = load_tapered_p<ALIGNED>(x + 1, yt0 - H + hrow[k], zt0 - ZH + hcol[k], a, plane);
            pp_next = load4<ALIGNED, false>(a.PP, (size_t)(x + 1) * plane, y, z0, a);
            v_next = load4<ALIGNED, true>(a.V, (size_t)(x + 1) * plane, y, z0, a);
        }

        if (!row_ok) continue;  // no block-level sync below, so an early continue is safe

        // centre row of the tile, z0-ZH .. z0+VZ+ZH
        float zr[kVZ + 2 * ZH];
#pragma unroll
        for (int k = 0; k < (kVZ + 2 * ZH) / 4; ++k) {
            float4 t4 = (k == ZH / 4) ? q[H] : *reinterpret_cast<const float4 *>(&s[(ty + H) * SPITCH + col - ZH + 4 * k]);
            zr[4 * k + 0] = t4.x; zr[4 * k + 1] = t4.y; zr[4 * k + 2] = t4.z; zr[4 * k + 3] = t4.w;
        }

        float lap[kVZ];
        if (EXACT) {
            float ax[kVZ], ay[kVZ], az[kVZ];
#pragma unroll
            for (int e = 0; e < kVZ; ++e) { ax[e] = 0.f; ay[e] = 0.f; az[e] = 0.f; }
#pragma unroll
            for (int io = 0; io < NQ; ++io) {
                const float4 ry = (io == H) ? q[H] : *reinterpret_cast<const float4 *>(&s[(ty + io) * SPITCH + col]);
#pragma unroll
                for (int e = 0; e < kVZ; ++e) {
                    ax[e] = ax[e] + get(q[io], e) * a.cx[io];
                    ay[e] = ay[e] + get(ry, e) * a.cy[io];
                    az[e] = az[e] + zr[ZH - H + e + io] * a.cz[io];
                }
            }
#pragma unroll
            for (int e = 0; e < kVZ; ++e) lap[e] = ax[e] + ay[e] + az[e];
        } else {
            const float cc = a.cx[H] + a.cy[H] + a.cz[H];
#pragma unroll
            for (int e = 0; e < kVZ; ++e) lap[e] = get(q[H], e) * cc;
#pragma unroll
            for (int io = 0; io < NQ; ++io) {
                if (io == H) continue;
                const float4 ry = *reinterpret_cast<const float4 *>(&s[(ty + io) * SPITCH + col]);
#pragma unroll
                for (int e = 0; e < kVZ; ++e) {
                    lap[e] = fmaf(get(q[io], e), a.cx[io], lap[e]);
                    lap[e] = fmaf(get(ry, e), a.cy[io], lap[e]);
                    lap[e] = fmaf(zr[ZH - H + e + io], a.cz[io], lap[e]);
                }
            }
        }

        float4 out = pp_raw;
        const size_t po = (size_t)x * plane + (size_t)y * a.nze;
        const bool y_ok = y < a.nye - H;
        bool any_img = false;
        float img_v[kVZ], ps_v[kVZ];
#pragma unroll
        for (int e = 0; e < kVZ; ++e) {
            const int z = z0 + e;
            if (!(y_ok && z >= H && z < a.nze - H)) continue;
            const float p = get(q[H], e);
            float pp = get(pp_raw, e);
            if (a.taper_mode != kTaperNone) {
                if (quirk_cell(x, y, z, a)) {
                    const float ty_ = face_factor(a.taper, a.blen, a.nye, y);
                    pp = a.quirk_in[(size_t)(y - (a.nye - a.blen)) * (a.nze - 2 * a.blen) + (z - a.blen)];
                    pp = pp * ty_;
                    pp = pp * ty_;
                    pp = pp * face_factor(a.taper, a.blen, a.nxe, x);
                    pp = pp * ty_;
                } else {
                    pp = taper_once(taper_once(pp, x, y, z, a), x, y, z, a);
                }
            }
            float npp;
            if (EXACT) {
                const float two_p = 2.f * p;
                const float d = two_p - pp;
                const float vl = get(vv, e) * lap[e];
                npp = d + vl;
            } else {
                npp = fmaf(get(vv, e), lap[e], 2.f * p - pp);
            }
            if (x == a.sxe && y == a.sye && z == a.sze) npp = npp + a.wavelet[a.it];
            if (a.rec_mode != kRecNone && z == a.rz) {
                const int dxr = x - a.rx0, dyr = y - a.ry0;
                if (dxr >= 0 && dyr >= 0 && dxr % a.rdx == 0 && dyr % a.rdy == 0) {
                    const int i = dxr / a.rdx, j = dyr / a.rdy;
                    if (i < a.rcx && j < a.rcy) {
                        float *rp = a.rec + a.rec_base + i * a.rec_si + j * a.rec_sj;
                        if (a.rec_mode == kRecSample) *rp = npp;
                        else if (a.rec_mode == kRecOverwrite) npp = *rp;
                        else npp = npp + *rp;
                    }
                }
            }
            if (a.upb_mode != kUpbNone && z >= a.blen - H && z < a.blen) {
                float *up = a.upb + ((size_t)x * a.nye + y) * H + (z - (a.blen - H));
                if (a.upb_mode == kUpbSave) *up = npp;
                else npp = *up;
            }
            if (a.quirk_out && x == a.blen && y >= a.nye - a.blen && z >= a.blen && z < a.nze - a.blen)
                a.quirk_out[(size_t)(y - (a.nye - a.blen)) * (a.nze - 2 * a.blen) + (z - a.blen)] = npp;
            bad |= (npp != npp);
            put(out, e, npp);
            if (a.img && z >= a.img_z0 && z < a.img_z1) any_img = true;
        }

        if (ALIGNED) {
            if (z0 >= a.nze) continue;  // thread past the end of the last z tile
            *reinterpret_cast<float4 *>(a.PP + po + z0) = out;
            if (any_img) {
                float4 im = *reinterpret_cast<const float4 *>(a.img + po + z0);
                const float4 ps4 = __ldg(reinterpret_cast<const float4 *>(a.ps + po + z0));
#pragma unroll
                for (int e = 0; e < kVZ; ++e) {
                    const int z = z0 + e;
                    if (y_ok && z >= H && z < a.nze - H && z >= a.img_z0 && z < a.img_z1)
                        put(im, e, get(im, e) + get(ps4, e) * get(out, e));
                }
                *reinterpret_cast<float4 *>(a.img + po + z0) = im;
            }
        } else {
#pragma unroll
            for (int e = 0; e < kVZ; ++e) {
                const int z = z0 + e;
                if (!(y_ok && z >= H && z < a.nze - H)) continue;
                a.PP[po + z] = get(out, e);
                if (a.img && z >= a.img_z0 && z < a.img_z1) {
                    img_v[e] = a.img[po + z];
                    ps_v[e] = __ldg(a.ps + po + z);
                    a.img[po + z] = img_v[e] + ps_v[e] * get(out, e);
                }
            }
        }
    }
    if (bad && a.err) atomicOr(a.err, 1u);
}

template <int H>
cudaError_t launch_h(const StepArgs &a, bool exact, bool aligned, dim3 grid, cudaStream_t s) {
    if (exact) {
        if (aligned) step_kernel<H, true, true><<<grid, kThreads, 0, s>>>(a);
        else step_kernel<H, true, false><<<grid, kThreads, 0, s>>>(a);
    } else {
        if (aligned) step_kernel<H, false, true><<<grid, kThreads, 0, s>>>(a);
        else step_kernel<H, false, false><<<grid, kThreads, 0, s>>>(a);
    }
    return cudaGetLastError();
}

}  // namespace detail
}  // namespace rtmb
