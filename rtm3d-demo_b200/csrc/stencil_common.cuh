// stencil_common.cuh -- device helpers shared by the step kernels: the reference taper
// (taper3D / taperUpper3D, RTMCPUPlatform.cpp:566-920) applied to single cells, and guarded loads.
#pragma once
#include "stencil.cuh"

namespace rtmb {
namespace detail {

__device__ __forceinline__ float face_factor(const float *t, int b, int n, int i) {
    return i < b ? t[b - 1 - i] : t[i - (n - b)];
}

// The reference taper applied once to value v held at (x, y, z): the multiply sequence of the
// loop of taper3D / taperUpper3D (RTMCPUPlatform.cpp:566-920) that owns the cell.  The
// front-right quirk cell is handled by the callers.
__device__ __forceinline__ float taper_once(float v, int x, int y, int z, const StepArgs &a) {
    const int b = a.blen;
    const bool xb = x < b || x >= a.nxe - b;
    const bool yb = y < b || y >= a.nye - b;
    const bool zb = a.taper_mode == kTaperAll ? (z < b || z >= a.nze - b) : (z < b);
    if (!zb && a.taper_mode == kTaperUpper) return v;
    if (!xb && !yb && !zb) return v;
    if (xb && zb) {  // x-z corners and edges: y, then x, then z
        if (yb) v = v * face_factor(a.taper, b, a.nye, y);
        v = v * face_factor(a.taper, b, a.nxe, x);
        return v * face_factor(a.taper, b, a.nze, z);
    }
    if (yb && zb) {  // y-z edges
        v = v * face_factor(a.taper, b, a.nye, y);
        return v * face_factor(a.taper, b, a.nze, z);
    }
    if (zb) return v * face_factor(a.taper, b, a.nze, z);
    if (xb && yb) {  // x-y edges (kTaperAll only)
        v = v * face_factor(a.taper, b, a.nxe, x);
        return v * face_factor(a.taper, b, a.nye, y);
    }
    if (yb) return v * face_factor(a.taper, b, a.nye, y);
    return v * face_factor(a.taper, b, a.nxe, x);
}

// The taper factor of index i on an axis of n cells (1.0f off the border) and whether i is in the
// border.  Multiplying by 1.0f is exact, so taper_by_factors below reproduces taper_once.
__device__ __forceinline__ float taper_factor(const float *t, int b, int n, int i, bool &in) {
    in = i < b || i >= n - b;
    return !in ? 1.f : (i < b ? __ldg(t + (b - 1 - i)) : __ldg(t + (i - (n - b))));
}

// taper_once for a cell whose per-axis factors and border flags are known: the reference's multiply
// order is y, x, z everywhere except on the x-y edges (x, then y); the upper form tapers only z < blen.
template <int TAPER>
__device__ __forceinline__ float taper_by_factors(float v, float fx, float fy, float fz, bool xb, bool yb,
                                                  bool zb) {
    if (TAPER == kTaperUpper) return zb ? ((v * fy) * fx) * fz : v;
    if (xb && yb && !zb) return (v * fx) * fy;
    return ((v * fy) * fx) * fz;
}

// Factor of a cell known to lie in the border of its axis (i < b or i >= n - b).
__device__ __forceinline__ float taper_factor_in(const float *t, int b, int n, int i) {
    return __ldg(t + (i < b ? b - 1 - i : i - (n - b)));
}

// The factors of taper_by_factors as three products in a fixed order: T(v) = ((v f1) f2) f3, with
// ones where taper_by_factors multiplies fewer times (a product by 1 is exact).  ALL: every face
// (kTaperAll); otherwise the upper slab (zb: z < blen).
template <bool ALL>
__device__ __forceinline__ void taper_factors3(float fx, float fy, float fz, bool xb, bool yb, bool zb, float &f1,
                                               float &f2, float &f3) {
    if (ALL) {
        const bool sw = xb && yb && !zb;  // the x-y edge off the z borders: (v fx) fy
        f1 = sw ? fx : fy;
        f2 = sw ? fy : fx;
        f3 = sw ? 1.f : fz;
    } else {
        f1 = zb ? fy : 1.f;
        f2 = zb ? fx : 1.f;
        f3 = zb ? fz : 1.f;
    }
}

__device__ __forceinline__ bool quirk_cell(int x, int y, int z, const StepArgs &a) {
    return a.quirk && a.taper_mode == kTaperAll && x < a.blen && y >= a.nye - a.blen &&
           z >= a.blen && z < a.nze - a.blen;
}

__device__ __forceinline__ float get(const float4 &v, int e) {
    return e == 0 ? v.x : (e == 1 ? v.y : (e == 2 ? v.z : v.w));
}
__device__ __forceinline__ void put(float4 &v, int e, float f) {
    if (e == 0) v.x = f; else if (e == 1) v.y = f; else if (e == 2) v.z = f; else v.w = f;
}

template <bool ALIGNED, bool RO>
__device__ __forceinline__ float4 load4(const float *A, size_t plane_off, int yy, int zz, const StepArgs &a) {
    float4 r = make_float4(0.f, 0.f, 0.f, 0.f);
    if (yy < 0 || yy >= a.nye) return r;
    const float *p = A + plane_off + (size_t)yy * a.nze;
    if (ALIGNED) {
        if (zz >= 0 && zz < a.nze) {
            r = RO ? __ldg(reinterpret_cast<const float4 *>(p + zz)) : *reinterpret_cast<const float4 *>(p + zz);
        }
    } else {
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            int z = zz + e;
            if (z >= 0 && z < a.nze) put(r, e, RO ? __ldg(p + z) : p[z]);
        }
    }
    return r;
}

// T(P) for four cells (x, yy, zz..zz+3): raw load, then the taper (with the quirk redirect).
template <bool ALIGNED>
__device__ __forceinline__ float4 load_tapered_p(int x, int yy, int zz, const StepArgs &a, size_t plane) {
    float4 r = load4<ALIGNED, true>(a.P, (size_t)x * plane, yy, zz, a);
    if (a.taper_mode != kTaperNone && yy >= 0 && yy < a.nye) {
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const int z = zz + e;
            if (z < 0 || z >= a.nze) continue;
            float v = get(r, e);
            if (quirk_cell(x, yy, z, a)) {
                // taper3D front-right edge (:900-904): value of (blen, y, z) after the right-face
                // taper, times the x factor, times the y factor.
                const float ty = face_factor(a.taper, a.blen, a.nye, yy);
                v = __ldg(a.P + (size_t)a.blen * plane + (size_t)yy * a.nze + z);
                v = v * ty;
                v = v * face_factor(a.taper, a.blen, a.nxe, x);
                v = v * ty;
            } else {
                v = taper_once(v, x, yy, z, a);
            }
            put(r, e, v);
        }
    }
    return r;
}

}  // namespace detail
}  // namespace rtmb
