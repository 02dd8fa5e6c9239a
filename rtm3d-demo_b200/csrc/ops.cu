// ops.cu -- per-operator kernels.  Each reproduces one reference CPU operator exactly (same
// multiply order, no contraction: the library is built with --fmad=false).
#include "ops.cuh"

namespace rtmb {
namespace {

__device__ __forceinline__ float fac(const float *t, int b, int n, int i) {
    return i < b ? t[b - 1 - i] : t[i - (n - b)];
}

// One thread owns a (y, z) column and walks x, so the front-right quirk of taper3D (a cell that
// takes its value from x = blen, RTMCPUPlatform.cpp:900-904) reads the raw value of its own column
// before anything in the column is written.
__global__ void taper_kernel(float *P, const float *__restrict__ t, Geom g, int upper, int quirk) {
    const int z = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    if (z >= g.nze) return;
    const int b = g.blen;
    const bool yb = y < b || y >= g.nye - b;
    const bool zb = upper ? (z < b) : (z < b || z >= g.nze - b);
    if (upper && !zb) return;
    const size_t plane = (size_t)g.nye * g.nze;
    float *col = P + (size_t)y * g.nze + z;
    const float ty = yb ? fac(t, b, g.nye, y) : 1.f;
    const float tz = zb ? fac(t, b, g.nze, z) : 1.f;
    // the x range that changes: the whole column if y or z is in a border, else the two x slabs
    const bool whole = yb || zb;
    const bool qcol = !upper && quirk && y >= g.nye - b && !zb;  // right y border, z interior
    float face = 0.f;
    if (qcol) face = col[(size_t)b * plane] * ty;  // (blen, y, z) after the right-face taper
    for (int x = 0; x < g.nxe; ++x) {
        const bool xb = x < b || x >= g.nxe - b;
        if (!whole && !xb) { x = g.nxe - b - 1; continue; }
        float v = col[(size_t)x * plane];
        if (xb && zb) {
            if (yb) v = v * ty;
            v = v * fac(t, b, g.nxe, x);
            v = v * tz;
        } else if (yb && zb) {
            v = v * ty;
            v = v * tz;
        } else if (zb) {
            v = v * tz;
        } else if (xb && yb) {
            if (qcol && x < b) {
                v = face * fac(t, b, g.nxe, x);
                v = v * ty;
            } else {
                v = v * fac(t, b, g.nxe, x);
                v = v * ty;
            }
        } else if (yb) {
            v = v * ty;
        } else {
            v = v * fac(t, b, g.nxe, x);
        }
        col[(size_t)x * plane] = v;
    }
}

__global__ void source_kernel(float *PP, const float *w, int it, size_t off) { PP[off] = PP[off] + w[it]; }

__global__ void receivers_kernel(float *PP, float *rec, int lt, int mode, RcvGeom r, Geom g) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = blockIdx.y;
    if (j >= r.rcy || i >= r.rcx) return;
    const int x = r.rx0 + i * r.rdx, y = r.ry0 + j * r.rdy;
    if (x < 0 || x >= g.nxe || y < 0 || y >= g.nye) return;
    const size_t o = ((size_t)x * g.nye + y) * g.nze + r.rz;
    const size_t ro = ((size_t)i * r.rcy + j) * r.ntstep + lt;
    if (mode == 1) rec[ro] = PP[o];
    else if (mode == 2) PP[o] = rec[ro];
    else PP[o] = PP[o] + rec[ro];
}

__global__ void upb_kernel(float *P, float *upb, int lt, int rw, Geom g) {
    const int y = blockIdx.x * blockDim.x + threadIdx.x;
    const int x = blockIdx.y;
    if (y >= g.nye) return;
    const size_t po = ((size_t)x * g.nye + y) * g.nze + (g.blen - g.h);
    const size_t uo = (((size_t)lt * g.nxe + x) * g.nye + y) * g.h;
    for (int k = 0; k < g.h; ++k) {
        if (rw) upb[uo + k] = P[po + k];
        else P[po + k] = upb[uo + k];
    }
}

__global__ void image_kernel(float *img, const float *__restrict__ ps, const float *__restrict__ pr,
                             int z0, int z1, Geom g) {
    const size_t n = (size_t)g.nxe * g.nye * g.nze;
    for (size_t o = blockIdx.x * (size_t)blockDim.x + threadIdx.x; o < n; o += (size_t)gridDim.x * blockDim.x) {
        const int z = (int)(o % g.nze);
        if (z >= z0 && z < z1) img[o] = img[o] + ps[o] * pr[o];
    }
}

__global__ void filter_remove_kernel(const float *__restrict__ img, float *out, Geom g, float c0x, float c1x,
                                     float c2x, float c0y, float c1y, float c2y, float c0z, float c1z, float c2z) {
    const int ny = g.nye - 2 * g.blen, nz = g.nze - 2 * g.blen;
    const int z = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y, x = blockIdx.z;
    if (z >= nz) return;
    const int ix = x + g.blen, iy = y + g.blen, iz = z + g.blen;
    auto at = [&](int a, int b, int c) { return img[((size_t)a * g.nye + b) * g.nze + c]; };
    float ax = 0.f, ay = 0.f, az = 0.f;
    ax = ax + at(ix - 1, iy, iz) * c0x; ay = ay + at(ix, iy - 1, iz) * c0y; az = az + at(ix, iy, iz - 1) * c0z;
    ax = ax + at(ix, iy, iz) * c1x;     ay = ay + at(ix, iy, iz) * c1y;     az = az + at(ix, iy, iz) * c1z;
    ax = ax + at(ix + 1, iy, iz) * c2x; ay = ay + at(ix, iy + 1, iz) * c2y; az = az + at(ix, iy, iz + 1) * c2z;
    out[((size_t)x * ny + y) * nz + z] = ax + ay + az;
}

__global__ void stack_kernel(float *acc, const float *__restrict__ img, size_t n) {
    for (size_t o = blockIdx.x * (size_t)blockDim.x + threadIdx.x; o < n; o += (size_t)gridDim.x * blockDim.x)
        acc[o] = acc[o] + img[o];
}

unsigned grid1d(size_t n) {
    size_t b = (n + 255) / 256;
    return (unsigned)(b > 148u * 64u ? 148u * 64u : (b == 0 ? 1 : b));
}

}  // namespace

cudaError_t launch_taper(float *P, const float *taper, const Geom &g, int upper, int quirk, cudaStream_t s) {
    if (g.blen <= 0) return cudaSuccess;
    dim3 grid((g.nze + 127) / 128, g.nye);
    taper_kernel<<<grid, 128, 0, s>>>(P, taper, g, upper, quirk);
    return cudaGetLastError();
}

cudaError_t launch_source(float *PP, const float *wavelet, int it, int x, int y, int z, const Geom &g,
                          cudaStream_t s) {
    source_kernel<<<1, 1, 0, s>>>(PP, wavelet, it, ((size_t)x * g.nye + y) * g.nze + z);
    return cudaGetLastError();
}

cudaError_t launch_receivers(float *PP, float *rec, int lt, int mode, const RcvGeom &r, const Geom &g,
                             cudaStream_t s) {
    if (r.rcx <= 0 || r.rcy <= 0) return cudaSuccess;
    dim3 grid((r.rcy + 127) / 128, r.rcx);
    receivers_kernel<<<grid, 128, 0, s>>>(PP, rec, lt, mode, r, g);
    return cudaGetLastError();
}

cudaError_t launch_upb(float *P, float *upb, int lt, int rw, const Geom &g, cudaStream_t s) {
    dim3 grid((g.nye + 127) / 128, g.nxe);
    upb_kernel<<<grid, 128, 0, s>>>(P, upb, lt, rw, g);
    return cudaGetLastError();
}

cudaError_t launch_image(float *img, const float *ps, const float *pr, int z0, int z1, const Geom &g,
                         cudaStream_t s) {
    image_kernel<<<grid1d((size_t)g.nxe * g.nye * g.nze), 256, 0, s>>>(img, ps, pr, z0, z1, g);
    return cudaGetLastError();
}

cudaError_t launch_filter_remove(const float *img, float *out, const float *c3, const Geom &g, cudaStream_t s) {
    const int nx = g.nxe - 2 * g.blen, ny = g.nye - 2 * g.blen, nz = g.nze - 2 * g.blen;
    if (nx <= 0 || ny <= 0 || nz <= 0) return cudaErrorInvalidValue;
    dim3 grid((nz + 127) / 128, ny, nx);
    filter_remove_kernel<<<grid, 128, 0, s>>>(img, out, g, c3[0], c3[1], c3[2], c3[3], c3[4], c3[5], c3[6],
                                               c3[7], c3[8]);
    return cudaGetLastError();
}

cudaError_t launch_stack(float *acc, const float *img, size_t n, cudaStream_t s) {
    stack_kernel<<<grid1d(n), 256, 0, s>>>(acc, img, n);
    return cudaGetLastError();
}

}  // namespace rtmb
