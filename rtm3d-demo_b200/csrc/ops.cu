// ops.cu -- per-operator kernels.  Each reproduces one reference CPU operator exactly (same
// multiply order, no contraction: the library is built with --fmad=false).  The kernels are
// templates on the wavefield type: float for the operator API, double for the FP64 GPU oracle.
#include "ops.cuh"

namespace rtmb {
namespace {

__device__ __forceinline__ float fac(const float *t, int b, int n, int i) {
    return i < b ? t[b - 1 - i] : t[i - (n - b)];
}

// Up to four fields tapered by one launch (the frequency-domain migration tapers four per step).
template <typename R>
struct Fields {
    R *f[4];
    int n;
};

// One thread per cell, z fastest (grid: z blocks, y blocks, x), for every field of fs: the cell's loads
// of the fields are independent, so they are in flight together.  Cells off every tapered border
// leave at once.  The front-right quirk of taper3D (a cell (x < blen, y >= nye - blen, z off the z
// borders) takes ((P(blen, y, z) ty) tx) ty, RTMCPUPlatform.cpp:900-904) needs the raw
// P(blen, y, z), which its own thread overwrites: so the thread of (blen, y, z) writes the quirk
// cells of its column and their own threads skip them.  Per cell the factors multiply in the
// reference's loop order.
template <typename R>
__global__ void taper_kernel(Fields<R> fs, const float *__restrict__ t, Geom g, int upper, int quirk) {
    const int z = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y, x = blockIdx.z;
    if (z >= g.nze || y >= g.nye) return;
    const int b = g.blen;
    const bool xb = x < b || x >= g.nxe - b;
    const bool yb = y < b || y >= g.nye - b;
    const bool zb = upper ? (z < b) : (z < b || z >= g.nze - b);
    if (upper ? !zb : !(xb || yb || zb)) return;
    const size_t plane = (size_t)g.nye * g.nze;
    const size_t o = ((size_t)x * g.nye + y) * g.nze + z;
    const bool qcol = !upper && quirk && y >= g.nye - b && !zb;  // right y border, z interior
    if (qcol && x < b) return;                                   // written by the thread of (blen, y, z)
    const R ty = yb ? (R)fac(t, b, g.nye, y) : (R)1;
    const R tz = zb ? (R)fac(t, b, g.nze, z) : (R)1;
    const R tx = xb ? (R)fac(t, b, g.nxe, x) : (R)1;
    R v[4];
#pragma unroll
    for (int k = 0; k < 4; ++k)
        if (k < fs.n) v[k] = fs.f[k][o];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        if (k >= fs.n) break;
        R w = v[k];
        if (xb && zb) {
            if (yb) w = w * ty;
            w = w * tx;
            w = w * tz;
        } else if (yb && zb) {
            w = w * ty;
            w = w * tz;
        } else if (zb) {
            w = w * tz;
        } else if (xb && yb) {
            w = w * tx;
            w = w * ty;
        } else if (yb) {
            w = w * ty;
            if (qcol && x == b) {  // the quirk cells of this column, from the raw P(blen, y, z)
                R *c0 = fs.f[k] + (o - (size_t)b * plane);
                for (int xq = 0; xq < b; ++xq) {
                    R q = w * (R)fac(t, b, g.nxe, xq);
                    q = q * ty;
                    c0[(size_t)xq * plane] = q;
                }
            }
        } else {
            w = w * tx;
        }
        fs.f[k][o] = w;
    }
}

template <typename R>
__global__ void source_kernel(R *PP, const float *w, int it, size_t off) { PP[off] = PP[off] + (R)w[it]; }

// R: wavefield type; RC: record type (the FP64 oracle samples into a double record and injects
// the FP32 record).
template <typename R, typename RC>
__global__ void receivers_kernel(R *PP, RC *rec, int lt, int mode, RcvGeom r, Geom g) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = blockIdx.y;
    if (j >= r.rcy || i >= r.rcx) return;
    const int x = r.rx0 + i * r.rdx, y = r.ry0 + j * r.rdy;
    if (x < 0 || x >= g.nxe || y < 0 || y >= g.nye) return;
    const size_t o = ((size_t)x * g.nye + y) * g.nze + r.rz;
    const size_t ro = ((size_t)i * r.rcy + j) * r.ntstep + lt;
    if (mode == 1) rec[ro] = (RC)PP[o];
    else if (mode == 2) PP[o] = (R)rec[ro];
    else PP[o] = PP[o] + (R)rec[ro];
}

template <typename R>
__global__ void upb_kernel(R *P, R *upb, int lt, int rw, Geom g) {
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

template <typename R>
__global__ void image_kernel(R *img, const R *__restrict__ ps, const R *__restrict__ pr, int z0, int z1, Geom g) {
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

// max |x| over n floats into *out (zero beforehand), as the bits of a non-negative float
__global__ void absmax_kernel(const float *__restrict__ x, size_t n, unsigned *out) {
    float m = 0.f;
    for (size_t o = blockIdx.x * (size_t)blockDim.x + threadIdx.x; o < n; o += (size_t)gridDim.x * blockDim.x)
        m = fmaxf(m, fabsf(x[o]));
    const unsigned b = __reduce_max_sync(0xffffffffu, __float_as_uint(m));
    if ((threadIdx.x & 31) == 0 && b) atomicMax(out, b);
}

// out[0] += sum (a - b)^2, out[1] += sum b^2 over n floats, in double (zero beforehand)
__global__ void sqdiff_kernel(const float *__restrict__ a, const float *__restrict__ b, size_t n, double *out) {
    double d2 = 0.0, b2 = 0.0;
    for (size_t o = blockIdx.x * (size_t)blockDim.x + threadIdx.x; o < n; o += (size_t)gridDim.x * blockDim.x) {
        const double d = (double)a[o] - (double)b[o];
        d2 += d * d;
        b2 += (double)b[o] * (double)b[o];
    }
    for (int k = 16; k; k >>= 1) {
        d2 += __shfl_xor_sync(0xffffffffu, d2, k);
        b2 += __shfl_xor_sync(0xffffffffu, b2, k);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(out, d2);
        atomicAdd(out + 1, b2);
    }
}

// max amax over n scale records into *out (zero beforehand)
__global__ void scale_max_kernel(const ScaleRec *__restrict__ r, int n, unsigned *out) {
    unsigned m = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) m = max(m, r[i].amax);
    m = __reduce_max_sync(0xffffffffu, m);
    if ((threadIdx.x & 31) == 0 && m) atomicMax(out, m);
}

__global__ void to_float_kernel(const double *__restrict__ a, float *out, size_t n) {
    for (size_t o = blockIdx.x * (size_t)blockDim.x + threadIdx.x; o < n; o += (size_t)gridDim.x * blockDim.x)
        out[o] = (float)a[o];
}

__global__ void stack64_kernel(double *acc, const float *__restrict__ img, size_t n) {
    for (size_t o = blockIdx.x * (size_t)blockDim.x + threadIdx.x; o < n; o += (size_t)gridDim.x * blockDim.x)
        acc[o] = acc[o] + (double)img[o];
}

// RTMGrid::stackRegion (src/grid/RTMGrid.cpp:168-223) of a shot image without its border into the
// survey volume, in FP64: one thread per (z) of each (x, y) row of the shot's interior.
template <typename I>
__global__ void stack_region_kernel(double *stack, int snx, int sny, int snz, const I *__restrict__ img, Geom g,
                                    int ox, int oy, int oz) {
    const int nx = g.nxe - 2 * g.blen, ny = g.nye - 2 * g.blen, nz = g.nze - 2 * g.blen;
    const int z = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y, x = blockIdx.z;
    if (z >= nz || x + ox >= snx || y + oy >= sny || z + oz >= snz) return;
    const size_t so = ((size_t)(x + ox) * sny + (y + oy)) * snz + (z + oz);
    const size_t io = ((size_t)(x + g.blen) * g.nye + (y + g.blen)) * g.nze + (z + g.blen);
    stack[so] = stack[so] + (double)img[io];
    (void)nx;
    (void)ny;
}

unsigned grid1d(size_t n) {
    size_t b = (n + 255) / 256;
    return (unsigned)(b > 148u * 64u ? 148u * 64u : (b == 0 ? 1 : b));
}

template <typename R>
cudaError_t taper_t(R *const *fields, int nf, const float *taper, const Geom &g, int upper, int quirk,
                    cudaStream_t s) {
    if (g.blen <= 0) return cudaSuccess;
    if (g.nye > 65535 || g.nxe > 65535 || nf < 1 || nf > 4) return cudaErrorInvalidValue;
    Fields<R> fs{};
    fs.n = nf;
    for (int k = 0; k < nf; ++k) fs.f[k] = fields[k];
    // threads over the z range that can change (the whole row, or z < blen for the upper form),
    // several y rows per block when that range is short
    const int zr = upper ? (g.blen < g.nze ? g.blen : g.nze) : g.nze;
    const int bx = zr >= 128 ? 128 : ((zr + 31) / 32) * 32;
    const int by = 256 / bx;
    dim3 block(bx, by), grid((zr + bx - 1) / bx, (g.nye + by - 1) / by, g.nxe);
    taper_kernel<R><<<grid, block, 0, s>>>(fs, taper, g, upper, quirk);
    return cudaGetLastError();
}

template <typename R>
cudaError_t source_t(R *PP, const float *wavelet, int it, int x, int y, int z, const Geom &g, cudaStream_t s) {
    source_kernel<R><<<1, 1, 0, s>>>(PP, wavelet, it, ((size_t)x * g.nye + y) * g.nze + z);
    return cudaGetLastError();
}

template <typename R, typename RC>
cudaError_t receivers_t(R *PP, RC *rec, int lt, int mode, const RcvGeom &r, const Geom &g, cudaStream_t s) {
    if (r.rcx <= 0 || r.rcy <= 0) return cudaSuccess;
    dim3 grid((r.rcy + 127) / 128, r.rcx);
    receivers_kernel<R, RC><<<grid, 128, 0, s>>>(PP, rec, lt, mode, r, g);
    return cudaGetLastError();
}

template <typename R>
cudaError_t upb_t(R *P, R *upb, int lt, int rw, const Geom &g, cudaStream_t s) {
    dim3 grid((g.nye + 127) / 128, g.nxe);
    upb_kernel<R><<<grid, 128, 0, s>>>(P, upb, lt, rw, g);
    return cudaGetLastError();
}

template <typename R>
cudaError_t image_t(R *img, const R *ps, const R *pr, int z0, int z1, const Geom &g, cudaStream_t s) {
    image_kernel<R><<<grid1d((size_t)g.nxe * g.nye * g.nze), 256, 0, s>>>(img, ps, pr, z0, z1, g);
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_taper(float *P, const float *taper, const Geom &g, int upper, int quirk, cudaStream_t s) {
    return taper_t(&P, 1, taper, g, upper, quirk, s);
}
cudaError_t launch_taper(double *P, const float *taper, const Geom &g, int upper, int quirk, cudaStream_t s) {
    return taper_t(&P, 1, taper, g, upper, quirk, s);
}
cudaError_t launch_taper_fields(float *const *fields, int nf, const float *taper, const Geom &g, int upper, int quirk,
                                cudaStream_t s) {
    return taper_t(fields, nf, taper, g, upper, quirk, s);
}
cudaError_t launch_source(float *PP, const float *wavelet, int it, int x, int y, int z, const Geom &g,
                          cudaStream_t s) {
    return source_t(PP, wavelet, it, x, y, z, g, s);
}
cudaError_t launch_source(double *PP, const float *wavelet, int it, int x, int y, int z, const Geom &g,
                          cudaStream_t s) {
    return source_t(PP, wavelet, it, x, y, z, g, s);
}
cudaError_t launch_receivers(float *PP, float *rec, int lt, int mode, const RcvGeom &r, const Geom &g,
                             cudaStream_t s) {
    return receivers_t(PP, rec, lt, mode, r, g, s);
}
cudaError_t launch_receivers(double *PP, float *rec, int lt, int mode, const RcvGeom &r, const Geom &g,
                             cudaStream_t s) {
    return receivers_t(PP, rec, lt, mode, r, g, s);
}
cudaError_t launch_receivers(double *PP, double *rec, int lt, int mode, const RcvGeom &r, const Geom &g,
                             cudaStream_t s) {
    return receivers_t(PP, rec, lt, mode, r, g, s);
}
cudaError_t launch_upb(float *P, float *upb, int lt, int rw, const Geom &g, cudaStream_t s) {
    return upb_t(P, upb, lt, rw, g, s);
}
cudaError_t launch_upb(double *P, double *upb, int lt, int rw, const Geom &g, cudaStream_t s) {
    return upb_t(P, upb, lt, rw, g, s);
}
cudaError_t launch_image(float *img, const float *ps, const float *pr, int z0, int z1, const Geom &g,
                         cudaStream_t s) {
    return image_t(img, ps, pr, z0, z1, g, s);
}
cudaError_t launch_image(double *img, const double *ps, const double *pr, int z0, int z1, const Geom &g,
                         cudaStream_t s) {
    return image_t(img, ps, pr, z0, z1, g, s);
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

cudaError_t launch_absmax(const float *x, size_t n, float *out, cudaStream_t s) {
    cudaError_t e = cudaMemsetAsync(out, 0, sizeof(float), s);
    if (e != cudaSuccess || n == 0) return e;
    absmax_kernel<<<grid1d(n), 256, 0, s>>>(x, n, reinterpret_cast<unsigned *>(out));
    return cudaGetLastError();
}

cudaError_t launch_scale_max(const ScaleRec *r, int n, float *out, cudaStream_t s) {
    cudaError_t e = cudaMemsetAsync(out, 0, sizeof(float), s);
    if (e != cudaSuccess || n <= 0) return e;
    scale_max_kernel<<<1, 256, 0, s>>>(r, n, reinterpret_cast<unsigned *>(out));
    return cudaGetLastError();
}

cudaError_t launch_sqdiff(const float *a, const float *b, size_t n, double *out, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    sqdiff_kernel<<<grid1d(n), 256, 0, s>>>(a, b, n, out);
    return cudaGetLastError();
}

cudaError_t launch_to_float(const double *a, float *out, size_t n, cudaStream_t s) {
    to_float_kernel<<<grid1d(n), 256, 0, s>>>(a, out, n);
    return cudaGetLastError();
}

cudaError_t launch_stack_region64(double *stack, int snx, int sny, int snz, const void *img, bool img64,
                                  const Geom &g, int ox, int oy, int oz, cudaStream_t s) {
    const int nx = g.nxe - 2 * g.blen, ny = g.nye - 2 * g.blen, nz = g.nze - 2 * g.blen;
    if (nx <= 0 || ny <= 0 || nz <= 0) return cudaErrorInvalidValue;
    dim3 grid((nz + 127) / 128, ny, nx);
    if (img64)
        stack_region_kernel<double><<<grid, 128, 0, s>>>(stack, snx, sny, snz, static_cast<const double *>(img), g,
                                                         ox, oy, oz);
    else
        stack_region_kernel<float><<<grid, 128, 0, s>>>(stack, snx, sny, snz, static_cast<const float *>(img), g, ox,
                                                        oy, oz);
    return cudaGetLastError();
}

cudaError_t launch_stack64(double *acc, const float *img, size_t n, cudaStream_t s) {
    stack64_kernel<<<grid1d(n), 256, 0, s>>>(acc, img, n);
    return cudaGetLastError();
}

}  // namespace rtmb
