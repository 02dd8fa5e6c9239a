// fmig.cu -- the frequency-domain part of frequency-domain RTM (fmig): the running DFT of the
// source and receiver wavefields and the frequency-domain imaging condition, one launch per time
// step for a group of frequencies.
//
// The reference runs two operators per frequency and time step (RTMCPUPlatform.cpp:20-64,
// rtmUpdateFreqContributions, then :66-102, rtmFreqDomainImageCondition), each a pass over the
// model interior.  Per point they form, for iw in the group, in this order:
//     sRe += kre ps;  sIm += kim ps;  rRe += kre pr;  rIm += kim pr;
//     img += w2 (sRe rRe - sIm rIm)
// Points are independent, so one thread per point runs the frequency loop in the same order and
// the image sum of every point sees the same sequence of additions: one pass over the frequency
// grids per step instead of two per frequency, and the image is read and written once.
//
// Layout: the four frequency grids are [nws][nx][ny][nz] over the unpadded interior (z fastest,
// ..._FreqDomain.cpp:53-103); ps, pr and img are padded volumes.  This pass is bound by HBM: per
// point and step it moves 32 B per frequency plus 16 B for ps, pr and the image.
#include "ops.cuh"

namespace rtmb {
namespace {

// grid: (ceil(nz / 128), ny, nx); one thread per interior point, z fastest.
template <bool EXACT>
__global__ void __launch_bounds__(128) fmig_freq_kernel(const float *__restrict__ ps, const float *__restrict__ pr,
                                                        float *img, float *sre, float *sim, float *rre, float *rim,
                                                        FmigStep f, Geom g, int nx, int ny, int nz) {
    const int z = blockIdx.x * blockDim.x + threadIdx.x;
    if (z >= nz) return;
    const int y = blockIdx.y, x = blockIdx.z;
    const size_t o = ((size_t)(x + g.blen) * g.nye + (y + g.blen)) * g.nze + (z + g.blen);
    const size_t ni = (size_t)nx * ny * nz;
    size_t fi = ((size_t)x * ny + y) * nz + z;
    const float s = ps[o], r = pr[o];
    float im = img[o];
#pragma unroll 2
    for (int lw = 0; lw < f.nws; ++lw, fi += ni) {
        const float kr = f.kre[lw], ki = f.kim[lw], w2 = f.w2[lw];
        float a = sre[fi], b = sim[fi], c = rre[fi], d = rim[fi];
        if (EXACT) {
            a = a + kr * s;
            b = b + ki * s;
            c = c + kr * r;
            d = d + ki * r;
            im = im + w2 * (a * c - b * d);
        } else {
            a = fmaf(kr, s, a);
            b = fmaf(ki, s, b);
            c = fmaf(kr, r, c);
            d = fmaf(ki, r, d);
            im = fmaf(w2, fmaf(a, c, -(b * d)), im);
        }
        sre[fi] = a;
        sim[fi] = b;
        rre[fi] = c;
        rim[fi] = d;
    }
    img[o] = im;
}

// The same, four consecutive z points per thread with 16-byte accesses (nz and the interior's
// padded offset multiples of 4): four times the bytes in flight per load.
template <bool EXACT>
__global__ void __launch_bounds__(128) fmig_freq4_kernel(const float *__restrict__ ps, const float *__restrict__ pr,
                                                         float *img, float *sre, float *sim, float *rre, float *rim,
                                                         FmigStep f, Geom g, int nx, int ny, int nz) {
    const int z = 4 * (blockIdx.x * blockDim.x + threadIdx.x);
    if (z >= nz) return;
    const int y = blockIdx.y, x = blockIdx.z;
    const size_t o = ((size_t)(x + g.blen) * g.nye + (y + g.blen)) * g.nze + (z + g.blen);
    const size_t ni = (size_t)nx * ny * nz;
    size_t fi = ((size_t)x * ny + y) * nz + z;
    const float4 s4 = *reinterpret_cast<const float4 *>(ps + o), r4 = *reinterpret_cast<const float4 *>(pr + o);
    float4 im4 = *reinterpret_cast<const float4 *>(img + o);
    const float s[4] = {s4.x, s4.y, s4.z, s4.w}, r[4] = {r4.x, r4.y, r4.z, r4.w};
    float im[4] = {im4.x, im4.y, im4.z, im4.w};
#pragma unroll 2
    for (int lw = 0; lw < f.nws; ++lw, fi += ni) {
        const float kr = f.kre[lw], ki = f.kim[lw], w2 = f.w2[lw];
        float4 *pa = reinterpret_cast<float4 *>(sre + fi), *pb = reinterpret_cast<float4 *>(sim + fi);
        float4 *pc = reinterpret_cast<float4 *>(rre + fi), *pd = reinterpret_cast<float4 *>(rim + fi);
        const float4 a4 = *pa, b4 = *pb, c4 = *pc, d4 = *pd;
        float a[4] = {a4.x, a4.y, a4.z, a4.w}, b[4] = {b4.x, b4.y, b4.z, b4.w};
        float c[4] = {c4.x, c4.y, c4.z, c4.w}, d[4] = {d4.x, d4.y, d4.z, d4.w};
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            if (EXACT) {
                a[e] = a[e] + kr * s[e];
                b[e] = b[e] + ki * s[e];
                c[e] = c[e] + kr * r[e];
                d[e] = d[e] + ki * r[e];
                im[e] = im[e] + w2 * (a[e] * c[e] - b[e] * d[e]);
            } else {
                a[e] = fmaf(kr, s[e], a[e]);
                b[e] = fmaf(ki, s[e], b[e]);
                c[e] = fmaf(kr, r[e], c[e]);
                d[e] = fmaf(ki, r[e], d[e]);
                im[e] = fmaf(w2, fmaf(a[e], c[e], -(b[e] * d[e])), im[e]);
            }
        }
        *pa = make_float4(a[0], a[1], a[2], a[3]);
        *pb = make_float4(b[0], b[1], b[2], b[3]);
        *pc = make_float4(c[0], c[1], c[2], c[3]);
        *pd = make_float4(d[0], d[1], d[2], d[3]);
    }
    *reinterpret_cast<float4 *>(img + o) = make_float4(im[0], im[1], im[2], im[3]);
}

// The reference's two per-frequency operators as they are (the per-operator entry points): one
// frequency lw of the grids, table values read on the device at [iw][it] and [iw].
__global__ void fmig_update_kernel(const float *__restrict__ ps, const float *__restrict__ pr, float *sre, float *sim,
                                   float *rre, float *rim, const float *__restrict__ kre,
                                   const float *__restrict__ kim, size_t kofs, size_t fofs, Geom g, int nx, int ny,
                                   int nz) {
    const int z = blockIdx.x * blockDim.x + threadIdx.x;
    if (z >= nz) return;
    const int y = blockIdx.y, x = blockIdx.z;
    const size_t o = ((size_t)(x + g.blen) * g.nye + (y + g.blen)) * g.nze + (z + g.blen);
    const size_t f = fofs + ((size_t)x * ny + y) * nz + z;
    const float kr = kre[kofs], ki = kim[kofs], s = ps[o], r = pr[o];
    sre[f] = sre[f] + (kr * s);
    sim[f] = sim[f] + (ki * s);
    rre[f] = rre[f] + (kr * r);
    rim[f] = rim[f] + (ki * r);
}

__global__ void fmig_image_kernel(float *img, const float *__restrict__ sre, const float *__restrict__ sim,
                                  const float *__restrict__ rre, const float *__restrict__ rim,
                                  const float *__restrict__ w2, int iw, size_t fofs, Geom g, int nx, int ny, int nz) {
    const int z = blockIdx.x * blockDim.x + threadIdx.x;
    if (z >= nz) return;
    const int y = blockIdx.y, x = blockIdx.z;
    const size_t o = ((size_t)(x + g.blen) * g.nye + (y + g.blen)) * g.nze + (z + g.blen);
    const size_t f = fofs + ((size_t)x * ny + y) * nz + z;
    img[o] = img[o] + (w2[iw]) * (sre[f] * rre[f] - sim[f] * rim[f]);
}

}  // namespace

cudaError_t launch_fmig_update(const float *ps, const float *pr, float *sre, float *sim, float *rre, float *rim,
                               const float *kre, const float *kim, int it, int iw, int lw, int nt, const Geom &g,
                               int nx, int ny, int nz, cudaStream_t s) {
    if (nx <= 0 || ny <= 0 || nz <= 0 || ny > 65535 || nx > 65535) return cudaErrorInvalidValue;
    dim3 grid((nz + 127) / 128, ny, nx);
    fmig_update_kernel<<<grid, 128, 0, s>>>(ps, pr, sre, sim, rre, rim, kre, kim, (size_t)iw * nt + it,
                                            (size_t)lw * nx * ny * nz, g, nx, ny, nz);
    return cudaGetLastError();
}

cudaError_t launch_fmig_image(float *img, const float *sre, const float *sim, const float *rre, const float *rim,
                              const float *w2, int iw, int lw, const Geom &g, int nx, int ny, int nz, cudaStream_t s) {
    if (nx <= 0 || ny <= 0 || nz <= 0 || ny > 65535 || nx > 65535) return cudaErrorInvalidValue;
    dim3 grid((nz + 127) / 128, ny, nx);
    fmig_image_kernel<<<grid, 128, 0, s>>>(img, sre, sim, rre, rim, w2, iw, (size_t)lw * nx * ny * nz, g, nx, ny, nz);
    return cudaGetLastError();
}

cudaError_t launch_fmig_freq(const float *ps, const float *pr, float *img, float *fq, const FmigStep &f, const Geom &g,
                             int nx, int ny, int nz, bool exact, cudaStream_t s) {
    if (f.nws <= 0 || f.nws > kFmigMaxGroup || nx <= 0 || ny <= 0 || nz <= 0 || ny > 65535 || nx > 65535)
        return cudaErrorInvalidValue;
    const size_t g4 = (size_t)f.nws * nx * ny * nz;  // one frequency grid of the group
    const uintptr_t al = reinterpret_cast<uintptr_t>(ps) | reinterpret_cast<uintptr_t>(pr) |
                         reinterpret_cast<uintptr_t>(img) | reinterpret_cast<uintptr_t>(fq);
    if (nz % 4 == 0 && g.nze % 4 == 0 && g.blen % 4 == 0 && al % 16 == 0) {
        dim3 grid4((nz / 4 + 127) / 128, ny, nx);
        if (exact)
            fmig_freq4_kernel<true><<<grid4, 128, 0, s>>>(ps, pr, img, fq, fq + g4, fq + 2 * g4, fq + 3 * g4, f, g, nx,
                                                          ny, nz);
        else
            fmig_freq4_kernel<false><<<grid4, 128, 0, s>>>(ps, pr, img, fq, fq + g4, fq + 2 * g4, fq + 3 * g4, f, g, nx,
                                                           ny, nz);
        return cudaGetLastError();
    }
    dim3 grid((nz + 127) / 128, ny, nx);
    if (exact)
        fmig_freq_kernel<true><<<grid, 128, 0, s>>>(ps, pr, img, fq, fq + g4, fq + 2 * g4, fq + 3 * g4, f, g, nx, ny, nz);
    else
        fmig_freq_kernel<false><<<grid, 128, 0, s>>>(ps, pr, img, fq, fq + g4, fq + 2 * g4, fq + 3 * g4, f, g, nx, ny, nz);
    return cudaGetLastError();
}

}  // namespace rtmb
