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

}  // namespace

cudaError_t launch_fmig_freq(const float *ps, const float *pr, float *img, float *fq, const FmigStep &f, const Geom &g,
                             int nx, int ny, int nz, bool exact, cudaStream_t s) {
    if (f.nws <= 0 || f.nws > kFmigMaxGroup || nx <= 0 || ny <= 0 || nz <= 0 || ny > 65535 || nx > 65535)
        return cudaErrorInvalidValue;
    const size_t g4 = (size_t)f.nws * nx * ny * nz;  // one frequency grid of the group
    dim3 grid((nz + 127) / 128, ny, nx);
    if (exact)
        fmig_freq_kernel<true><<<grid, 128, 0, s>>>(ps, pr, img, fq, fq + g4, fq + 2 * g4, fq + 3 * g4, f, g, nx, ny, nz);
    else
        fmig_freq_kernel<false><<<grid, 128, 0, s>>>(ps, pr, img, fq, fq + g4, fq + 2 * g4, fq + 3 * g4, f, g, nx, ny, nz);
    return cudaGetLastError();
}

}  // namespace rtmb
