// ops.cuh -- the small per-operator kernels of librtm3d_b200 (one launch per reference operator).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "stencil.cuh"

namespace rtmb {

struct Geom {
    int nxe, nye, nze, blen, h;
};

struct RcvGeom {
    int rx0, ry0, rz;   // padded coordinates of receiver (0, 0)
    int rdx, rdy, rcx, rcy;
    int ntstep;
};

// taper3D / taperUpper3D in place (RTMCPUPlatform.cpp:566-920); upper != 0 for the upper form.
cudaError_t launch_taper(float *P, const float *taper, const Geom &g, int upper, int quirk, cudaStream_t s);
// The same on up to four fields of one geometry in one launch.
cudaError_t launch_taper_fields(float *const *fields, int nf, const float *taper, const Geom &g, int upper, int quirk,
                                cudaStream_t s);
// PP[x, y, z] += wavelet[it] (padded coordinates; RTMCPUPlatform.cpp:103-113).
cudaError_t launch_source(float *PP, const float *wavelet, int it, int x, int y, int z, const Geom &g,
                          cudaStream_t s);
// mode 1: rec[i][j][lt] = PP; 2: PP = rec (CPU path); 3: PP += rec (reference GPU kernel).
cudaError_t launch_receivers(float *PP, float *rec, int lt, int mode, const RcvGeom &r, const Geom &g,
                             cudaStream_t s);
// rw 1: upb[lt][x][y][k] = P[x][y][blen-h+k]; rw 0: the reverse (RTMCPUPlatform.cpp:153-189).
cudaError_t launch_upb(float *P, float *upb, int lt, int rw, const Geom &g, cudaStream_t s);
// img += ps * pr on all x, y and z in [z0, z1) (RTMCPUPlatform.cpp:513-540).
cudaError_t launch_image(float *img, const float *ps, const float *pr, int z0, int z1, const Geom &g,
                         cudaStream_t s);
// order-2 Laplacian filter then border removal (RTMGrid.cpp:129-300); c3 = [3][3] coefficients.
cudaError_t launch_filter_remove(const float *img, float *out, const float *c3, const Geom &g, cudaStream_t s);
// acc += img over n floats.
cudaError_t launch_stack(float *acc, const float *img, size_t n, cudaStream_t s);

// Frequency-domain RTM (fmig.cu): one time step of the running DFT of both wavefields and of the
// frequency-domain image for a group of at most kFmigMaxGroup frequencies.  The per-step table
// values (kre = cos(w it), kim = sin(w it), w2 = w^2 for each frequency of the group) travel as
// kernel parameters.  fq holds the four grids [4][nws][nx][ny][nz] (sRe, sIm, rRe, rIm).
constexpr int kFmigMaxGroup = 256;
struct FmigStep {
    int nws;
    float kre[kFmigMaxGroup], kim[kFmigMaxGroup], w2[kFmigMaxGroup];
};
cudaError_t launch_fmig_freq(const float *ps, const float *pr, float *img, float *fq, const FmigStep &f, const Geom &g,
                             int nx, int ny, int nz, bool exact, cudaStream_t s);
// The reference's per-frequency operators one by one (RTMCPUPlatform.cpp:20-64 and :66-102): the
// DFT update of frequency iw into slot lw of the grids ([nws][nx][ny][nz]) from kre/kim[iw][it]
// ([nw][nt]), and img += w2[iw] (sRe rRe - sIm rIm) from slot lw.
cudaError_t launch_fmig_update(const float *ps, const float *pr, float *sre, float *sim, float *rre, float *rim,
                               const float *kre, const float *kim, int it, int iw, int lw, int nt, const Geom &g,
                               int nx, int ny, int nz, cudaStream_t s);
cudaError_t launch_fmig_image(float *img, const float *sre, const float *sim, const float *rre, const float *rim,
                              const float *w2, int iw, int lw, const Geom &g, int nx, int ny, int nz, cudaStream_t s);

// FP64 overloads of the operators above, for the FP64 GPU oracle (same operator sequence and
// multiply order, double arithmetic).
cudaError_t launch_taper(double *P, const float *taper, const Geom &g, int upper, int quirk, cudaStream_t s);
cudaError_t launch_source(double *PP, const float *wavelet, int it, int x, int y, int z, const Geom &g,
                          cudaStream_t s);
cudaError_t launch_receivers(double *PP, float *rec, int lt, int mode, const RcvGeom &r, const Geom &g,
                             cudaStream_t s);
cudaError_t launch_receivers(double *PP, double *rec, int lt, int mode, const RcvGeom &r, const Geom &g,
                             cudaStream_t s);
cudaError_t launch_upb(double *P, double *upb, int lt, int rw, const Geom &g, cudaStream_t s);
cudaError_t launch_image(double *img, const double *ps, const double *pr, int z0, int z1, const Geom &g,
                         cudaStream_t s);

// Increment storage (RTMB_FLAG_STORE_DIFF): from the forward pass's last level p and increment d
// (16-bit, StoreType store, records sp and sd) to the backward pass's start: pout = p - d (record so,
// written here), d = -d in place.  n % 8 == 0.
cudaError_t launch_diff_rewind(int store, const void *p, void *d, void *pout, const ScaleRec *sp, const ScaleRec *sd,
                               ScaleRec *so, size_t n, cudaStream_t s);
// *out = max |x| over n floats.
cudaError_t launch_absmax(const float *x, size_t n, float *out, cudaStream_t s);
// out[0] += sum (a - b)^2, out[1] += sum b^2 over n floats (double accumulators, zero beforehand).
cudaError_t launch_sqdiff(const float *a, const float *b, size_t n, double *out, cudaStream_t s);
// *out = max amax over n scale records.
cudaError_t launch_scale_max(const ScaleRec *r, int n, float *out, cudaStream_t s);
// out = (float) a over n values.
cudaError_t launch_to_float(const double *a, float *out, size_t n, cudaStream_t s);
// acc += (double) img over n values.
cudaError_t launch_stack64(double *acc, const float *img, size_t n, cudaStream_t s);
// Stacking of a padded shot image (g: its padded geometry; img64: doubles, else floats) without
// its border into a survey volume (snx, sny, snz) of doubles at origin (ox, oy, oz).
cudaError_t launch_stack_region64(double *stack, int snx, int sny, int snz, const void *img, bool img64,
                                  const Geom &g, int ox, int oy, int oz, cudaStream_t s);

}  // namespace rtmb
