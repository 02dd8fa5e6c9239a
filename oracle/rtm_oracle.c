/*
 * rtm_oracle.c -- TEST INFRASTRUCTURE ONLY.  CPU restatement of the reference hot path.
 *
 * Every function cites the reference code it restates (S/ = source/rtm-3d/).  The arithmetic
 * follows the reference's types and evaluation order exactly (float vs double intermediates,
 * summation order, no fused multiply-add: built with -ffp-contract=off), so that results are
 * bit-identical to the reference CPU build on the same inputs; tests/test_oracle_pin.py checks
 * that claim against the reference itself.
 */
#define _DEFAULT_SOURCE
#include "rtm_oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define IDX(x, y, z) ((((size_t)(x)) * (size_t)nye + (size_t)(y)) * (size_t)nze + (size_t)(z))

/* ---------------------------------------------------------------- host-side math */

/* S/src/misc/Misc.cpp:106-137 (makeo2).  In the reference C++ build cos() and pow() on float
 * arguments resolve to the float overloads (cosf, powf). */
static void orc_makeo2(float *coef, int order) {
    float h_beta, alpha1, alpha2, central_term, coef_filt, arg, coef_wind;
    int msign, ix;
    float alpha = .54f;
    float beta = 6.f;
    h_beta = (float)(0.5 * beta);
    alpha1 = (float)(2. * alpha - 1.0);
    alpha2 = (float)(2. * (1.0 - alpha));
    central_term = 0.0f;
    msign = -1;
    for (ix = 1; ix <= order / 2; ix++) {
        msign = -msign;
        coef_filt = (float)((2. * msign) / (ix * ix));
        arg = (float)(M_PI * ix / (2. * (order / 2 + 2)));
        coef_wind = powf(alpha1 + alpha2 * cosf(arg) * cosf(arg), h_beta);
        coef[order / 2 + ix] = coef_filt * coef_wind;
        central_term = central_term + coef[order / 2 + ix];
        coef[order / 2 - ix] = coef[order / 2 + ix];
    }
    coef[order / 2] = (float)(-2. * central_term);
}

/* S/src/misc/Misc.cpp:139-176 (laplacian_coefs): double literals stored as float. */
void orc_laplacian_coefs(int order, float *c) {
    switch (order) {
    case 2: c[0] = 1.f; c[1] = -2.f; c[2] = 1.f; break;
    case 4:
        c[0] = (float)(-1. / 12.); c[1] = (float)(4. / 3.); c[2] = (float)(-5. / 2.);
        c[3] = (float)(4. / 3.); c[4] = (float)(-1. / 12.);
        break;
    case 6:
        c[0] = (float)(1. / 90.); c[1] = (float)(-3. / 20.); c[2] = (float)(3. / 2.);
        c[3] = (float)(-49. / 18.); c[4] = (float)(3. / 2.); c[5] = (float)(-3. / 20.);
        c[6] = (float)(1. / 90.);
        break;
    case 8:
        c[0] = (float)(-1. / 560.); c[1] = (float)(8. / 315.); c[2] = (float)(-1. / 5.);
        c[3] = (float)(8. / 5.); c[4] = (float)(-205. / 72.); c[5] = (float)(8. / 5.);
        c[6] = (float)(-1. / 5.); c[7] = (float)(8. / 315.); c[8] = (float)(-1. / 560.);
        break;
    default: orc_makeo2(c, order);
    }
}

/* S/include/RTMGrid.hpp:433-446 (setStencilCoefficients): devinv computed in double, stored as
 * float, then a float product with the Laplacian coefficient.  out is [3][order+1], x,y,z. */
void orc_stencil_coefs(int order, float dx, float dy, float dz, float *out) {
    float c[64];
    float d[3] = {dx, dy, dz};
    orc_laplacian_coefs(order, c);
    for (int k = 0; k < 3; ++k) {
        float dev = d[k];
        float devinv = (float)((1.0 / dev) * (1.0 / dev));
        for (int io = 0; io <= order; ++io) out[k * (order + 1) + io] = devinv * c[io];
    }
}

/* S/include/RTMSeismic.hpp:294-305 (inittaper).  log/sqrt of a float resolve to the float
 * overloads; pow(float, int) is evaluated in double; exp of that double is double. */
void orc_taper_vector(int blen, float factor, float *out) {
    float dfrac = (float)(sqrtf(-logf(factor)) / (1. * blen));
    for (int i = 0; i < blen; ++i) {
        float a = dfrac * (float)i;
        out[i] = (float)exp(-pow((double)a, 2.0));
    }
}

/* S/include/RTMSeismic.hpp:135-144 and 191-198 (loadSamples, ricker).  t = it*dt - 1/fpeak with
 * it*dt a float product and 1.0/fpeak in double; x is a float; exp(-xx) is the float exp;
 * the bracket (1 - 2xx) is double. */
void orc_ricker(int nt, float dt, float fpeak, float *out) {
    for (int it = 0; it < nt; ++it) {
        float t = (float)((double)((float)it * dt) - 1.0 / fpeak);
        float x = (float)(M_PI * fpeak * t);
        float xx = x * x;
        out[it] = (float)((double)expf(-xx) * (1.0 - 2.0 * xx));
    }
}

/* ---------------------------------------------------------------- velocity preparation */

/* S/src/grid/RTMGrid.cpp:47-86 (extendBorders).  The reference leaves stale data in border
 * cells until initBorders overwrites every one of them; here they start at zero. */
void orc_extend_borders(const float *v, int nx, int ny, int nz, int blen, float *ve) {
    int nxe = nx + 2 * blen, nye = ny + 2 * blen, nze = nz + 2 * blen;
    memset(ve, 0, sizeof(float) * (size_t)nxe * nye * nze);
    for (int x = 0; x < nx; ++x)
        for (int y = 0; y < ny; ++y)
            memcpy(ve + IDX(x + blen, y + blen, blen), v + ((size_t)x * ny + y) * nz,
                   sizeof(float) * nz);
}

static inline int clampi(int i, int blen, int l) {
    if (i <= blen) return blen;
    if (i >= l + blen) return l + blen - 1;
    return i;
}

/* S/src/grid/RTMGrid.cpp:371-434 (initBorders_ABC): edge replication, index <= blen -> blen. */
void orc_init_borders_abc(float *ve, int nxe, int nye, int nze, int blen) {
    int lx = nxe - 2 * blen, ly = nye - 2 * blen, lz = nze - 2 * blen;
    for (int x = 0; x < nxe; ++x)
        for (int y = 0; y < nye; ++y)
            for (int z = 0; z < nze; ++z)
                ve[IDX(x, y, z)] = ve[IDX(clampi(x, blen, lx), clampi(y, blen, ly), clampi(z, blen, lz))];
}

/* S/src/misc/Misc.cpp:91-104 (randlinearval, via randbetween :51-54).  rand() is consumed on
 * every call.  The reference draws from an unseeded libc rand() inside OpenMP loops; with one
 * thread and a common srand() seed the sequence below is the reference's own. */
static float randlinearval(float v, int k, int nkb) {
    float vrand = v;
    float dist = (float)(k * 1.0);
    float range = (float)(nkb * 1.0);
    float perc = (dist / range) * 100;
    float seed = (float)((rand() % 100) * 1.0);
    if (seed < perc && perc > 70.) vrand = (float)(v * (1.0 / perc) + v * (seed / 100.0));
    return vrand;
}

/* S/src/grid/RTMGrid.cpp:437-635 (initBorders_RBC), single-threaded loop order. */
void orc_init_borders_rbc(float *ve, int nxe, int nye, int nze, int blen) {
    int nx = nxe, ny = nye, nz = nze;
    float v0;
    /* top and bottom */
    for (int ix = blen; ix < nx - blen; ix++)
        for (int iy = blen; iy < ny - blen; iy++)
            for (int iz = 0; iz < blen; iz++) {
                int dist = blen - iz;
                v0 = randlinearval(ve[IDX(ix, iy, blen)], dist, blen);
                ve[IDX(ix, iy, iz)] = v0;
                v0 = randlinearval(ve[IDX(ix, iy, nz - blen - 1)], dist, blen);
                ve[IDX(ix, iy, (nz - 1) - iz)] = v0;
            }
    /* left and right */
    for (int ix = blen; ix < nx - blen; ix++)
        for (int iz = blen; iz < nz - blen; iz++)
            for (int iy = 0; iy < blen; iy++) {
                v0 = randlinearval(ve[IDX(ix, blen, iz)], blen - iy, blen);
                ve[IDX(ix, iy, iz)] = v0;
                v0 = randlinearval(ve[IDX(ix, ny - blen - 1, iz)], iy, blen);
                ve[IDX(ix, (ny - blen) + iy, iz)] = v0;
            }
    /* front and back */
    for (int iy = blen; iy < ny - blen; iy++)
        for (int iz = blen; iz < nz - blen; iz++)
            for (int ix = 0; ix < blen; ix++) {
                v0 = randlinearval(ve[IDX(blen, iy, iz)], blen - ix, blen);
                ve[IDX(ix, iy, iz)] = v0;
                v0 = randlinearval(ve[IDX(nx - blen - 1, iy, iz)], ix, blen);
                ve[IDX((nx - blen) + ix, iy, iz)] = v0;
            }
    /* x-z corners and edges */
    for (int ix = 0; ix < blen; ix++)
        for (int iz = 0; iz < blen; iz++)
            for (int iy = 0; iy < ny; iy++) {
                int ky = iy;
                if (iy < blen) ky = blen;
                else if (iy >= ny - blen) ky = ny - blen - 1;
                const int zsrc[4] = {blen, blen, nz - blen - 1, nz - blen - 1};
                const int xsrc[4] = {blen, nx - blen - 1, blen, nx - blen - 1};
                const int xd[4] = {blen - ix, ix, blen - ix, ix};
                const int zd[4] = {blen - iz, blen - iz, iz, iz};
                const int xdst[4] = {ix, (nx - blen) + ix, ix, (nx - blen) + ix};
                const int zdst[4] = {iz, iz, (nz - blen) + iz, (nz - blen) + iz};
                for (int c = 0; c < 4; ++c) {
                    v0 = ve[IDX(xsrc[c], ky, zsrc[c])];
                    if (iy < blen) v0 = randlinearval(v0, blen - iy, blen);
                    else if (iy >= ny - blen) v0 = randlinearval(v0, iy - (ny - blen), blen);
                    v0 = randlinearval(v0, xd[c], blen);
                    v0 = randlinearval(v0, zd[c], blen);
                    ve[IDX(xdst[c], iy, zdst[c])] = v0;
                }
            }
    /* y-z edges */
    for (int iy = 0; iy < blen; iy++)
        for (int iz = 0; iz < blen; iz++)
            for (int ix = blen; ix < nx - blen; ix++) {
                const int ysrc[4] = {blen, ny - blen - 1, blen, ny - blen - 1};
                const int zsrc[4] = {blen, blen, nz - blen - 1, nz - blen - 1};
                const int yd[4] = {blen - iy, iy, blen - iy, iy};
                const int zd[4] = {blen - iz, blen - iz, iz, iz};
                const int ydst[4] = {iy, (ny - blen) + iy, iy, (ny - blen) + iy};
                const int zdst[4] = {iz, iz, (nz - blen) + iz, (nz - blen) + iz};
                for (int c = 0; c < 4; ++c) {
                    v0 = ve[IDX(ix, ysrc[c], zsrc[c])];
                    v0 = randlinearval(v0, yd[c], blen);
                    v0 = randlinearval(v0, zd[c], blen);
                    ve[IDX(ix, ydst[c], zdst[c])] = v0;
                }
            }
    /* x-y edges */
    for (int ix = 0; ix < blen; ix++)
        for (int iy = 0; iy < blen; iy++)
            for (int iz = blen; iz < nz - blen; iz++) {
                const int xsrc[4] = {blen, blen, nx - blen - 1, nx - blen - 1};
                const int ysrc[4] = {blen, ny - blen - 1, blen, ny - blen - 1};
                const int xd[4] = {blen - ix, blen - ix, ix, ix};
                const int yd[4] = {blen - iy, iy, blen - iy, iy};
                const int xdst[4] = {ix, ix, (nx - blen) + ix, (nx - blen) + ix};
                const int ydst[4] = {iy, (ny - blen) + iy, iy, (ny - blen) + iy};
                for (int c = 0; c < 4; ++c) {
                    v0 = ve[IDX(xsrc[c], ysrc[c], iz)];
                    v0 = randlinearval(v0, xd[c], blen);
                    v0 = randlinearval(v0, yd[c], blen);
                    ve[IDX(xdst[c], ydst[c], iz)] = v0;
                }
            }
}

/* S/src/grid/RTMGrid.cpp:638-696 (initBorders_HBC): ABC, RBC, then the top blen planes
 * replicated from z = blen with clamped x, y. */
void orc_init_borders_hbc(float *ve, int nxe, int nye, int nze, int blen) {
    int lx = nxe - 2 * blen, ly = nye - 2 * blen;
    orc_init_borders_abc(ve, nxe, nye, nze, blen);
    orc_init_borders_rbc(ve, nxe, nye, nze, blen);
    for (int x = 0; x < nxe; ++x)
        for (int y = 0; y < nye; ++y)
            for (int z = 0; z < blen; ++z)
                ve[IDX(x, y, z)] = ve[IDX(clampi(x, blen, lx), clampi(y, blen, ly), blen)];
}

/* S/src/controller/RTMController.cpp:110-111 (power2, multiplyBy(dt*dt)); S/include/Grid.hpp:212-235.
 * dt*dt is a float product. */
void orc_v2dt2(float *v, size_t n, float dt) {
    float dt2 = dt * dt;
    for (size_t i = 0; i < n; ++i) v[i] *= v[i];
    for (size_t i = 0; i < n; ++i) v[i] *= dt2;
}

/* ---------------------------------------------------------------- per-step operators */

/* S/src/platform/host/RTMCPUPlatform.cpp:325-395 (rtmStep3D): interior [h, n-h) on all axes,
 * acmx, acmy, acmz accumulated in io order from 0.0, lapl = acmx + acmy + acmz,
 * PP = 2*p - pp + v2dt2*lapl in place.  Returns 1 if a NaN was met (the reference throws). */
int orc_step(int nxe, int nye, int nze, int order, const float *coefs,
             const float *P, float *PP, const float *v2dt2) {
    const int h = order / 2;
    const float *cx = coefs, *cy = coefs + (order + 1), *cz = coefs + 2 * (order + 1);
    int nan = 0;
#pragma omp parallel for collapse(2) reduction(| : nan)
    for (int ix = h; ix < nxe - h; ix++)
        for (int iy = h; iy < nye - h; iy++)
            for (int iz = h; iz < nze - h; iz++) {
                float acmx = 0.0f, acmy = 0.0f, acmz = 0.0f, lapl;
                for (int io = 0; io <= order; io++) {
                    acmx += P[IDX(ix - h + io, iy, iz)] * cx[io];
                    acmy += P[IDX(ix, iy - h + io, iz)] * cy[io];
                    acmz += P[IDX(ix, iy, iz - h + io)] * cz[io];
                }
                lapl = acmx + acmy + acmz;
                size_t o = IDX(ix, iy, iz);
                float pp = PP[o], p = P[o], v = v2dt2[o];
                float npp = 2 * p - pp + (v)*lapl;
                PP[o] = npp;
                if (npp != npp || p != p || pp != pp || lapl != lapl) nan = 1;
            }
    return nan;
}

/* S/src/platform/host/RTMCPUPlatform.cpp:191-256 (rtmStep2D; rtmStep picks it when nx == 1, :474-490):
 * only the plane x = blen, the y and z terms of the Laplacian, lapl = acmy + acmz. */
int orc_step2d(int nxe, int nye, int nze, int blen, int order, const float *coefs,
               const float *P, float *PP, const float *v2dt2) {
    const int h = order / 2, ix = blen;
    const float *cy = coefs + (order + 1), *cz = coefs + 2 * (order + 1);
    int nan = 0;
    (void)nxe;
#pragma omp parallel for collapse(2) reduction(| : nan)
    for (int iy = h; iy < nye - h; iy++)
        for (int iz = h; iz < nze - h; iz++) {
            float acmy = 0.0f, acmz = 0.0f, lapl;
            for (int io = 0; io <= order; io++) {
                acmy += P[IDX(ix, iy - h + io, iz)] * cy[io];
                acmz += P[IDX(ix, iy, iz - h + io)] * cz[io];
            }
            lapl = acmy + acmz;
            size_t o = IDX(ix, iy, iz);
            float pp = PP[o], p = P[o], v = v2dt2[o];
            float npp = 2 * p - pp + (v)*lapl;
            PP[o] = npp;
            if (npp != npp || p != p || pp != pp || lapl != lapl) nan = 1;
        }
    return nan;
}

/* S/src/platform/host/RTMCPUPlatform.cpp:710-920 (taper3D).  The six loops run in the
 * reference's order; the "front-right" x-y edge reads its value from x = blen (:901), which
 * the left/right loop has already tapered. */
void orc_taper_all(int nxe, int nye, int nze, int blen, const float *t, float *g) {
    const int nx = nxe, ny = nye, nz = nze, b = blen;
    /* top and bottom */
#pragma omp parallel for collapse(2)
    for (int ix = b; ix < nx - b; ix++)
        for (int iy = b; iy < ny - b; iy++)
            for (int iz = 0; iz < b; iz++) {
                g[IDX(ix, iy, iz)] *= t[b - 1 - iz];
                g[IDX(ix, iy, (nz - b) + iz)] *= t[iz];
            }
    /* left and right */
#pragma omp parallel for collapse(2)
    for (int ix = b; ix < nx - b; ix++)
        for (int iz = b; iz < nz - b; iz++)
            for (int iy = 0; iy < b; iy++) {
                g[IDX(ix, iy, iz)] *= t[b - 1 - iy];
                g[IDX(ix, (ny - b) + iy, iz)] *= t[iy];
            }
    /* front and back */
#pragma omp parallel for collapse(2)
    for (int iy = b; iy < ny - b; iy++)
        for (int iz = b; iz < nz - b; iz++)
            for (int ix = 0; ix < b; ix++) {
                g[IDX(ix, iy, iz)] *= t[b - 1 - ix];
                g[IDX((nx - b) + ix, iy, iz)] *= t[ix];
            }
    /* x-z corners and edges: y factor first (when in a y border), then x, then z */
#pragma omp parallel for collapse(2)
    for (int ix = 0; ix < b; ix++)
        for (int iz = 0; iz < b; iz++)
            for (int iy = 0; iy < ny; iy++) {
                float ty = 1.0f;
                int yb = 0;
                if (iy < b) { ty = t[b - 1 - iy]; yb = 1; }
                else if (iy >= ny - b) { ty = t[iy - (ny - b)]; yb = 1; }
                const int xs[4] = {ix, (nx - b) + ix, ix, (nx - b) + ix};
                const int zs[4] = {iz, iz, (nz - b) + iz, (nz - b) + iz};
                const float tx[4] = {t[b - 1 - ix], t[ix], t[b - 1 - ix], t[ix]};
                const float tz[4] = {t[b - 1 - iz], t[b - 1 - iz], t[iz], t[iz]};
                for (int c = 0; c < 4; ++c) {
                    float v = g[IDX(xs[c], iy, zs[c])];
                    if (yb) v *= ty;
                    v *= tx[c];
                    v *= tz[c];
                    g[IDX(xs[c], iy, zs[c])] = v;
                }
            }
    /* y-z edges */
#pragma omp parallel for collapse(2)
    for (int iy = 0; iy < b; iy++)
        for (int iz = 0; iz < b; iz++)
            for (int ix = b; ix < nx - b; ix++) {
                const int ys[4] = {iy, (ny - b) + iy, iy, (ny - b) + iy};
                const int zs[4] = {iz, iz, (nz - b) + iz, (nz - b) + iz};
                const float ty[4] = {t[b - 1 - iy], t[iy], t[b - 1 - iy], t[iy]};
                const float tz[4] = {t[b - 1 - iz], t[b - 1 - iz], t[iz], t[iz]};
                for (int c = 0; c < 4; ++c) {
                    float v = g[IDX(ix, ys[c], zs[c])];
                    v *= ty[c];
                    v *= tz[c];
                    g[IDX(ix, ys[c], zs[c])] = v;
                }
            }
    /* x-y edges; front-right takes its value from x = blen */
#pragma omp parallel for collapse(2)
    for (int ix = 0; ix < b; ix++)
        for (int iy = 0; iy < b; iy++)
            for (int iz = b; iz < nz - b; iz++) {
                float v;
                v = g[IDX(ix, iy, iz)];
                v *= t[b - 1 - ix]; v *= t[b - 1 - iy];
                g[IDX(ix, iy, iz)] = v;
                v = g[IDX(b, (ny - b) + iy, iz)];
                v *= t[b - 1 - ix]; v *= t[iy];
                g[IDX(ix, (ny - b) + iy, iz)] = v;
                v = g[IDX((nx - b) + ix, iy, iz)];
                v *= t[ix]; v *= t[b - 1 - iy];
                g[IDX((nx - b) + ix, iy, iz)] = v;
                v = g[IDX((nx - b) + ix, (ny - b) + iy, iz)];
                v *= t[ix]; v *= t[iy];
                g[IDX((nx - b) + ix, (ny - b) + iy, iz)] = v;
            }
}

/* S/src/platform/host/RTMCPUPlatform.cpp:566-657 (taperUpper3D). */
void orc_taper_upper(int nxe, int nye, int nze, int blen, const float *t, float *g) {
    const int nx = nxe, ny = nye, b = blen;
    (void)nze;
#pragma omp parallel for collapse(2)
    for (int ix = b; ix < nx - b; ix++)
        for (int iy = b; iy < ny - b; iy++)
            for (int iz = 0; iz < b; iz++) g[IDX(ix, iy, iz)] *= t[b - 1 - iz];
#pragma omp parallel for collapse(2)
    for (int ix = 0; ix < b; ix++)
        for (int iz = 0; iz < b; iz++)
            for (int iy = 0; iy < ny; iy++) {
                float ty = 1.0f;
                int yb = 0;
                if (iy < b) { ty = t[b - 1 - iy]; yb = 1; }
                else if (iy >= ny - b) { ty = t[iy - (ny - b)]; yb = 1; }
                float v = g[IDX(ix, iy, iz)];
                if (yb) v *= ty;
                v *= t[b - 1 - ix]; v *= t[b - 1 - iz];
                g[IDX(ix, iy, iz)] = v;
                v = g[IDX(nx - b + ix, iy, iz)];
                if (yb) v *= ty;
                v *= t[ix]; v *= t[b - 1 - iz];
                g[IDX(nx - b + ix, iy, iz)] = v;
            }
#pragma omp parallel for collapse(2)
    for (int iy = 0; iy < b; iy++)
        for (int iz = 0; iz < b; iz++)
            for (int ix = b; ix < nx - b; ix++) {
                float v = g[IDX(ix, iy, iz)];
                v *= t[b - 1 - iy]; v *= t[b - 1 - iz];
                g[IDX(ix, iy, iz)] = v;
                v = g[IDX(ix, ny - b + iy, iz)];
                v *= t[iy]; v *= t[b - 1 - iz];
                g[IDX(ix, ny - b + iy, iz)] = v;
            }
}

/* S/src/platform/host/RTMCPUPlatform.cpp:103-113 and S/src/grid/RTMGrid.cpp:36-40.
 * (x, y, z) are padded coordinates. */
void orc_apply_source(int nxe, int nye, int nze, int x, int y, int z, float val, float *PP) {
    (void)nxe;
    PP[IDX(x, y, z)] = PP[IDX(x, y, z)] + val;
}

/* S/src/platform/host/RTMCPUPlatform.cpp:133-151.  rec chunk is [rcx][rcy][ntstep]. */
void orc_save_receivers(const orc_params *p, int lt, const float *PP, float *rec) {
    int b = p->blen, nye = p->ny + 2 * b, nze = p->nz + 2 * b, nxe = p->nx + 2 * b;
    for (int ix = 0; ix < p->rcx; ix++)
        for (int iy = 0; iy < p->rcy; iy++) {
            int rx = p->rsx + ix * p->rdx + b, ry = p->rsy + iy * p->rdy + b, rz = p->rdz + b;
            if (rx >= 0 && rx < nxe && ry >= 0 && ry < nye)
                rec[((size_t)ix * p->rcy + iy) * p->ntstep + lt] = PP[IDX(rx, ry, rz)];
        }
}

/* S/src/platform/host/RTMCPUPlatform.cpp:114-131: the CPU path OVERWRITES the receiver cell. */
void orc_restore_receivers(const orc_params *p, int lt, float *PP, const float *rec) {
    int b = p->blen, nye = p->ny + 2 * b, nze = p->nz + 2 * b, nxe = p->nx + 2 * b;
    for (int ix = 0; ix < p->rcx; ix++)
        for (int iy = 0; iy < p->rcy; iy++) {
            int rx = p->rsx + ix * p->rdx + b, ry = p->rsy + iy * p->rdy + b, rz = p->rdz + b;
            if (rx >= 0 && rx < nxe && ry >= 0 && ry < nye)
                PP[IDX(rx, ry, rz)] = rec[((size_t)ix * p->rcy + iy) * p->ntstep + lt];
        }
}

/* S/src/platform/host/RTMCPUPlatform.cpp:153-189.  upb is [ntstep][nxe][nye][h] holding
 * z in [blen-h, blen). */
void orc_save_upb(int nxe, int nye, int nze, int blen, int h, int lt, const float *P, float *upb) {
    for (int x = 0; x < nxe; ++x)
        for (int y = 0; y < nye; ++y)
            for (int z = blen - h; z < blen; ++z)
                upb[(((size_t)lt * nxe + x) * nye + y) * h + (z - (blen - h))] = P[IDX(x, y, z)];
}

void orc_restore_upb(int nxe, int nye, int nze, int blen, int h, int lt, float *P, const float *upb) {
    for (int x = 0; x < nxe; ++x)
        for (int y = 0; y < nye; ++y)
            for (int z = blen - h; z < blen; ++z)
                P[IDX(x, y, z)] = upb[(((size_t)lt * nxe + x) * nye + y) * h + (z - (blen - h))];
}

/* S/src/platform/host/RTMCPUPlatform.cpp:513-540: IMG += PS*PR for all x, y and
 * z in [blen, nze-blen). */
void orc_image(int nxe, int nye, int nze, int blen, float *img, const float *ps, const float *pr) {
#pragma omp parallel for collapse(2)
    for (int x = 0; x < nxe; ++x)
        for (int y = 0; y < nye; ++y)
            for (int z = blen; z < nze - blen; ++z) {
                size_t o = IDX(x, y, z);
                img[o] = img[o] + (ps[o] * pr[o]);
            }
}

/* ---------------------------------------------------------------- image finalisation */

/* S/src/grid/RTMGrid.cpp:226-300 (filter with the order-2 stencil, RTM_LAPFILTER_ORDER at
 * S/include/RTMBase.hpp:14) followed by :129-166 (removeBorders).  The reference leaves the
 * outermost cells of the filtered cube uninitialised; removeBorders discards them (blen >= 1). */
void orc_filter_remove(int nxe, int nye, int nze, int blen, float dx, float dy, float dz,
                       const float *img, float *out) {
    float c[9];
    orc_stencil_coefs(2, dx, dy, dz, c);
    const float *cx = c, *cy = c + 3, *cz = c + 6;
    int nx = nxe - 2 * blen, ny = nye - 2 * blen, nz = nze - 2 * blen;
#pragma omp parallel for collapse(2)
    for (int x = 0; x < nx; ++x)
        for (int y = 0; y < ny; ++y)
            for (int z = 0; z < nz; ++z) {
                int ix = x + blen, iy = y + blen, iz = z + blen;
                float acmx = 0.0f, acmy = 0.0f, acmz = 0.0f;
                for (int io = 0; io <= 2; ++io) {
                    acmx += img[IDX(ix - 1 + io, iy, iz)] * cx[io];
                    acmy += img[IDX(ix, iy - 1 + io, iz)] * cy[io];
                    acmz += img[IDX(ix, iy, iz - 1 + io)] * cz[io];
                }
                out[((size_t)x * ny + y) * nz + z] = acmx + acmy + acmz;
            }
}

/* ---------------------------------------------------------------- time loops */

typedef struct {
    int nxe, nye, nze, h;
    size_t n;
    float coefs[3 * 17];
    float *taper, *wavelet;
} loopctx;

static int loop_init(const orc_params *p, loopctx *c) {
    if (p->ntstep <= 0 || p->nt % p->ntstep != 0 || p->order < 2 || p->order > 16) return 2;
    c->nxe = p->nx + 2 * p->blen;
    c->nye = p->ny + 2 * p->blen;
    c->nze = p->nz + 2 * p->blen;
    c->h = p->order / 2;
    c->n = (size_t)c->nxe * c->nye * c->nze;
    orc_stencil_coefs(p->order, p->dx, p->dy, p->dz, c->coefs);
    c->taper = (float *)malloc(sizeof(float) * (p->blen > 0 ? p->blen : 1));
    c->wavelet = (float *)malloc(sizeof(float) * p->nt);
    if (p->blen > 0) orc_taper_vector(p->blen, p->taper_factor, c->taper);
    orc_ricker(p->nt, p->dt, p->fpeak, c->wavelet);
    return 0;
}

static void loop_free(loopctx *c) { free(c->taper); free(c->wavelet); }

#define SWAP(a, b) do { float *t_ = a; a = b; b = t_; } while (0)

/* rtmStep of the loops: the 2D form for nx == 1 (RTMCPUPlatform.cpp:474-490). */
static int step(const orc_params *p, const loopctx *c, const float *P, float *PP, const float *v2dt2) {
    if (p->nx == 1) return orc_step2d(c->nxe, c->nye, c->nze, p->blen, p->order, c->coefs, P, PP, v2dt2);
    return orc_step(c->nxe, c->nye, c->nze, p->order, c->coefs, P, PP, v2dt2);
}

/* S/src/kernel/RTMFiniteDifferencesKernel.cpp:129-246 (rtmAcousticFiniteDiffModeling). */
int orc_model_shot(const orc_params *p, const float *v2dt2, float *rec) {
    loopctx c;
    int rc = loop_init(p, &c), nan = 0;
    if (rc) return rc;
    float *P = (float *)calloc(c.n, sizeof(float)), *PP = (float *)calloc(c.n, sizeof(float));
    size_t chunk = (size_t)p->rcx * p->rcy * p->ntstep;
    int sx = p->sx + p->blen, sy = p->sy + p->blen, sz = p->sz + p->blen;
    for (int itstep = 0; itstep < p->nt; itstep += p->ntstep) {
        float *rchunk = rec + (size_t)(itstep / p->ntstep) * chunk;
        for (int lt = 0; lt < p->ntstep; ++lt) {
            int it = itstep + lt;
            SWAP(P, PP);
            orc_taper_all(c.nxe, c.nye, c.nze, p->blen, c.taper, P);
            orc_taper_all(c.nxe, c.nye, c.nze, p->blen, c.taper, PP);
            nan |= step(p, &c, P, PP, v2dt2);
            orc_apply_source(c.nxe, c.nye, c.nze, sx, sy, sz, c.wavelet[it], PP);
            orc_save_receivers(p, lt, PP, rchunk);
        }
    }
    free(P); free(PP); loop_free(&c);
    return nan;
}

/* Forward pass of S/src/kernel/RTMFiniteDifferencesKernel_HBC.cpp:96-210 (hbc = 1, keeps the
 * upper-border planes in upb[nt][nxe][nye][h]) and of ..._RBC.cpp:54-144 (hbc = 0).
 * On return snap0 = P, snap1 = PP (the last two source wavefields). */
static int forward(const orc_params *p, loopctx *c, const float *v2dt2, int hbc,
                   float *upb, float *snap0, float *snap1) {
    float *P = (float *)calloc(c->n, sizeof(float)), *PP = (float *)calloc(c->n, sizeof(float));
    int sx = p->sx + p->blen, sy = p->sy + p->blen, sz = p->sz + p->blen, nan = 0;
    for (int it = 0; it < p->nt; ++it) {
        SWAP(P, PP);
        if (hbc) {
            orc_taper_upper(c->nxe, c->nye, c->nze, p->blen, c->taper, P);
            orc_taper_upper(c->nxe, c->nye, c->nze, p->blen, c->taper, PP);
        }
        nan |= step(p, c, P, PP, v2dt2);
        orc_apply_source(c->nxe, c->nye, c->nze, sx, sy, sz, c->wavelet[it], PP);
        if (hbc) orc_save_upb(c->nxe, c->nye, c->nze, p->blen, c->h, it, PP, upb);
    }
    memcpy(snap0, P, c->n * sizeof(float));
    memcpy(snap1, PP, c->n * sizeof(float));
    free(P); free(PP);
    return nan;
}

/* Backward pass of ..._HBC.cpp:212-364 (hbc = 1) and ..._RBC.cpp:146-274 (hbc = 0). */
static int backward(const orc_params *p, loopctx *c, const float *v2dt2, int hbc,
                    const float *upb, const float *snap0, const float *snap1,
                    const float *rec, float *img) {
    float *P = (float *)calloc(c->n, sizeof(float)), *PP = (float *)calloc(c->n, sizeof(float));
    float *PR = (float *)calloc(c->n, sizeof(float)), *PPR = (float *)calloc(c->n, sizeof(float));
    size_t chunk = (size_t)p->rcx * p->rcy * p->ntstep;
    int nan = 0;
    memset(img, 0, c->n * sizeof(float));
    for (int itstep = p->nt - p->ntstep; itstep >= 0; itstep -= p->ntstep) {
        const float *rchunk = rec + (size_t)(itstep / p->ntstep) * chunk;
        for (int lt = p->ntstep - 1; lt >= 0; --lt) {
            int it = itstep + lt;
            if (it == p->nt - 1) memcpy(PP, snap1, c->n * sizeof(float));
            else if (it == p->nt - 2) memcpy(PP, snap0, c->n * sizeof(float));
            else {
                nan |= step(p, c, P, PP, v2dt2);
                if (hbc) orc_restore_upb(c->nxe, c->nye, c->nze, p->blen, c->h, it, PP, upb);
            }
            SWAP(P, PP);
            if (hbc) {
                orc_taper_upper(c->nxe, c->nye, c->nze, p->blen, c->taper, PR);
                orc_taper_upper(c->nxe, c->nye, c->nze, p->blen, c->taper, PPR);
            }
            nan |= step(p, c, PR, PPR, v2dt2);
            orc_restore_receivers(p, lt, PPR, rchunk);
            orc_image(c->nxe, c->nye, c->nze, p->blen, img, P, PPR);
            SWAP(PR, PPR);
        }
    }
    free(P); free(PP); free(PR); free(PPR);
    return nan;
}

static int migrate(const orc_params *p, const float *v2dt2, const float *rec, float *img, int hbc) {
    loopctx c;
    int rc = loop_init(p, &c);
    if (rc) return rc;
    float *upb = NULL;
    if (hbc) upb = (float *)calloc((size_t)p->nt * c.nxe * c.nye * c.h, sizeof(float));
    float *s0 = (float *)malloc(c.n * sizeof(float)), *s1 = (float *)malloc(c.n * sizeof(float));
    int nan = forward(p, &c, v2dt2, hbc, upb, s0, s1);
    nan |= backward(p, &c, v2dt2, hbc, upb, s0, s1, rec, img);
    free(s0); free(s1); free(upb); loop_free(&c);
    return nan;
}

/* S/src/kernel/RTMFiniteDifferencesKernel_HBC.cpp:64-94 (rtmMigrate). */
int orc_migrate_hbc(const orc_params *p, const float *v2dt2, const float *rec, float *img) {
    return migrate(p, v2dt2, rec, img, 1);
}

/* S/src/kernel/RTMFiniteDifferencesKernel_RBC.cpp:36-51 (rtmMigrate). */
int orc_migrate_rbc(const orc_params *p, const float *v2dt2, const float *rec, float *img) {
    return migrate(p, v2dt2, rec, img, 0);
}

/* ---------------------------------------------------------------- frequency-domain RTM (fmig) */

/* S/src/kernel/RTMFiniteDifferencesKernel_FreqDomain.cpp:133-137: df = 1 / (nt dt) and
 * nw = (size_t)((fmax - fmin) / df), in the reference's float / double mix. */
int orc_fmig_nw(int nt, float dt, float fmin, float fmax) {
    const float df = (float)(1. / ((nt * 1.0) * dt));
    const float nf = ((fmax - fmin) / df);
    return nf > 0.f ? (int)(size_t)nf : 0;
}

/* ..._FreqDomain.cpp:17-51 and :151-156: the angular frequencies per time step
 * w[iw] = 2 pi (iw df + fmin) dt, the DFT kernels kre/kim[iw][it] = cos/sin(w[iw] it), and w2 = w^2
 * (wList->power2()). */
void orc_fmig_tables(int nt, float dt, float fmin, float fmax, int nw, float *w2, float *kre, float *kim) {
    const float df = (float)(1. / ((nt * 1.0) * dt));
    (void)fmax;
    const float pi = acosf(-1.);
    for (int iw = 0; iw < nw; ++iw) {
        const float lw = (float)iw * 1.0;
        const float w = (float)(2. * pi * ((lw * df) + fmin) * dt);
        for (int it = 0; it < nt; ++it) {
            kre[(size_t)iw * nt + it] = cosf((float)(w * (it * 1.0)));
            kim[(size_t)iw * nt + it] = sinf((float)(w * (it * 1.0)));
        }
        w2[iw] = w * w;
    }
}

/* ..._FreqDomain.cpp:220-357 (rtmFreqDomainPropagation) with the CPU platform's operators
 * (S/src/platform/host/RTMCPUPlatform.cpp:20-102, :397-472).  Both wavefields advance together
 * in forward time st = nt-1-rt: the source one from the Ricker wavelet, the receiver one from the
 * record read backwards (rt).  Each step: the two steps, the taper of all four fields, the source,
 * the receivers (overwritten), then for every frequency of the group the running DFT of both
 * fields over the model interior and img += w2 (sRe rRe - sIm rIm) with the running sums.
 * nwstep: frequencies per pass over time (0: all nw in one pass, the CPU build's choice,
 * ..._FreqDomain.cpp:139-149).  img: padded volume, zeroed here (one shot). */
int orc_migrate_fmig(const orc_params *p, const float *v2dt2, const float *rec, float fmin, float fmax, int nwstep,
                     float *img) {
    loopctx c;
    int rc = loop_init(p, &c), nan = 0;
    if (rc) return rc;
    const int nw = orc_fmig_nw(p->nt, p->dt, fmin, fmax);
    if (nwstep <= 0 || nwstep > nw) nwstep = nw;
    const int nxe = c.nxe, nye = c.nye, nze = c.nze, b = p->blen, nx = p->nx, ny = p->ny, nz = p->nz;
    const size_t ni = (size_t)nx * ny * nz;
    float *w2 = (float *)malloc(sizeof(float) * (nw > 0 ? nw : 1));
    float *kre = (float *)malloc(sizeof(float) * (size_t)(nw > 0 ? nw : 1) * p->nt);
    float *kim = (float *)malloc(sizeof(float) * (size_t)(nw > 0 ? nw : 1) * p->nt);
    orc_fmig_tables(p->nt, p->dt, fmin, fmax, nw, w2, kre, kim);
    float *P = (float *)calloc(c.n, sizeof(float)), *PP = (float *)calloc(c.n, sizeof(float));
    float *PR = (float *)calloc(c.n, sizeof(float)), *PPR = (float *)calloc(c.n, sizeof(float));
    float *sRe = (float *)calloc(ni * (nwstep > 0 ? nwstep : 1), sizeof(float));
    float *sIm = (float *)calloc(ni * (nwstep > 0 ? nwstep : 1), sizeof(float));
    float *rRe = (float *)calloc(ni * (nwstep > 0 ? nwstep : 1), sizeof(float));
    float *rIm = (float *)calloc(ni * (nwstep > 0 ? nwstep : 1), sizeof(float));
    const size_t chunk = (size_t)p->rcx * p->rcy * p->ntstep;
    const int sx = p->sx + b, sy = p->sy + b, sz = p->sz + b;
    memset(img, 0, c.n * sizeof(float));
    for (int gw = 0; gw < nw; gw += nwstep) {
        memset(P, 0, c.n * sizeof(float)); memset(PP, 0, c.n * sizeof(float));
        memset(PR, 0, c.n * sizeof(float)); memset(PPR, 0, c.n * sizeof(float));
        memset(sRe, 0, ni * nwstep * sizeof(float)); memset(sIm, 0, ni * nwstep * sizeof(float));
        memset(rRe, 0, ni * nwstep * sizeof(float)); memset(rIm, 0, ni * nwstep * sizeof(float));
        for (int itstep = p->nt - p->ntstep; itstep >= 0; itstep -= p->ntstep) {
            const float *rchunk = rec + (size_t)(itstep / p->ntstep) * chunk;
            for (int lt = p->ntstep - 1; lt >= 0; --lt) {
                const int rt = itstep + lt, st = p->nt - 1 - rt;
                nan |= step(p, &c, P, PP, v2dt2);
                nan |= step(p, &c, PR, PPR, v2dt2);
                orc_taper_all(nxe, nye, nze, b, c.taper, P);
                orc_taper_all(nxe, nye, nze, b, c.taper, PP);
                orc_taper_all(nxe, nye, nze, b, c.taper, PR);
                orc_taper_all(nxe, nye, nze, b, c.taper, PPR);
                orc_apply_source(nxe, nye, nze, sx, sy, sz, c.wavelet[st], PP);
                orc_restore_receivers(p, lt, PPR, rchunk);
                for (int lw = 0, iw = gw; lw < nwstep && iw < nw; ++lw, ++iw) {
                    const float kr = kre[(size_t)iw * p->nt + st], ki = kim[(size_t)iw * p->nt + st];
                    const float w2v = w2[iw];
                    float *fr = sRe + lw * ni, *fi = sIm + lw * ni, *gr = rRe + lw * ni, *gi = rIm + lw * ni;
#pragma omp parallel for collapse(2)
                    for (int ix = 0; ix < nx; ++ix)
                        for (int iy = 0; iy < ny; ++iy) {
                            size_t o = IDX(ix + b, iy + b, b), f = ((size_t)ix * ny + iy) * nz;
                            for (int iz = 0; iz < nz; ++iz, ++o, ++f) {
                                const float ps = PP[o], pr = PPR[o];
                                fr[f] += (kr * ps);
                                fi[f] += (ki * ps);
                                gr[f] += (kr * pr);
                                gi[f] += (ki * pr);
                            }
                        }
#pragma omp parallel for collapse(2)
                    for (int ix = 0; ix < nx; ++ix)
                        for (int iy = 0; iy < ny; ++iy) {
                            size_t o = IDX(ix + b, iy + b, b), f = ((size_t)ix * ny + iy) * nz;
                            for (int iz = 0; iz < nz; ++iz, ++o, ++f)
                                img[o] += (w2v) * (fr[f] * gr[f] - fi[f] * gi[f]);
                        }
                }
                SWAP(P, PP);
                SWAP(PR, PPR);
            }
        }
    }
    free(P); free(PP); free(PR); free(PPR); free(sRe); free(sIm); free(rRe); free(rIm);
    free(w2); free(kre); free(kim); loop_free(&c);
    return nan;
}
