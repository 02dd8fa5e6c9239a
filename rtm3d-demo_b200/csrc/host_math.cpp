// host_math.cpp -- host-side tables and velocity preparation.  These are the reference's own
// host computations (it runs them on the CPU in its GPU build as well); every result is
// bit-identical to the reference, which the test-suite checks.
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "host_math.hpp"
#include "rtm3d_b200.h"

namespace {

// Misc.cpp:106-137 (makeo2): windowed coefficients for orders other than 2/4/6/8.  On float
// arguments cos and pow are the float overloads.
void makeo2(float *coef, int order) {
    const float alpha = .54f, beta = 6.f;
    const float h_beta = static_cast<float>(0.5 * beta);
    const float alpha1 = static_cast<float>(2. * alpha - 1.0);
    const float alpha2 = static_cast<float>(2. * (1.0 - alpha));
    float central = 0.0f;
    int msign = -1;
    for (int ix = 1; ix <= order / 2; ix++) {
        msign = -msign;
        const float coef_filt = static_cast<float>((2. * msign) / (ix * ix));
        const float arg = static_cast<float>(M_PI * ix / (2. * (order / 2 + 2)));
        const float c = std::cos(arg);
        const float coef_wind = std::pow(alpha1 + alpha2 * c * c, h_beta);
        coef[order / 2 + ix] = coef_filt * coef_wind;
        central = central + coef[order / 2 + ix];
        coef[order / 2 - ix] = coef[order / 2 + ix];
    }
    coef[order / 2] = static_cast<float>(-2. * central);
}

// Misc.cpp:139-176 (laplacian_coefs).
void laplacian(float *c, int order) {
    switch (order) {
    case 2: c[0] = 1.f; c[1] = -2.f; c[2] = 1.f; return;
    case 4: {
        const double k[5] = {-1. / 12., 4. / 3., -5. / 2., 4. / 3., -1. / 12.};
        for (int i = 0; i < 5; ++i) c[i] = static_cast<float>(k[i]);
        return;
    }
    case 6: {
        const double k[7] = {1. / 90., -3. / 20., 3. / 2., -49. / 18., 3. / 2., -3. / 20., 1. / 90.};
        for (int i = 0; i < 7; ++i) c[i] = static_cast<float>(k[i]);
        return;
    }
    case 8: {
        const double k[9] = {-1. / 560., 8. / 315., -1. / 5., 8. / 5., -205. / 72.,
                             8. / 5.,    -1. / 5.,   8. / 315., -1. / 560.};
        for (int i = 0; i < 9; ++i) c[i] = static_cast<float>(k[i]);
        return;
    }
    default: makeo2(c, order);
    }
}

inline size_t at(int x, int y, int z, int nye, int nze) {
    return (static_cast<size_t>(x) * nye + y) * nze + z;
}

inline int clampi(int i, int b, int l) { return i <= b ? b : (i >= l + b ? l + b - 1 : i); }

// Misc.cpp:91-104 (randlinearval): one rand() per call.
float randlinear(float v, int k, int nkb) {
    const float dist = static_cast<float>(k * 1.0);
    const float range = static_cast<float>(nkb * 1.0);
    const float perc = (dist / range) * 100;
    const float seed = static_cast<float>((rand() % 100) * 1.0);
    if (seed < perc && perc > 70.) return static_cast<float>(v * (1.0 / perc) + v * (seed / 100.0));
    return v;
}

// RTMGrid.cpp:371-434 (initBorders_ABC).
void borders_abc(float *ve, int nxe, int nye, int nze, int b) {
    const int lx = nxe - 2 * b, ly = nye - 2 * b, lz = nze - 2 * b;
    for (int x = 0; x < nxe; ++x)
        for (int y = 0; y < nye; ++y)
            for (int z = 0; z < nze; ++z)
                ve[at(x, y, z, nye, nze)] = ve[at(clampi(x, b, lx), clampi(y, b, ly), clampi(z, b, lz), nye, nze)];
}

// RTMGrid.cpp:437-635 (initBorders_RBC), in the single-thread loop order of the reference.
void borders_rbc(float *ve, int nx, int ny, int nz, int b) {
    auto V = [&](int x, int y, int z) -> float & { return ve[at(x, y, z, ny, nz)]; };
    for (int ix = b; ix < nx - b; ix++)
        for (int iy = b; iy < ny - b; iy++)
            for (int iz = 0; iz < b; iz++) {
                const int dist = b - iz;
                V(ix, iy, iz) = randlinear(V(ix, iy, b), dist, b);
                V(ix, iy, nz - 1 - iz) = randlinear(V(ix, iy, nz - b - 1), dist, b);
            }
    for (int ix = b; ix < nx - b; ix++)
        for (int iz = b; iz < nz - b; iz++)
            for (int iy = 0; iy < b; iy++) {
                V(ix, iy, iz) = randlinear(V(ix, b, iz), b - iy, b);
                V(ix, ny - b + iy, iz) = randlinear(V(ix, ny - b - 1, iz), iy, b);
            }
    for (int iy = b; iy < ny - b; iy++)
        for (int iz = b; iz < nz - b; iz++)
            for (int ix = 0; ix < b; ix++) {
                V(ix, iy, iz) = randlinear(V(b, iy, iz), b - ix, b);
                V(nx - b + ix, iy, iz) = randlinear(V(nx - b - 1, iy, iz), ix, b);
            }
    for (int ix = 0; ix < b; ix++)
        for (int iz = 0; iz < b; iz++)
            for (int iy = 0; iy < ny; iy++) {
                const int ky = iy < b ? b : (iy >= ny - b ? ny - b - 1 : iy);
                const int xs[4] = {b, nx - b - 1, b, nx - b - 1}, zs[4] = {b, b, nz - b - 1, nz - b - 1};
                const int xd[4] = {b - ix, ix, b - ix, ix}, zd[4] = {b - iz, b - iz, iz, iz};
                const int xo[4] = {ix, nx - b + ix, ix, nx - b + ix}, zo[4] = {iz, iz, nz - b + iz, nz - b + iz};
                for (int c = 0; c < 4; ++c) {
                    float v = V(xs[c], ky, zs[c]);
                    if (iy < b) v = randlinear(v, b - iy, b);
                    else if (iy >= ny - b) v = randlinear(v, iy - (ny - b), b);
                    v = randlinear(v, xd[c], b);
                    v = randlinear(v, zd[c], b);
                    V(xo[c], iy, zo[c]) = v;
                }
            }
    for (int iy = 0; iy < b; iy++)
        for (int iz = 0; iz < b; iz++)
            for (int ix = b; ix < nx - b; ix++) {
                const int ys[4] = {b, ny - b - 1, b, ny - b - 1}, zs[4] = {b, b, nz - b - 1, nz - b - 1};
                const int yd[4] = {b - iy, iy, b - iy, iy}, zd[4] = {b - iz, b - iz, iz, iz};
                const int yo[4] = {iy, ny - b + iy, iy, ny - b + iy}, zo[4] = {iz, iz, nz - b + iz, nz - b + iz};
                for (int c = 0; c < 4; ++c) {
                    float v = V(ix, ys[c], zs[c]);
                    v = randlinear(v, yd[c], b);
                    v = randlinear(v, zd[c], b);
                    V(ix, yo[c], zo[c]) = v;
                }
            }
    for (int ix = 0; ix < b; ix++)
        for (int iy = 0; iy < b; iy++)
            for (int iz = b; iz < nz - b; iz++) {
                const int xs[4] = {b, b, nx - b - 1, nx - b - 1}, ys[4] = {b, ny - b - 1, b, ny - b - 1};
                const int xd[4] = {b - ix, b - ix, ix, ix}, yd[4] = {b - iy, iy, b - iy, iy};
                const int xo[4] = {ix, ix, nx - b + ix, nx - b + ix}, yo[4] = {iy, ny - b + iy, iy, ny - b + iy};
                for (int c = 0; c < 4; ++c) {
                    float v = V(xs[c], ys[c], iz);
                    v = randlinear(v, xd[c], b);
                    v = randlinear(v, yd[c], b);
                    V(xo[c], yo[c], iz) = v;
                }
            }
}

}  // namespace

float rtmb::ricker_sample(uint32_t it, float dt, float fpeak) {
    const float t = static_cast<float>(static_cast<double>(static_cast<float>(it) * dt) - 1.0 / fpeak);
    const float x = static_cast<float>(M_PI * fpeak * t);
    const float xx = x * x;
    return static_cast<float>(static_cast<double>(std::exp(-xx)) * (1.0 - 2.0 * xx));
}

extern "C" {

int rtmb_stencil_coefs(uint32_t order, float dx, float dy, float dz, float *out) {
    if (!out || order < 2 || order > 16 || (order & 1u)) return RTMB_EINVAL;
    float c[17];
    laplacian(c, static_cast<int>(order));
    const float d[3] = {dx, dy, dz};
    for (int k = 0; k < 3; ++k) {
        const float devinv = static_cast<float>((1.0 / d[k]) * (1.0 / d[k]));
        for (uint32_t io = 0; io <= order; ++io) out[k * (order + 1) + io] = devinv * c[io];
    }
    return RTMB_OK;
}

int rtmb_taper_vector(uint32_t blen, float taper_factor, float *out) {
    if (!out && blen) return RTMB_EINVAL;
    const float dfrac = static_cast<float>(std::sqrt(std::log(taper_factor) * -1.0f) / (1. * blen));
    for (uint32_t i = 0; i < blen; ++i) {
        const float a = dfrac * static_cast<float>(i);
        out[i] = static_cast<float>(std::exp(-std::pow(static_cast<double>(a), 2.0)));
    }
    return RTMB_OK;
}

int rtmb_ricker(uint32_t nt, float dt, float fpeak, float *out) {
    if (!out && nt) return RTMB_EINVAL;
    for (uint32_t it = 0; it < nt; ++it) out[it] = rtmb::ricker_sample(it, dt, fpeak);
    return RTMB_OK;
}

int rtmb_prepare_velocity(const float *v, uint32_t nx, uint32_t ny, uint32_t nz, uint32_t blen, int32_t bc,
                          int64_t seed, float *ve) {
    if (!v || !ve || !nx || !ny || !nz) return RTMB_EINVAL;
    const int b = static_cast<int>(blen);
    const int nxe = nx + 2 * b, nye = ny + 2 * b, nze = nz + 2 * b;
    std::memset(ve, 0, sizeof(float) * static_cast<size_t>(nxe) * nye * nze);
    for (uint32_t x = 0; x < nx; ++x)
        for (uint32_t y = 0; y < ny; ++y)
            std::memcpy(ve + at(x + b, y + b, b, nye, nze), v + (static_cast<size_t>(x) * ny + y) * nz,
                        sizeof(float) * nz);
    if (bc == 0 || b == 0) return RTMB_OK;
    if (seed >= 0) srand(static_cast<unsigned>(seed));
    switch (bc) {
    case RTMB_BC_ABC: borders_abc(ve, nxe, nye, nze, b); break;
    case RTMB_BC_RBC: borders_rbc(ve, nxe, nye, nze, b); break;
    case RTMB_BC_HBC: {
        // RTMGrid.cpp:638-696: ABC, RBC, then the top planes replicated from z = blen
        borders_abc(ve, nxe, nye, nze, b);
        borders_rbc(ve, nxe, nye, nze, b);
        const int lx = nxe - 2 * b, ly = nye - 2 * b;
        for (int x = 0; x < nxe; ++x)
            for (int y = 0; y < nye; ++y)
                for (int z = 0; z < b; ++z)
                    ve[at(x, y, z, nye, nze)] = ve[at(clampi(x, b, lx), clampi(y, b, ly), b, nye, nze)];
        break;
    }
    default: return RTMB_EINVAL;
    }
    return RTMB_OK;
}

int rtmb_v2dt2_host(float *ve, size_t n, float dt) {
    if (!ve) return RTMB_EINVAL;
    const float dt2 = dt * dt;
    for (size_t i = 0; i < n; ++i) ve[i] *= ve[i];
    for (size_t i = 0; i < n; ++i) ve[i] *= dt2;
    return RTMB_OK;
}

}  // extern "C"
