/*
 * ref_shim.cpp -- TEST INFRASTRUCTURE ONLY (part of the oracle).
 *
 * A thin extern "C" shim over the reference's own CPU platform
 * (source/rtm-3d/src/platform/host/RTMCPUPlatform.cpp) and its grid / seismic
 * helpers, so that tests can run the reference operators on arbitrary arrays
 * and pin the oracle restatement (oracle/rtm_oracle.c) against them.
 *
 * This file is compiled against the reference headers and linked with the
 * reference objects by oracle/Makefile (target `ref`); the result lands in
 * oracle/_ref/librtmref.so.  Nothing in the product links it.
 *
 * Every entry point copies the caller's arrays into reference grid objects,
 * calls exactly one reference method, and copies the result back.
 */
#include <cstring>
#include <cstdlib>
#include <omp.h>
#include <RTM.hpp>

namespace {

struct Ctx {
    RTMParam param;
    RTMProcessLimits limits;
    Ctx(int nx, int ny, int nz, int blen, int order) {
        param.nx = nx; param.ny = ny; param.nz = nz; param.blen = blen;
        param.stencil_order = order;
        param.verbose = false;
        param.dx = param.dy = param.dz = 10.0f;
        param.receiver_start_x = param.receiver_start_y = param.receiver_depth_z = 0;
        param.receiver_distance_x = param.receiver_distance_y = 1;
        param.receiver_count_x = param.receiver_count_y = 1;
        std::memset(&limits, 0, sizeof(limits));
        limits.processArea.xStart = 0; limits.processArea.xEnd = nx + 2 * blen;
        limits.processArea.yStart = 0; limits.processArea.yEnd = ny + 2 * blen;
        limits.nProcesses = 1; limits.validProcessArea = true;
        limits.shadowLength = order / 2;
    }
};

template <class G>
void load(G &g, const float *src) { std::memcpy(g.data(), src, g.size() * sizeof(float)); }
template <class G>
void store(G &g, float *dst) { std::memcpy(dst, g.data(), g.size() * sizeof(float)); }

}  // namespace

extern "C" {

void ref_set_threads(int n) { omp_set_num_threads(n); }
void ref_srand(unsigned seed) { srand(seed); }

/* RTMStencil::setStencilCoefficients (RTMGrid.hpp:433-446) -> 3*(order+1) floats. */
void ref_stencil_coefs(int order, float dx, float dy, float dz, float *out) {
    RTMData_t d[3] = {dx, dy, dz};
    RTMStencil<RTMData_t, RTMDevPtr_t, RTM_NDIM_3D> st(order, d);
    for (int dim = 0; dim < 3; ++dim)
        for (int io = 0; io <= order; ++io)
            out[dim * (order + 1) + io] = st.getStencilCoef(RTMDim(dim), io);
}

/* RTMTaperFunction::inittaper (RTMSeismic.hpp:294-305). */
void ref_taper_vector(int blen, float factor, float *out) {
    RTMTaperFunction<RTMData_t, RTMDevPtr_t> t(blen, factor);
    for (int i = 0; i < blen; ++i) out[i] = t[i];
}

/* RTMSeismicSource::loadSamples / ricker (RTMSeismic.hpp:135-144, 191-198). */
void ref_ricker(int nt, float dt, float fpeak, float *out) {
    RTMSeismicSource<RTMData_t, RTMDevPtr_t> s(0, 0, 0, nt, dt, fpeak);
    for (int i = 0; i < nt; ++i) out[i] = s[i];
}

/* RTMCPUPlatform::rtmStep (RTMCPUPlatform.cpp:474-490 -> rtmStep3D :325-395).
 * nx,ny,nz are the UNPADDED model sizes; arrays are padded (nx+2b)(ny+2b)(nz+2b). */
int ref_step(int nx, int ny, int nz, int blen, int order, float dx, float dy, float dz,
             const float *P, float *PP, const float *v2dt2) {
    Ctx c(nx, ny, nz, blen, order);
    size_t nxe = nx + 2 * blen, nye = ny + 2 * blen, nze = nz + 2 * blen;
    RTMCube<RTMData_t, RTMDevPtr_t> gp(nxe, nye, nze), gpp(nxe, nye, nze);
    RTMVelocityModel<RTMData_t, RTMDevPtr_t> gv(nxe, nye, nze);
    load(gp, P); load(gpp, PP); load(gv, v2dt2);
    RTMData_t d[3] = {dx, dy, dz};
    RTMStencil<RTMData_t, RTMDevPtr_t, RTM_NDIM_3D> st(order, d);
    RTMCPUPlatform plat(c.param, c.limits);
    try {
        plat.rtmStep(&gp, &gpp, &st, gv);
    } catch (...) {
        store(gpp, PP);
        return 1;  /* "Numerical Dispersion" (NaN) exception */
    }
    store(gpp, PP);
    return 0;
}

/* RTMCPUPlatform::rtmTaperAllBorders / rtmTaperUpperBorders (:542-564 -> taper3D :710-920,
 * taperUpper3D :566-657). */
void ref_taper(int upper, int nx, int ny, int nz, int blen, float factor, float *grid) {
    Ctx c(nx, ny, nz, blen, 8);
    size_t nxe = nx + 2 * blen, nye = ny + 2 * blen, nze = nz + 2 * blen;
    RTMCube<RTMData_t, RTMDevPtr_t> g(nxe, nye, nze);
    load(g, grid);
    RTMTaperFunction<RTMData_t, RTMDevPtr_t> t(blen, factor);
    RTMCPUPlatform plat(c.param, c.limits);
    if (upper) plat.rtmTaperUpperBorders(&g, &t);
    else plat.rtmTaperAllBorders(&g, &t);
    store(g, grid);
}

/* RTMCPUPlatform::rtmApplySource (:103-113). sx,sy,sz are unpadded coordinates. */
void ref_apply_source(int nx, int ny, int nz, int blen, int sx, int sy, int sz, int nt,
                      float dt, float fpeak, int it, float *PP) {
    Ctx c(nx, ny, nz, blen, 8);
    size_t nxe = nx + 2 * blen, nye = ny + 2 * blen, nze = nz + 2 * blen;
    RTMCube<RTMData_t, RTMDevPtr_t> g(nxe, nye, nze);
    load(g, PP);
    RTMSeismicSource<RTMData_t, RTMDevPtr_t> s(sx, sy, sz, nt, dt, fpeak);
    RTMCPUPlatform plat(c.param, c.limits);
    plat.rtmApplySource(&g, &s, it);
    store(g, PP);
}

static RTMReceiverGrid<RTMData_t, RTMDevPtr_t> *make_rcv(const int *geo, int ntstep) {
    /* geo = {start_x, start_y, depth_z, dist_x, dist_y, count_x, count_y} */
    auto *r = new RTMReceiverGrid<RTMData_t, RTMDevPtr_t>(geo[5], geo[6], ntstep);
    r->setOffsetX(geo[0]); r->setOffsetY(geo[1]); r->setOffsetZ(geo[2]);
    r->setDistanceX(geo[3]); r->setDistanceY(geo[4]);
    return r;
}

/* RTMCPUPlatform::rtmSaveReceiverData (:133-151). rec is [count_x][count_y][ntstep]. */
void ref_save_receivers(int nx, int ny, int nz, int blen, const int *geo, int ntstep, int lt,
                        const float *PP, float *rec) {
    Ctx c(nx, ny, nz, blen, 8);
    size_t nxe = nx + 2 * blen, nye = ny + 2 * blen, nze = nz + 2 * blen;
    RTMCube<RTMData_t, RTMDevPtr_t> g(nxe, nye, nze);
    load(g, PP);
    auto *r = make_rcv(geo, ntstep);
    load(*r, rec);
    RTMCPUPlatform plat(c.param, c.limits);
    plat.rtmSaveReceiverData(&g, r, lt);
    store(*r, rec);
    delete r;
}

/* RTMCPUPlatform::rtmRestoreReceiverData (:114-131) -- overwrites. */
void ref_restore_receivers(int nx, int ny, int nz, int blen, const int *geo, int ntstep, int lt,
                           float *PP, const float *rec) {
    Ctx c(nx, ny, nz, blen, 8);
    size_t nxe = nx + 2 * blen, nye = ny + 2 * blen, nze = nz + 2 * blen;
    RTMCube<RTMData_t, RTMDevPtr_t> g(nxe, nye, nze);
    load(g, PP);
    auto *r = make_rcv(geo, ntstep);
    load(*r, rec);
    RTMCPUPlatform plat(c.param, c.limits);
    plat.rtmRestoreReceiverData(&g, r, lt);
    store(g, PP);
    delete r;
}

/* RTMCPUPlatform::rtmSaveUpperBorder / rtmRestoreUpperBorder (:153-189).
 * upb is [ntstep][nxe][nye][order/2]. */
void ref_upb(int rw, int nx, int ny, int nz, int blen, int order, int ntstep, int lt,
             float *P, float *upb) {
    Ctx c(nx, ny, nz, blen, order);
    size_t nxe = nx + 2 * blen, nye = ny + 2 * blen, nze = nz + 2 * blen;
    RTMCube<RTMData_t, RTMDevPtr_t> g(nxe, nye, nze);
    load(g, P);
    RTMGridCollection<RTMData_t, RTMDevPtr_t> u(ntstep, nxe, nye, order / 2);
    load(u, upb);
    RTMCPUPlatform plat(c.param, c.limits);
    if (rw) { plat.rtmSaveUpperBorder(&g, &u, lt); store(u, upb); }
    else { plat.rtmRestoreUpperBorder(&g, &u, lt); store(g, P); }
}

/* RTMCPUPlatform::rtmImageCondition (:513-540). */
void ref_image(int nx, int ny, int nz, int blen, float *img, const float *ps, const float *pr) {
    Ctx c(nx, ny, nz, blen, 8);
    size_t nxe = nx + 2 * blen, nye = ny + 2 * blen, nze = nz + 2 * blen;
    RTMCube<RTMData_t, RTMDevPtr_t> gi(nxe, nye, nze), gs(nxe, nye, nze), gr(nxe, nye, nze);
    load(gi, img); load(gs, ps); load(gr, pr);
    RTMCPUPlatform plat(c.param, c.limits);
    plat.rtmImageCondition(&gi, &gs, &gr);
    store(gi, img);
}

/* RTMCube::extendBorders (RTMGrid.cpp:47-86) followed by initBorders (:698-714).
 * bc: 1 ABC, 2 HBC, 3 RBC (RTMBoundaryCondition order, RTMGrid.hpp:27-33). */
void ref_extend_init_borders(int nx, int ny, int nz, int blen, int bc, const float *v, float *ve) {
    RTMCube<RTMData_t, RTMDevPtr_t> g(nx, ny, nz);
    load(g, v);
    g.extendBorders(blen);
    g.setBorderLength(blen);
    if (bc > 0) g.initBorders(RTMBoundaryCondition(bc));
    store(g, ve);
}

/* RTMCube::filter with the order-2 Laplacian stencil (RTMGrid.cpp:226-300;
 * RTM_LAPFILTER_ORDER, RTMBase.hpp:14) then removeBorders (:129-166). */
void ref_filter_remove(int nxe, int nye, int nze, int blen, float dx, float dy, float dz,
                       const float *img, float *out) {
    RTMCube<RTMData_t, RTMDevPtr_t> g(nxe, nye, nze);
    load(g, img);
    RTMData_t d[3] = {dx, dy, dz};
    RTMStencil<RTMData_t, RTMDevPtr_t, RTM_NDIM_3D> st(RTM_LAPFILTER_ORDER, d);
    g.filter(st);
    g.removeBorders(blen);
    store(g, out);
}

}  // extern "C"
