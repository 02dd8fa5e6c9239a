/*
 * rtm_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of the reference's time-stepping hot path (sc4ii-cimatec/rtm3d-demo,
 * source/rtm-3d, abbreviated S/ below), used by the test-suite as the parity checker and by
 * bench.py as a CPU baseline.  Nothing in the product links or calls it.
 *
 * Parity is pinned: tests/test_oracle_pin.py compares every function here against the
 * reference's own code built from its sources (oracle/_ref/librtmref.so, oracle/_ref/RTM3D.bin)
 * and against committed golden fixtures generated from it (tests/golden/).
 *
 * Layout (S/include/RTMGrid.hpp:217-221): a padded volume of (nxe, nye, nze) floats with
 * x slowest and z fastest, offset = (x*nye + y)*nze + z.  nxe = nx + 2*blen etc.
 */
#ifndef RTM_ORACLE_H
#define RTM_ORACLE_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* One shot's worth of reference parameters (the subset of S/include/RTMParam.hpp:188-249 on
 * the path).  Source and receiver coordinates are in the UNPADDED model, as in input.json. */
typedef struct orc_params {
    int nx, ny, nz, blen, order, nt, ntstep;
    float dx, dy, dz, dt, fpeak, taper_factor;
    int sx, sy, sz;
    int rsx, rsy, rdz, rdx, rdy, rcx, rcy;
} orc_params;

/* host-side math */
void orc_laplacian_coefs(int order, float *c);
void orc_stencil_coefs(int order, float dx, float dy, float dz, float *out);
void orc_taper_vector(int blen, float factor, float *out);
void orc_ricker(int nt, float dt, float fpeak, float *out);

/* velocity preparation */
void orc_extend_borders(const float *v, int nx, int ny, int nz, int blen, float *ve);
void orc_init_borders_abc(float *ve, int nxe, int nye, int nze, int blen);
void orc_init_borders_rbc(float *ve, int nxe, int nye, int nze, int blen);
void orc_init_borders_hbc(float *ve, int nxe, int nye, int nze, int blen);
void orc_v2dt2(float *v, size_t n, float dt);

/* per-step operators */
int orc_step(int nxe, int nye, int nze, int order, const float *coefs,
             const float *P, float *PP, const float *v2dt2);
/* the 2D step (nx == 1): plane x = blen only, no x term */
int orc_step2d(int nxe, int nye, int nze, int blen, int order, const float *coefs,
               const float *P, float *PP, const float *v2dt2);
void orc_taper_all(int nxe, int nye, int nze, int blen, const float *taper, float *g);
void orc_taper_upper(int nxe, int nye, int nze, int blen, const float *taper, float *g);
void orc_apply_source(int nxe, int nye, int nze, int x, int y, int z, float val, float *PP);
void orc_save_receivers(const orc_params *p, int lt, const float *PP, float *rec);
void orc_restore_receivers(const orc_params *p, int lt, float *PP, const float *rec);
void orc_save_upb(int nxe, int nye, int nze, int blen, int h, int lt, const float *P, float *upb);
void orc_restore_upb(int nxe, int nye, int nze, int blen, int h, int lt, float *P, const float *upb);
void orc_image(int nxe, int nye, int nze, int blen, float *img, const float *ps, const float *pr);

/* image finalisation */
void orc_filter_remove(int nxe, int nye, int nze, int blen, float dx, float dy, float dz,
                       const float *img, float *out);

/* time loops.  rec is the shot record in the reference's file layout: nt/ntstep chunks, each
 * [rcx][rcy][ntstep] with time fastest (what the .seism files hold, concatenated).
 * Return 0, or 1 when the step met a NaN (the reference throws "Numerical Dispersion"). */
int orc_model_shot(const orc_params *p, const float *v2dt2, float *rec);
int orc_migrate_hbc(const orc_params *p, const float *v2dt2, const float *rec, float *img);
int orc_migrate_rbc(const orc_params *p, const float *v2dt2, const float *rec, float *img);

/* frequency-domain RTM (S/src/kernel/RTMFiniteDifferencesKernel_FreqDomain.cpp).  nw: number of
 * frequencies; tables: w2[nw], kre/kim[nw][nt].  orc_migrate_fmig: one shot, img padded (zeroed
 * here); nwstep frequencies per pass over time (0: all). */
int orc_fmig_nw(int nt, float dt, float fmin, float fmax);
void orc_fmig_tables(int nt, float dt, float fmin, float fmax, int nw, float *w2, float *kre, float *kim);
int orc_migrate_fmig(const orc_params *p, const float *v2dt2, const float *rec, float fmin, float fmax, int nwstep,
                     float *img);

#ifdef __cplusplus
}
#endif
#endif
