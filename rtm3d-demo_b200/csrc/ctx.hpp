// ctx.hpp -- the library's context object and the driver helpers shared by api.cu and noalloc.cu.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "rtm3d_b200.h"
#include "stencil.cuh"

struct rtmb_ctx {
    rtmb_params p{};
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t own_stream = nullptr;
    int nxe = 0, nye = 0, nze = 0, h = 0;
    size_t n = 0;
    float coefs[3 * (rtmb::kMaxOrder + 1)] = {};
    float *d_taper = nullptr, *d_wavelet = nullptr;
    unsigned *d_err = nullptr;
    // driver state
    float *d_v2dt2 = nullptr;
    float *d_w[4] = {};          // source pair, receiver pair
    float *d_quirk[3] = {};      // front-right taper side buffers (modeling)
    float *d_upb = nullptr;      // [nt][nxe][nye][h] (HBC)
    float *d_rec = nullptr, *d_img = nullptr;  // staging for the host-buffer forms
    int chunk = 0;
    int dual_chunk = 0;  // x planes per CTA of the dual-wavefield backward step
    int variant = 0;     // launch variant of the TMA step kernel (rtmb_autotune_full)
    int use_dual = -1;   // -1: the default rule; 0 / 1: the autotuner's choice
    int dual_variant = 5;  // launch variant of the dual backward step (5: merged form, 32 x 16 tiles)
    int batch_group = 12;  // shots per launch of rtmb_migrate_batch (rtmb_autotune_batch)
    uint64_t launches = 0;
    // storage forms (RTMB_FLAG_STORE_*): element type of d_w, one scale record per stored level
    int store = rtmb::kStoreF32;
    bool img64 = false;              // RTMB_FLAG_IMG_F64
    bool diff = false;               // RTMB_FLAG_STORE_DIFF: d_w[0..1] / [2..3] hold p levels, d_inc the increments
    void *d_inc[2] = {};             // increment of the source and of the receiver wavefield
    float wmax = 0.f;                // max |Ricker sample|
    rtmb::ScaleRec *d_scale = nullptr;
    int sc_cap = 0, sc_next = 0;
    float *d_inj = nullptr;          // device scalars: [0] max |record|, [1] max forward level
    double *d_img64 = nullptr;       // FP64 image of the FP32-output migration with RTMB_FLAG_IMG_F64
    // RTMB_FLAG_USE_GRAPH: executable graph per driver kind (0 modeling, 1 migration)
    cudaGraphExec_t gexec[4] = {};  // modeling, migration, batched migration, frequency-domain migration
    // frequency-domain migration: the four frequency grids of a group, and their capacity in floats
    float *d_fq = nullptr;
    size_t fq_cap = 0;
    float *d_fquirk[6] = {};  // taper side buffers of its two wavefields (stored-taper steps)
    bool capturing = false;
    // learned boundary closure (closure.cu): strip cells of the padded grid, parameters, and the
    // strip values of the next level computed before each step
    uint32_t *d_cells = nullptr;
    uint8_t *d_faces = nullptr;
    long long ncells = 0;
    float *d_side = nullptr;
    float *d_cparams = nullptr;
    float closure_min_scale = 0.f, closure_damp = 0.f;
    int closure_verdict = 0;  // rtmb_closure_judge: 0 not judged, 1 passed, 2 fell back to the taper border
    // FP64 GPU oracle (f64.cu)
    double *d_f64[4] = {};
    double *d_upb64 = nullptr;
    std::string err;
    // optional per-kernel timing of the drivers (rtmb_profile): an event pair around each launch
    bool prof = false;
    std::vector<cudaEvent_t> ev;        // pool, two per recorded launch
    std::vector<int> ev_cat;            // category of each recorded launch
    size_t ev_used = 0;
    double prof_ms[RTMB_PROF_CATEGORIES] = {};
    uint64_t prof_n[RTMB_PROF_CATEGORIES] = {};
};

namespace rtmb {
namespace driver {

// Forward time loop shared by modeling and the migration forward pass (see api.cu).
// Work a driver adds around each step of the forward loop: before(it) runs with P = u(it) and
// PP = u(it-1), after(it) with PP = u(it+1).  Non-zero return values end the loop.
struct StepHook {
    virtual int before(int it, const float *P, float *PP) { return 0; }
    virtual int after(int it, const float *P, float *PP) { return 0; }
    virtual ~StepHook() {}
};
// With a storage form, sc_out (if not null) receives the scale records of *P_out and *PP_out.
int run_forward(rtmb_ctx *ctx, uint32_t sx, uint32_t sy, uint32_t sz, int taper_mode, float *rec,
                float *upb, float **P_out, float **PP_out, int cat, rtmb::ScaleRec **sc_out = nullptr,
                StepHook *hook = nullptr);
// The learned closure around one modeling step (closure.cu): the strip's next level from
// (P, PP) before the step, scattered into PP after it.
int closure_hook_before(rtmb_ctx *ctx, const float *P, float *PP);
int closure_hook_after(rtmb_ctx *ctx, float *PP);
// Reads and clears the device error flag after synchronising the context's stream.
int check_err_flag(rtmb_ctx *ctx);
// Fills the derived sizes and the host copy of the stencil coefficients of a context.
void init_geometry(rtmb_ctx *ctx);
// Argument checks of a modeling shot (source inside the model, receivers inside the computed region).
int check_model_shot(rtmb_ctx *ctx, uint32_t sx, uint32_t sy, uint32_t sz);
// Records a message for a call that has no context (rtmb_last_error(NULL) returns it).
int fail_noctx(int code, const char *msg);

}  // namespace driver
}  // namespace rtmb
