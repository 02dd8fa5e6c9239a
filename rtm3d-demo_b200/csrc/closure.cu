// closure.cu -- kernels and entry points of the learned absorbing-boundary closure (closure.cuh):
// strip-cell lists, feature gathering, the tcgen05 MLP forward (training and inference), the
// backward pass, Adam, training-pair collection on a wide domain, and the per-step inference that
// the modeling driver runs for boundary RTMB_BC_LEARNED.  No reference counterpart: the reference's
// absorbing layers are the taper of taper3D / taperUpper3D (RTMCPUPlatform.cpp:566-920).
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <vector>

#include <cuda_bf16.h>

#include "closure.cuh"
#include "ctx.hpp"
#include "ops.cuh"
#include "umma.cuh"

namespace rtmb {
namespace closure {
namespace {

// ------------------------------------------------------------------ geometry and features

// Face code (axis * 2 + side) of the box face nearest to box cell (cx, cy, cz) (box-relative), or
// -1 if the cell is kNet or more cells from every face.  Ties go to the first face in x-low,
// x-high, y-low, ...
__host__ __device__ inline int face_of(int cx, int cy, int cz, int nx, int ny, int nz) {
    const int d[6] = {cx, nx - 1 - cx, cy, ny - 1 - cy, cz, nz - 1 - cz};
    int best = 0;
    for (int f = 1; f < 6; ++f)
        if (d[f] < d[best]) best = f;
    return d[best] < kNet ? best : -1;
}

// The 55 features of the cell at array offset off (box-relative coordinates c[3], face f), in
// FP32, normalised by s (returned; 0 when the neighbourhood is all zero).  base: the first-order
// one-way (upwind) update of an outgoing wave, p + C (p_in - p) with p_in the inward neighbour at
// t and C the Courant number; the network predicts the correction to it.
__device__ inline float gather(const float *__restrict__ P, const float *__restrict__ PP,
                               const float *__restrict__ V, const Box &b, int cx, int cy, int cz, int f,
                               float inv_dx, float (&feat)[kUsed], float *base) {
    const int axis = f >> 1, side = f & 1;
    const int t1 = axis == 0 ? 1 : 0, t2 = axis == 2 ? 1 : 2;
    const int c[3] = {cx, cy, cz};
    const int n[3] = {b.nx, b.ny, b.nz};
    const size_t plane = (size_t)b.ay * b.az;
    float s = 0.f;
#pragma unroll
    for (int u = -1; u <= 1; ++u)
#pragma unroll
        for (int v = -1; v <= 1; ++v)
#pragma unroll
            for (int w = -1; w <= 1; ++w) {
                int q[3] = {c[0], c[1], c[2]};
                q[axis] += side ? -u : u;
                q[t1] += v;
                q[t2] += w;
                float a = 0.f, bb = 0.f;
                if (q[0] >= 0 && q[0] < n[0] && q[1] >= 0 && q[1] < n[1] && q[2] >= 0 && q[2] < n[2]) {
                    const size_t o = (size_t)(q[0] + b.ox) * plane + (size_t)(q[1] + b.oy) * b.az + (q[2] + b.oz);
                    a = __ldg(P + o);
                    bb = __ldg(PP + o);
                }
                const int j = (u + 1) * 9 + (v + 1) * 3 + (w + 1);
                feat[j] = a;
                feat[27 + j] = bb;
                s = fmaxf(s, fmaxf(fabsf(a), fabsf(bb)));
            }
    const size_t o = (size_t)(cx + b.ox) * plane + (size_t)(cy + b.oy) * b.az + (cz + b.oz);
    const float courant = sqrtf(__ldg(V + o)) * inv_dx;
    *base = fmaf(courant, feat[22] - feat[13], feat[13]);  // feat[22]: (u, v, w) = (+1, 0, 0)
    const float inv = s > 0.f ? 1.f / s : 0.f;
#pragma unroll
    for (int j = 0; j < 54; ++j) feat[j] *= inv;
    feat[54] = courant;
    return s;
}

// ------------------------------------------------------------------ tcgen05 MLP tile

constexpr int kTile = 128;  // cells per tile = MMA M
constexpr int kLboA = (kTile / 8) * 128;      // A tiles: 16 row groups of 128 bytes per K chunk
constexpr int kLboB = (kHid / 8) * 128;       // B tiles: 4 row groups per K chunk
constexpr uint32_t kIdesc = umma::idesc_bf16_f32(kTile, kHid);
constexpr uint32_t kTmemCols = 64;            // [0, 32): layer 1, [32, 64): layer 2
constexpr float kMaxCorr = 0.5f;              // bound on the network's correction, in units of s

struct __align__(128) MlpSmem {
    unsigned char a1[kTile * kIn * 2];   // features, BF16, K-major
    unsigned char a2[kTile * kHid * 2];  // hidden layer 1, BF16, K-major
    unsigned char w1[kHid * kIn * 2];    // W1 (N = 32 rows, K = 64)
    unsigned char w2[kHid * kHid * 2];   // W2
    float b1[kHid], b2[kHid], w3[kHid], b3;
    uint64_t bar;
    uint32_t tmem;
    // keeps every descriptor-addressed read of the MMAs inside this CTA's shared memory even if
    // the operand strides were read the other way round (A would then span 44 KB from a1)
    unsigned char pad[16384];
};

__device__ __forceinline__ bool bar_wait(uint64_t *bar, uint32_t parity) {
    auto try_wait = [&]() {
        uint32_t ok;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(ok)
            : "r"(umma::smem_addr(bar)), "r"(parity)
            : "memory");
        return ok != 0;
    };
    if (try_wait()) return true;
    const long long t0 = clock64();
    while (!try_wait())
        if (clock64() - t0 > (1ll << 32)) return false;
    return true;
}

// Weights into shared memory (BF16, canonical K-major), biases and w3 in FP32; TMEM allocation and
// the MMA barrier.  Every thread of the 128-thread CTA calls it.
template <class SM, uint32_t NCOLS = kTmemCols>
__device__ void mlp_setup(SM &sm, const float *__restrict__ prm) {
    const int tid = threadIdx.x;
    if (tid < 32) umma::tmem_alloc(&sm.tmem, NCOLS);
    for (int i = tid; i < kHid * kIn; i += kTile) {
        const int r = i / kIn, k = i % kIn;
        *reinterpret_cast<__nv_bfloat16 *>(sm.w1 + umma::kmajor_offset(r, k, kLboB)) =
            __float2bfloat16_rn(prm[kOffW1 + i]);
    }
    for (int i = tid; i < kHid * kHid; i += kTile) {
        const int r = i / kHid, k = i % kHid;
        *reinterpret_cast<__nv_bfloat16 *>(sm.w2 + umma::kmajor_offset(r, k, kLboB)) =
            __float2bfloat16_rn(prm[kOffW2 + i]);
    }
    if (tid < kHid) {
        sm.b1[tid] = prm[kOffB1 + tid];
        sm.b2[tid] = prm[kOffB2 + tid];
        sm.w3[tid] = prm[kOffW3 + tid];
    }
    if (tid == 0) {
        sm.b3 = prm[kOffB3];
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(umma::smem_addr(&sm.bar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
}

// Writes row m of the feature tile from 64 FP32 values (BF16-rounded), 16 bytes at a time.
__device__ __forceinline__ void put_row(unsigned char *tile, int m, const float *f, int nk, int lbo) {
    for (int c = 0; c < nk / 8; ++c) {
        __nv_bfloat162 h[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) h[j] = __floats2bfloat162_rn(f[8 * c + 2 * j], f[8 * c + 2 * j + 1]);
        *reinterpret_cast<uint4 *>(tile + umma::kmajor_offset(m, 8 * c, lbo)) = *reinterpret_cast<uint4 *>(h);
    }
}

// One tile: the caller has written every row of a1.  Returns, for this thread's row, y (the network
// output) and optionally the hidden activations (h1 rounded to BF16, as layer 2 sees it; h2 FP32).
// phase: the MMA barrier's next parity, advanced by two.  false: a wait ran out (uniform).
template <class SM>
__device__ bool mlp_tile(SM &sm, uint32_t &phase, float *y, float *h1_out, float *h2_out) {
    const int tid = threadIdx.x, warp = tid >> 5;
    const uint32_t lane_base = sm.tmem + ((uint32_t)(warp * 32) << 16);
    umma::fence_smem_to_async();
    umma::fence_before_sync();
    __syncthreads();
    if (tid == 0) {
        umma::fence_after_sync();
#pragma unroll
        for (int s = 0; s < kIn / 16; ++s)
            umma::mma_bf16(sm.tmem, umma::smem_desc(sm.a1 + s * 2 * kLboA, kLboA, 128),
                           umma::smem_desc(sm.w1 + s * 2 * kLboB, kLboB, 128), kIdesc, s > 0);
        umma::commit(&sm.bar);
    }
    bool ok = __syncthreads_and(bar_wait(&sm.bar, phase & 1));
    phase ^= 1;
    if (!ok) return false;
    umma::fence_after_sync();
    float h[32];
    umma::tmem_ld32(lane_base, h);
    float hb[32];
#pragma unroll
    for (int j = 0; j < kHid; ++j) {
        const float t = tanhf(h[j] + sm.b1[j]);
        hb[j] = __bfloat162float(__float2bfloat16_rn(t));
        if (h1_out) h1_out[j] = hb[j];
    }
    put_row(sm.a2, tid, hb, kHid, kLboA);
    umma::fence_smem_to_async();
    umma::fence_before_sync();
    __syncthreads();
    if (tid == 0) {
        umma::fence_after_sync();
#pragma unroll
        for (int s = 0; s < kHid / 16; ++s)
            umma::mma_bf16(sm.tmem + kHid, umma::smem_desc(sm.a2 + s * 2 * kLboA, kLboA, 128),
                           umma::smem_desc(sm.w2 + s * 2 * kLboB, kLboB, 128), kIdesc, s > 0);
        umma::commit(&sm.bar);
    }
    ok = __syncthreads_and(bar_wait(&sm.bar, phase & 1));
    phase ^= 1;
    if (!ok) return false;
    umma::fence_after_sync();
    umma::tmem_ld32(lane_base + kHid, h);
    float acc = sm.b3;
#pragma unroll
    for (int j = 0; j < kHid; ++j) {
        const float t = tanhf(h[j] + sm.b2[j]);
        if (h2_out) h2_out[j] = t;
        acc = fmaf(sm.w3[j], t, acc);
    }
    *y = acc;
    umma::fence_before_sync();  // the next tile's MMAs overwrite TMEM after the next barrier
    return true;
}

template <class SM, uint32_t NCOLS = kTmemCols>
__device__ void mlp_teardown(SM &sm) {
    umma::fence_before_sync();
    __syncthreads();
    if (threadIdx.x < 32) {
        umma::fence_after_sync();
        umma::tmem_dealloc(sm.tmem, NCOLS);
    }
}

// ------------------------------------------------------------------ kernels

// y[i] = MLP(X[i]) for n rows of BF16 features; optionally the hidden activations (training).
__global__ void __launch_bounds__(kTile) mlp_forward_kernel(const float *__restrict__ prm,
                                                            const __nv_bfloat16 *__restrict__ X, long long n,
                                                            float *y, float *H1, float *H2, unsigned *err) {
    __shared__ MlpSmem sm;
    mlp_setup(sm, prm);
    uint32_t phase = 0;
    const long long ntiles = (n + kTile - 1) / kTile;
    for (long long t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const long long row = t * kTile + threadIdx.x;
        float f[kIn];
        if (row < n) {
            const uint4 *src = reinterpret_cast<const uint4 *>(X + row * kIn);
#pragma unroll
            for (int c = 0; c < kIn / 8; ++c) {
                const uint4 u = __ldg(src + c);
                const __nv_bfloat162 *h = reinterpret_cast<const __nv_bfloat162 *>(&u);
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const float2 v = __bfloat1622float2(h[j]);
                    f[8 * c + 2 * j] = v.x;
                    f[8 * c + 2 * j + 1] = v.y;
                }
            }
        } else {
#pragma unroll
            for (int k = 0; k < kIn; ++k) f[k] = 0.f;
        }
        put_row(sm.a1, threadIdx.x, f, kIn, kLboA);
        float out, h1[kHid], h2[kHid];
        const bool train = H1 != nullptr;
        if (!mlp_tile(sm, phase, &out, train ? h1 : nullptr, train ? h2 : nullptr)) {
            if (threadIdx.x == 0 && err) atomicOr(err, 2u);
            break;
        }
        if (row < n) {
            y[row] = out;
            if (train) {
#pragma unroll
                for (int j = 0; j < kHid; ++j) {
                    H1[row * kHid + j] = h1[j];
                    H2[row * kHid + j] = h2[j];
                }
            }
        }
    }
    mlp_teardown(sm);
}

// Per-step inference on the strip: side[i] = p(t+1) of strip cell i.
__global__ void __launch_bounds__(kTile) strip_step_kernel(const float *__restrict__ prm,
                                                           const float *__restrict__ P,
                                                           const float *__restrict__ PP,
                                                           const float *__restrict__ V, Box b,
                                                           const uint32_t *__restrict__ cells,
                                                           const uint8_t *__restrict__ faces, long long ncells,
                                                           float inv_dx, float min_scale, float damp, float *side,
                                                           unsigned *err) {
    __shared__ MlpSmem sm;
    mlp_setup(sm, prm);
    uint32_t phase = 0;
    const long long ntiles = (ncells + kTile - 1) / kTile;
    const size_t plane = (size_t)b.ay * b.az;
    for (long long t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const long long i = t * kTile + threadIdx.x;
        float f[kIn];
        float s = 0.f, base = 0.f, keep = 1.f;
        if (i < ncells) {
            const uint32_t off = cells[i];
            const int cx = (int)(off / plane) - b.ox, cy = (int)((off % plane) / b.az) - b.oy,
                      cz = (int)(off % b.az) - b.oz;
            const int fc = faces[i], ax = fc >> 1;
            const int c[3] = {cx, cy, cz}, n[3] = {b.nx, b.ny, b.nz};
            const int depth = (fc & 1) ? n[ax] - 1 - c[ax] : c[ax];  // 0 at the outer face
            const float u = (float)(kNet - depth) / kNet;
            keep = 1.f - damp * u * u;
            float feat[kUsed];
            s = gather(P, PP, V, b, cx, cy, cz, fc, inv_dx, feat, &base);
#pragma unroll
            for (int k = 0; k < kUsed; ++k) f[k] = feat[k];
        } else {
#pragma unroll
            for (int k = 0; k < kUsed; ++k) f[k] = 0.f;
        }
#pragma unroll
        for (int k = kUsed; k < kIn; ++k) f[k] = 0.f;
        put_row(sm.a1, threadIdx.x, f, kIn, kLboA);
        float r;
        if (!mlp_tile(sm, phase, &r, nullptr, nullptr)) {
            if (threadIdx.x == 0 && err) atomicOr(err, 2u);
            break;
        }
        if (i < ncells) {
            // below min_scale the neighbourhood holds only the stencil's numerical tail ahead of
            // the wavefront (the network was not trained there): the strip cell stays at zero.
            // The new value is kept within the neighbourhood's range [-s, s], so the network can
            // never amplify what reaches the strip from one step to the next.
            const float rc = fminf(kMaxCorr, fmaxf(-kMaxCorr, r));
            const float o = s < min_scale ? 0.f : fminf(s, fmaxf(-s, keep * fmaf(s, rc, base)));
            side[i] = o;
            if (o != o && err) atomicOr(err, 1u);
        }
    }
    mlp_teardown(sm);
}

__global__ void strip_scatter_kernel(float *PP, const uint32_t *__restrict__ cells, const float *__restrict__ side,
                                     long long ncells) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < ncells; i += (long long)gridDim.x * blockDim.x)
        PP[cells[i]] = side[i];
}

__host__ __device__ inline uint64_t mix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

// Training-pair collection, before the step: features of cells_per_step strip cells drawn at
// random (seeded) from p(t) = P and p(t-1) = PP, into staging row j.  Cells whose neighbourhood max
// |p| is below min_scale are marked invalid: far ahead of the wavefront the stencil's numerical tail
// is orders of magnitude below the waves the closure must absorb.
__global__ void sample_features_kernel(const float *__restrict__ P, const float *__restrict__ PP,
                                       const float *__restrict__ V, Box b, const uint32_t *__restrict__ cells,
                                       const uint8_t *__restrict__ faces, long long ncells, int per_step,
                                       uint64_t key, float inv_dx, float min_scale, __nv_bfloat16 *Xs,
                                       long long *slot_of, float *stash) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= per_step) return;
    const long long i = (long long)(mix64(key + (uint64_t)j) % (uint64_t)ncells);
    const uint32_t off = cells[i];
    const size_t plane = (size_t)b.ay * b.az;
    const int cx = (int)(off / plane) - b.ox, cy = (int)((off % plane) / b.az) - b.oy, cz = (int)(off % b.az) - b.oz;
    float feat[kUsed], base;
    const float s = gather(P, PP, V, b, cx, cy, cz, faces[i], inv_dx, feat, &base);
    const bool valid = s > 0.f && s >= min_scale;
    slot_of[j] = valid ? 1 : 0;
    stash[3 * j] = __uint_as_float(off);
    stash[3 * j + 1] = base;
    stash[3 * j + 2] = s;
    __nv_bfloat16 *row = Xs + (long long)j * kIn;
    for (int k = 0; k < kIn; ++k) row[k] = __float2bfloat16_rn(valid && k < kUsed ? feat[k] : 0.f);
}

// The valid staging rows of this step appended to (X, count) in staging order, so that the data
// set (and the training that draws from it) does not depend on thread timing: one block scans the
// valid flags; slot_of[j] becomes the row's slot, or -1.
__global__ void __launch_bounds__(1024) compact_rows_kernel(const __nv_bfloat16 *__restrict__ Xs, int per_step,
                                                             __nv_bfloat16 *X, unsigned long long cap,
                                                             unsigned long long *count, long long *slot_of) {
    __shared__ int warp_sums[32];
    __shared__ unsigned long long base_s;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) base_s = *count;
    __syncthreads();
    for (int j0 = 0; j0 < per_step; j0 += 1024) {
        const int j = j0 + tid;
        const int v = j < per_step ? (int)slot_of[j] : 0;
        const unsigned ballot = __ballot_sync(0xffffffffu, v);
        const int in_warp = __popc(ballot & ((1u << lane) - 1u));
        if (lane == 31) warp_sums[warp] = in_warp + v;
        __syncthreads();
        if (warp == 0) {
            int w = warp_sums[lane];
            for (int o = 1; o < 32; o <<= 1) {
                const int t = __shfl_up_sync(0xffffffffu, w, o);
                if (lane >= o) w += t;
            }
            warp_sums[lane] = w;  // inclusive prefix over warps
        }
        __syncthreads();
        const int before = (warp > 0 ? warp_sums[warp - 1] : 0) + in_warp;
        const unsigned long long slot = base_s + (unsigned long long)before;
        if (j < per_step) {
            if (v && slot < cap) {
                slot_of[j] = (long long)slot;
                const uint4 *src = reinterpret_cast<const uint4 *>(Xs + (long long)j * kIn);
                uint4 *dst = reinterpret_cast<uint4 *>(X + slot * kIn);
                for (int c = 0; c < kIn / 8; ++c) dst[c] = src[c];
            } else {
                slot_of[j] = -1;
            }
        }
        __syncthreads();
        if (tid == 0) base_s += (unsigned long long)warp_sums[31];
        __syncthreads();
    }
    if (tid == 0) *count = base_s;
}

// ... after the step: the target r = (p(t+1) - base) / s.
__global__ void sample_target_kernel(const float *__restrict__ PPnew, int per_step, const long long *slot_of,
                                     const float *stash, float *R) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= per_step || slot_of[j] < 0) return;
    const uint32_t off = __float_as_uint(stash[3 * j]);
    R[slot_of[j]] = (PPnew[off] - stash[3 * j + 1]) / stash[3 * j + 2];
}

// Random mini-batch (with replacement, seeded): rows of (X, R) into (Xb, Rb).
// With noise > 0 the 54 wavefield features get Gaussian noise of that standard deviation (the
// features are normalised to max 1), so that the network is trained on inputs a little off the
// data, as it meets them when its own outputs feed back step after step.
__global__ void gather_batch_kernel(const __nv_bfloat16 *__restrict__ X, const float *__restrict__ R, long long n,
                                    int B, uint64_t key, float noise, __nv_bfloat16 *Xb, float *Rb) {
    const int i = blockIdx.x;
    const long long src = (long long)(mix64(key + (uint64_t)i) % (uint64_t)n);
    const int k0 = 2 * threadIdx.x;  // 32 threads x 2 features
    __nv_bfloat162 v = reinterpret_cast<const __nv_bfloat162 *>(X + src * kIn)[threadIdx.x];
    if (noise > 0.f && k0 < 54) {
        const uint64_t h = mix64(key ^ (0xD1B54A32D192ED03ull * (uint64_t)(i * 32 + threadIdx.x + 1)));
        const float u1 = ((h >> 40) + 1) * (1.0f / 16777217.0f), u2 = ((h >> 16) & 0xFFFFFF) * (1.0f / 16777216.0f);
        const float r = sqrtf(-2.f * logf(u1));
        float2 f = __bfloat1622float2(v);
        f.x += noise * r * cosf(6.2831853f * u2);
        f.y += noise * r * sinf(6.2831853f * u2);
        v = __floats2bfloat162_rn(f.x, f.y);
    }
    reinterpret_cast<__nv_bfloat162 *>(Xb + (long long)i * kIn)[threadIdx.x] = v;
    if (threadIdx.x == 0) Rb[i] = R[src];
}

// ------------------------------------------------------------------ tensor-core training step

// The gradient of one batch on the tensor cores.  Per tile of 128 rows (one row per thread): the
// forward pass (mlp_tile), then dz2 = dy w3 (1 - h2^2) and the MMA dh1 = dz2 W2 (M 128, N 32,
// K 32: A = dz2 in BF16, B = W2^T) with dz1 = dh1 (1 - h1^2), then ONE MMA for every weight and
// bias gradient of the two hidden layers over the tile's rows (M 128, N 64, K 128):
//     A = [X^T; H1^T; ones; 0]  (rows: 64 features, 32 hidden units, one row of ones, padding)
//     B = [dZ1^T; dZ2^T]        (rows: 32 + 32 pre-activation gradients)
// so D[0:64, 0:32] = X^T dZ1 = dW1^T, D[64:96, 32:64] = H1^T dZ2 = dW2^T and the ones row gives
// db1, db2 (D[96, 0:64]); the other blocks of D are not read.  D accumulates in TMEM over the CTA's
// tiles.  dw3, db3 and the loss are sums over rows of scalars, reduced per CTA.  Each CTA writes its
// partial gradient (and loss) to part[blockIdx.x]; grad_sum_kernel adds the CTAs in order, so a
// gradient is reproducible for a given batch size.  dz1 and dz2 enter the MMAs rounded to BF16
// (the operand type), the bias gradients included; everything accumulates in FP32.
constexpr int kGradN = 2 * kHid;                    // B rows of the weight-gradient MMA
constexpr int kLboGA = (kTile / 8) * 128;           // A: 16 row groups per K chunk
constexpr int kLboGB = (kGradN / 8) * 128;          // B: 8 row groups per K chunk
constexpr uint32_t kIdescG = umma::idesc_bf16_f32(kTile, kGradN);
constexpr uint32_t kTmemColsG = 256;                // [0, 64): forward, [64, 96): dh1, [128, 192): D
constexpr uint32_t kColDh1 = 64, kColG = 128;
constexpr int kRowOnes = kIn + kHid;                // the ones row of A (96)
constexpr int kPartStride = kNParam + 1;            // a CTA's partial gradient and loss

struct __align__(128) GradSmem {
    unsigned char a1[kTile * kIn * 2];     // features, BF16, K-major
    unsigned char a2[kTile * kHid * 2];    // hidden layer 1, then dz2 (BF16, K-major)
    unsigned char w1[kHid * kIn * 2];      // W1 (N = 32 rows, K = 64)
    unsigned char w2[kHid * kHid * 2];     // W2
    unsigned char w2t[kHid * kHid * 2];    // W2^T, the backward B operand
    unsigned char ga[kTile * kTile * 2];   // A of the weight-gradient MMA (M 128, K 128)
    unsigned char gb[kGradN * kTile * 2];  // B of the weight-gradient MMA (N 64, K 128)
    float b1[kHid], b2[kHid], w3[kHid], b3;
    float red[kTile / 32][kHid + 2];       // per-warp sums of dw3, db3 and the loss
    uint64_t bar;
    uint32_t tmem;
    unsigned char pad[16384];              // as in MlpSmem
};

__device__ __forceinline__ void put_bf16(unsigned char *tile, int r, int m, int lbo, float v) {
    *reinterpret_cast<__nv_bfloat16 *>(tile + umma::kmajor_offset(r, m, lbo)) = __float2bfloat16_rn(v);
}

// One K-major MMA chain D (+)= A B^T of nk16 K steps, issued by thread 0, completion awaited by all.
__device__ __forceinline__ bool mma_chain(uint64_t *bar, uint32_t &phase, uint32_t tmem_d, const unsigned char *A,
                                          int lbo_a, const unsigned char *B, int lbo_b, uint32_t idesc, int nk16,
                                          bool accumulate) {
    umma::fence_smem_to_async();
    umma::fence_before_sync();
    __syncthreads();
    if (threadIdx.x == 0) {
        umma::fence_after_sync();
        for (int s = 0; s < nk16; ++s)
            umma::mma_bf16(tmem_d, umma::smem_desc(A + s * 2 * lbo_a, lbo_a, 128),
                           umma::smem_desc(B + s * 2 * lbo_b, lbo_b, 128), idesc, accumulate || s > 0);
        umma::commit(bar);
    }
    const bool ok = __syncthreads_and(bar_wait(bar, phase & 1));
    phase ^= 1;
    umma::fence_after_sync();
    return ok;
}

__global__ void __launch_bounds__(kTile) mlp_grad_kernel(const float *__restrict__ prm,
                                                         const __nv_bfloat16 *__restrict__ X,
                                                         const float *__restrict__ R, long long n, float *part,
                                                         unsigned *err) {
    extern __shared__ __align__(128) unsigned char gsm_raw[];
    GradSmem &sm = *reinterpret_cast<GradSmem *>(gsm_raw);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    // W2^T, and the rows of A the tiles never write: the ones row and the padding
    for (int i = tid; i < kHid * kHid; i += kTile) {
        const int r = i / kHid, k = i % kHid;  // W2^T[r][k] = W2[k][r]
        put_bf16(sm.w2t, r, k, (kHid / 8) * 128, prm[kOffW2 + k * kHid + r]);
    }
    for (int i = tid; i < (kTile - kRowOnes) * kTile; i += kTile) {
        const int r = kRowOnes + i / kTile, m = i % kTile;
        put_bf16(sm.ga, r, m, kLboGA, r == kRowOnes ? 1.f : 0.f);
    }
    mlp_setup<GradSmem, kTmemColsG>(sm, prm);
    const uint32_t lane_base = sm.tmem + ((uint32_t)(warp * 32) << 16);
    const float inv_n = 1.f / (float)n;
    float dw3[kHid], db3 = 0.f, lsum = 0.f;
#pragma unroll
    for (int j = 0; j < kHid; ++j) dw3[j] = 0.f;
    uint32_t phase = 0;
    int done = 0;
    bool ok = true;
    const long long ntiles = (n + kTile - 1) / kTile;
    for (long long t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
        const long long row = t * kTile + tid;
        const bool valid = row < n;
        {
            float f[kIn];
            if (valid) {
                const uint4 *src = reinterpret_cast<const uint4 *>(X + row * kIn);
#pragma unroll
                for (int c = 0; c < kIn / 8; ++c) {
                    const uint4 u = __ldg(src + c);
                    const __nv_bfloat162 *h = reinterpret_cast<const __nv_bfloat162 *>(&u);
#pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        const float2 v = __bfloat1622float2(h[j]);
                        f[8 * c + 2 * j] = v.x;
                        f[8 * c + 2 * j + 1] = v.y;
                    }
                }
            } else {
#pragma unroll
                for (int k = 0; k < kIn; ++k) f[k] = 0.f;
            }
            put_row(sm.a1, tid, f, kIn, kLboA);
#pragma unroll
            for (int k = 0; k < kIn; ++k) put_bf16(sm.ga, k, tid, kLboGA, f[k]);  // X^T
        }
        float y, h1[kHid], h2[kHid];
        if (!(ok = mlp_tile(sm, phase, &y, h1, h2))) break;
        const float e = valid ? y - R[row] : 0.f;
        const float dy = 2.f * e * inv_n;
        lsum += e * e * inv_n;
        db3 += dy;
        float dz[kHid];
#pragma unroll
        for (int j = 0; j < kHid; ++j) {
            dz[j] = dy * sm.w3[j] * (1.f - h2[j] * h2[j]);
            dw3[j] = fmaf(dy, h2[j], dw3[j]);
            put_bf16(sm.gb, kHid + j, tid, kLboGB, dz[j]);  // dZ2^T
            put_bf16(sm.ga, kIn + j, tid, kLboGA, h1[j]);    // H1^T (h1 holds BF16 values)
        }
        put_row(sm.a2, tid, dz, kHid, kLboA);  // the layer-2 MMA has completed (mlp_tile waited)
        // dh1 = dz2 W2
        if (!(ok = mma_chain(&sm.bar, phase, sm.tmem + kColDh1, sm.a2, kLboA, sm.w2t, (kHid / 8) * 128, kIdesc,
                             kHid / 16, false)))
            break;
        umma::tmem_ld32(lane_base + kColDh1, dz);
#pragma unroll
        for (int k = 0; k < kHid; ++k) put_bf16(sm.gb, k, tid, kLboGB, dz[k] * (1.f - h1[k] * h1[k]));  // dZ1^T
        // every weight and bias gradient of the hidden layers, accumulated over the tiles
        if (!(ok = mma_chain(&sm.bar, phase, sm.tmem + kColG, sm.ga, kLboGA, sm.gb, kLboGB, kIdescG, kTile / 16,
                             done > 0)))
            break;
        ++done;
    }
    if (!ok) {
        if (tid == 0 && err) atomicOr(err, 2u);
    } else if (done > 0) {
        float *out = part + (size_t)blockIdx.x * kPartStride;
        float g[32];
        umma::tmem_ld32(lane_base + kColG, g);  // D row tid, columns 0 .. 31 (the dZ1 block)
        if (tid < kIn) {
#pragma unroll
            for (int i = 0; i < kHid; ++i) out[kOffW1 + i * kIn + tid] = g[i];   // dW1[i][tid]
        } else if (tid == kRowOnes) {
#pragma unroll
            for (int i = 0; i < kHid; ++i) out[kOffB1 + i] = g[i];
        }
        umma::tmem_ld32(lane_base + kColG + kHid, g);  // columns 32 .. 63 (the dZ2 block)
        if (tid >= kIn && tid < kRowOnes) {
#pragma unroll
            for (int i = 0; i < kHid; ++i) out[kOffW2 + i * kHid + (tid - kIn)] = g[i];  // dW2[i][tid - 64]
        } else if (tid == kRowOnes) {
#pragma unroll
            for (int i = 0; i < kHid; ++i) out[kOffB2 + i] = g[i];
        }
        // dw3, db3 and the loss: warp sums, then the warps in order
#pragma unroll
        for (int j = 0; j < kHid + 2; ++j) {
            float v = j < kHid ? dw3[j] : (j == kHid ? db3 : lsum);
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            if (lane == 0) sm.red[warp][j] = v;
        }
        __syncthreads();
        if (tid < kHid + 2) {
            float v = 0.f;
            for (int w = 0; w < kTile / 32; ++w) v += sm.red[w][tid];
            out[tid < kHid ? kOffW3 + tid : (tid == kHid ? kOffB3 : kNParam)] = v;
        }
    }
    mlp_teardown<GradSmem, kTmemColsG>(sm);
}

// g[p] = sum over the CTAs' partials, in CTA order; the loss (index kNParam) into *loss.
__global__ void grad_sum_kernel(const float *__restrict__ part, int nparts, float *g, float *loss) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p > kNParam) return;
    float a = 0.f;
    for (int c = 0; c < nparts; ++c) a += part[(size_t)c * kPartStride + p];
    if (p < kNParam) g[p] = a;
    else if (loss) *loss = a;
}

// Adam (beta1 0.9, beta2 0.999, eps 1e-8) with bias correction; step counts from 1.
__global__ void adam_kernel(float *prm, const float *__restrict__ g, float *m, float *v, int step, float lr) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= kNParam) return;
    const float b1 = 0.9f, b2 = 0.999f;
    const float mm = b1 * m[p] + (1.f - b1) * g[p];
    const float vv = b2 * v[p] + (1.f - b2) * g[p] * g[p];
    m[p] = mm;
    v[p] = vv;
    const float mh = mm / (1.f - powf(b1, (float)step)), vh = vv / (1.f - powf(b2, (float)step));
    prm[p] -= lr * mh / (sqrtf(vh) + 1e-8f);
}

// Grid of mlp_grad_kernel (one CTA per tile up to two per SM; its dynamic shared memory opted in
// once per device), or 0 when the attribute cannot be set.
int grad_grid(long long tiles) {
    static unsigned long long done = 0;
    int dev = 0;
    cudaGetDevice(&dev);
    const unsigned long long bit = 1ull << (dev & 63);
    if (!(done & bit)) {
        if (cudaFuncSetAttribute(mlp_grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(GradSmem)) !=
            cudaSuccess)
            return 0;
        done |= bit;
    }
    return (int)(tiles < 2 * 148 ? tiles : 2 * 148);
}

int grid_for(long long tiles) {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const long long g = (long long)sms * 6;
    return (int)(tiles < g ? (tiles > 0 ? tiles : 1) : g);
}

}  // namespace

// The network's cells of box b (the outer kNet cells of its strip), ordered by array offset, with
// their face codes.
void strip_cells(const Box &b, std::vector<uint32_t> &cells, std::vector<uint8_t> &faces) {
    cells.clear();
    faces.clear();
    for (int x = 0; x < b.nx; ++x)
        for (int y = 0; y < b.ny; ++y) {
            const bool full = x < kNet || x >= b.nx - kNet || y < kNet || y >= b.ny - kNet;
            for (int z = 0; z < b.nz; ++z) {
                if (!full && z == kNet && b.nz - kNet > kNet) z = b.nz - kNet;
                const int f = face_of(x, y, z, b.nx, b.ny, b.nz);
                if (f < 0) continue;
                cells.push_back((uint32_t)(((size_t)(x + b.ox) * b.ay + (y + b.oy)) * b.az + (z + b.oz)));
                faces.push_back((uint8_t)f);
            }
        }
}

cudaError_t launch_strip_step(const float *prm, const float *P, const float *PP, const float *V, const Box &b,
                              const uint32_t *cells, const uint8_t *faces, long long ncells, float inv_dx,
                              float min_scale, float damp, float *side, unsigned *err, cudaStream_t s) {
    const long long tiles = (ncells + kTile - 1) / kTile;
    strip_step_kernel<<<grid_for(tiles), kTile, 0, s>>>(prm, P, PP, V, b, cells, faces, ncells, inv_dx, min_scale,
                                                        damp, side, err);
    return cudaGetLastError();
}

cudaError_t launch_strip_scatter(float *PP, const uint32_t *cells, const float *side, long long ncells,
                                 cudaStream_t s) {
    const long long blocks = (ncells + 255) / 256;
    strip_scatter_kernel<<<(unsigned)(blocks < 148 * 32 ? (blocks > 0 ? blocks : 1) : 148 * 32), 256, 0, s>>>(
        PP, cells, side, ncells);
    return cudaGetLastError();
}

}  // namespace closure
}  // namespace rtmb

// ------------------------------------------------------------------ entry points

using namespace rtmb::closure;

namespace {

thread_local std::string g_closure_err;

int cfail(int code, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    return rtmb::driver::fail_noctx(code, buf);
}

#define CKC(call)                                                                                 \
    do {                                                                                          \
        cudaError_t e_ = (call);                                                                  \
        if (e_ != cudaSuccess)                                                                    \
            return cfail(e_ == cudaErrorMemoryAllocation ? RTMB_ENOMEM : RTMB_ECUDA, "%s: %s", #call, \
                         cudaGetErrorString(e_));                                                 \
    } while (0)

// Reads and clears an error word; maps bit 1 to ETIMEOUT and bit 0 to ENAN.
int read_err(unsigned *d_err, cudaStream_t s) {
    unsigned h = 0;
    CKC(cudaMemcpyAsync(&h, d_err, sizeof h, cudaMemcpyDeviceToHost, s));
    CKC(cudaStreamSynchronize(s));
    if (h & 2u) return cfail(RTMB_ETIMEOUT, "closure: a bounded wait for a tensor-core MMA ran out");
    if (h & 1u) return cfail(RTMB_ENAN, "closure: a NaN appeared");
    return RTMB_OK;
}

}  // namespace

extern "C" {

int rtmb_closure_param_count(void) { return kNParam; }

int rtmb_closure_init(float *params, uint64_t seed) {
    if (!params) return cfail(RTMB_EINVAL, "rtmb_closure_init: null pointer");
    std::memset(params, 0, sizeof(float) * kNParam);
    uint64_t st = seed ? seed : 1;
    auto uni = [&]() {  // xorshift64*, uniform in [-1, 1)
        st ^= st >> 12; st ^= st << 25; st ^= st >> 27;
        return (double)((st * 2685821657736338717ull) >> 11) / 4503599627370496.0 - 1.0;
    };
    const double a1 = std::sqrt(6.0 / (kUsed + kHid)), a2 = std::sqrt(6.0 / (2 * kHid)), a3 = std::sqrt(6.0 / (kHid + 1));
    for (int j = 0; j < kHid; ++j)
        for (int k = 0; k < kUsed; ++k) params[kOffW1 + j * kIn + k] = (float)(a1 * uni());
    for (int i = 0; i < kHid * kHid; ++i) params[kOffW2 + i] = (float)(a2 * uni());
    for (int j = 0; j < kHid; ++j) params[kOffW3 + j] = (float)(a3 * uni());
    return RTMB_OK;
}

int rtmb_closure_forward(const float *params, const void *X, uint64_t n, float *y, void *stream) {
    if (!params || (!X && n) || (!y && n)) return cfail(RTMB_EINVAL, "rtmb_closure_forward: null pointer");
    if (!n) return RTMB_OK;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    unsigned *err = nullptr;
    CKC(cudaMallocAsync(&err, sizeof(unsigned), s));
    CKC(cudaMemsetAsync(err, 0, sizeof(unsigned), s));
    const long long tiles = ((long long)n + kTile - 1) / kTile;
    mlp_forward_kernel<<<grid_for(tiles), kTile, 0, s>>>(params, static_cast<const __nv_bfloat16 *>(X), (long long)n,
                                                         y, nullptr, nullptr, err);
    CKC(cudaGetLastError());
    const int rc = read_err(err, s);
    cudaFreeAsync(err, s);
    return rc;
}

int rtmb_closure_grad(const float *params, const void *X, const float *R, uint32_t n, float *grad, float *loss,
                      void *stream) {
    if (!params || !X || !R || !grad || !loss || !n) return cfail(RTMB_EINVAL, "rtmb_closure_grad: bad argument");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const long long tiles = ((long long)n + kTile - 1) / kTile;
    const int grid = grad_grid(tiles);
    if (grid <= 0) return cfail(RTMB_ECUDA, "rtmb_closure_grad: kernel set-up failed");
    float *part = nullptr;
    CKC(cudaMallocAsync(&part, ((size_t)grid * kPartStride + 4) * sizeof(float), s));
    unsigned *err = reinterpret_cast<unsigned *>(part + (size_t)grid * kPartStride);
    CKC(cudaMemsetAsync(part, 0, ((size_t)grid * kPartStride + 4) * sizeof(float), s));
    mlp_grad_kernel<<<grid, kTile, sizeof(GradSmem), s>>>(params, static_cast<const __nv_bfloat16 *>(X), R, n, part, err);
    grad_sum_kernel<<<(kNParam + 1 + 127) / 128, 128, 0, s>>>(part, grid, grad, loss);
    CKC(cudaGetLastError());
    const int rc = read_err(err, s);
    cudaFreeAsync(part, s);
    return rc;
}

int rtmb_closure_train(float *params, const void *X, const float *R, uint64_t n, uint32_t steps, uint32_t batch,
                       float lr, float noise, uint64_t seed, float *loss_host, void *stream) {
    if (!params || !X || !R || !n || !batch || batch > 65536) return cfail(RTMB_EINVAL, "rtmb_closure_train: bad argument");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const size_t B = batch;
    const long long tiles = ((long long)B + kTile - 1) / kTile;
    const int grid = grad_grid(tiles);
    if (grid <= 0) return cfail(RTMB_ECUDA, "rtmb_closure_train: kernel set-up failed");
    const size_t nf = 3 * kNParam + B + (size_t)grid * kPartStride + steps + 4;
    float *buf = nullptr;
    __nv_bfloat16 *Xb = nullptr;
    CKC(cudaMallocAsync(&buf, nf * sizeof(float), s));
    CKC(cudaMallocAsync(&Xb, B * kIn * sizeof(__nv_bfloat16), s));
    CKC(cudaMemsetAsync(buf, 0, nf * sizeof(float), s));
    float *g = buf, *m = g + kNParam, *v = m + kNParam, *Rb = v + kNParam, *part = Rb + B,
          *losses = part + (size_t)grid * kPartStride;
    unsigned *err = reinterpret_cast<unsigned *>(losses + steps);
    const auto *Xd = static_cast<const __nv_bfloat16 *>(X);
    for (uint32_t st = 0; st < steps; ++st) {
        gather_batch_kernel<<<(unsigned)B, 32, 0, s>>>(Xd, R, (long long)n, (int)B, mix64(seed * 1000003ull + st), noise,
                                                       Xb, Rb);
        // forward, backward and every weight gradient on the tensor cores, then the CTAs' sums
        mlp_grad_kernel<<<grid, kTile, sizeof(GradSmem), s>>>(params, Xb, Rb, (long long)B, part, err);
        grad_sum_kernel<<<(kNParam + 1 + 127) / 128, 128, 0, s>>>(part, grid, g, losses + st);
        adam_kernel<<<(kNParam + 127) / 128, 128, 0, s>>>(params, g, m, v, (int)st + 1, lr);
        CKC(cudaGetLastError());
    }
    if (loss_host) CKC(cudaMemcpyAsync(loss_host, losses, steps * sizeof(float), cudaMemcpyDeviceToHost, s));
    const int rc = read_err(err, s);
    cudaFreeAsync(Xb, s);
    cudaFreeAsync(buf, s);
    return rc;
}

}  // extern "C"

namespace {

// Collection of training pairs around the steps of a wide-domain modeling shot.
struct CollectHook : rtmb::driver::StepHook {
    rtmb_ctx *ctx;
    Box box;
    const uint32_t *cells;
    const uint8_t *faces;
    long long ncells;
    int t0, tstride, per_step;
    uint64_t seed;
    float inv_dx, min_scale;
    __nv_bfloat16 *X, *Xs;
    float *R;
    unsigned long long cap, *count;
    long long *slot_of;
    float *stash;
    bool due(int it) const { return it >= t0 && (it - t0) % tstride == 0; }
    int before(int it, const float *P, float *PP) override {
        if (!due(it)) return 0;
        sample_features_kernel<<<(per_step + 127) / 128, 128, 0, ctx->stream>>>(
            P, PP, ctx->d_v2dt2, box, cells, faces, ncells, per_step, mix64(seed ^ (0x5851F42D4C957F2Dull * (it + 1))),
            inv_dx, min_scale, Xs, slot_of, stash);
        compact_rows_kernel<<<1, 1024, 0, ctx->stream>>>(Xs, per_step, X, cap, count, slot_of);
        ctx->launches += 2;
        return cudaGetLastError() == cudaSuccess ? 0 : RTMB_ECUDA;
    }
    int after(int it, const float *, float *PP) override {
        if (!due(it)) return 0;
        sample_target_kernel<<<(per_step + 127) / 128, 128, 0, ctx->stream>>>(PP, per_step, slot_of, stash, R);
        ++ctx->launches;
        return cudaGetLastError() == cudaSuccess ? 0 : RTMB_ECUDA;
    }
};

}  // namespace

int rtmb::driver::closure_hook_before(rtmb_ctx *ctx, const float *P, float *PP) {
    const Box b{ctx->nxe, ctx->nye, ctx->nze, 0, 0, 0, ctx->nxe, ctx->nye, ctx->nze};
    return launch_strip_step(ctx->d_cparams, P, PP, ctx->d_v2dt2, b, ctx->d_cells, ctx->d_faces, ctx->ncells,
                             1.f / ctx->p.dx, ctx->closure_min_scale, ctx->closure_damp, ctx->d_side, ctx->d_err,
                             ctx->stream) == cudaSuccess
               ? 0
               : RTMB_ECUDA;
}

int rtmb::driver::closure_hook_after(rtmb_ctx *ctx, float *PP) {
    return launch_strip_scatter(PP, ctx->d_cells, ctx->d_side, ctx->ncells, ctx->stream) == cudaSuccess ? 0 : RTMB_ECUDA;
}

extern "C" {

int rtmb_closure_set(rtmb_ctx *ctx, const float *params, float min_scale, float damp) {
    if (!ctx || !params || !(min_scale >= 0.f) || !(damp >= 0.f && damp < 1.f)) return RTMB_EINVAL;
    ctx->closure_min_scale = min_scale;
    ctx->closure_damp = damp;
    if (ctx->p.boundary != RTMB_BC_LEARNED || ctx->p.blen != (uint32_t)kStrip || ctx->p.nx == 1) {
        ctx->err = "rtmb_closure_set: the context needs boundary RTMB_BC_LEARNED, blen 8 and a 3D model";
        return RTMB_EINVAL;
    }
    if (cudaSetDevice(ctx->device) != cudaSuccess) return RTMB_ECUDA;
    if (!ctx->d_cells) {
        const Box b{ctx->nxe, ctx->nye, ctx->nze, 0, 0, 0, ctx->nxe, ctx->nye, ctx->nze};
        std::vector<uint32_t> cells;
        std::vector<uint8_t> faces;
        if (ctx->n > 0xFFFFFFFFull) {
            ctx->err = "rtmb_closure_set: grids above 2^32 points are not supported";
            return RTMB_EINVAL;
        }
        strip_cells(b, cells, faces);
        ctx->ncells = (long long)cells.size();
        if (cudaMalloc(&ctx->d_cells, cells.size() * sizeof(uint32_t)) != cudaSuccess ||
            cudaMalloc(&ctx->d_faces, faces.size()) != cudaSuccess ||
            cudaMalloc(&ctx->d_side, cells.size() * sizeof(float)) != cudaSuccess ||
            cudaMalloc(&ctx->d_cparams, kNParam * sizeof(float)) != cudaSuccess) {
            ctx->err = "rtmb_closure_set: device allocation failed";
            return RTMB_ENOMEM;
        }
        if (cudaMemcpy(ctx->d_cells, cells.data(), cells.size() * sizeof(uint32_t), cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemcpy(ctx->d_faces, faces.data(), faces.size(), cudaMemcpyHostToDevice) != cudaSuccess)
            return RTMB_ECUDA;
    }
    if (cudaMemcpyAsync(ctx->d_cparams, params, kNParam * sizeof(float), cudaMemcpyDefault, ctx->stream) != cudaSuccess ||
        cudaStreamSynchronize(ctx->stream) != cudaSuccess)
        return RTMB_ECUDA;
    return RTMB_OK;
}

// Reflected energy of a bordered run: the record rel-L2 against the wide run's record, both modeled
// on device (the same model, receivers and shot; only the border differs).
namespace {
int model_record(rtmb_ctx *c, uint32_t sx, uint32_t sy, uint32_t sz, float *rec) {
    const int rc = rtmb_model_shot(c, sx, sy, sz, rec);
    return rc ? rc : rtmb_sync(c);
}
}  // namespace

int rtmb_closure_judge(rtmb_ctx *learned, rtmb_ctx *hbc, rtmb_ctx *wide, uint32_t sx, uint32_t sy, uint32_t sz,
                       float *refl_learned, float *refl_hbc) {
    if (!learned || !hbc || !wide) return RTMB_EINVAL;
    const rtmb_params &a = learned->p, &b = hbc->p, &w = wide->p;
    auto same = [](const rtmb_params &x, const rtmb_params &y) {
        return x.nx == y.nx && x.ny == y.ny && x.nz == y.nz && x.nt == y.nt && x.ntstep == y.ntstep &&
               x.receiver_start_x == y.receiver_start_x && x.receiver_start_y == y.receiver_start_y &&
               x.receiver_depth_z == y.receiver_depth_z && x.receiver_distance_x == y.receiver_distance_x &&
               x.receiver_distance_y == y.receiver_distance_y && x.receiver_count_x == y.receiver_count_x &&
               x.receiver_count_y == y.receiver_count_y && x.device == y.device;
    };
    if (a.boundary != RTMB_BC_LEARNED || !learned->d_cparams || b.boundary == RTMB_BC_LEARNED ||
        w.boundary == RTMB_BC_LEARNED || !same(a, b) || !same(a, w) || w.blen <= b.blen) {
        learned->err = "rtmb_closure_judge: a learned context with its closure installed, a taper-border context "
                       "and a wider one, on the same model, receivers, nt and device";
        return RTMB_EINVAL;
    }
    if (cudaSetDevice(learned->device) != cudaSuccess) return RTMB_ECUDA;
    const size_t nrec = (size_t)a.nt * a.receiver_count_x * a.receiver_count_y;
    float *rec = nullptr;
    double *acc = nullptr;
    if (cudaMalloc(&rec, 3 * nrec * sizeof(float)) != cudaSuccess || cudaMalloc(&acc, 4 * sizeof(double)) != cudaSuccess) {
        if (rec) cudaFree(rec);
        learned->err = "rtmb_closure_judge: device allocation failed";
        return RTMB_ENOMEM;
    }
    int rc = model_record(wide, sx, sy, sz, rec);
    if (!rc) rc = model_record(learned, sx, sy, sz, rec + nrec);
    if (!rc) rc = model_record(hbc, sx, sy, sz, rec + 2 * nrec);
    double h[4] = {0, 0, 0, 0};
    if (!rc) {
        cudaStream_t s = learned->stream;
        const bool ok = cudaMemsetAsync(acc, 0, 4 * sizeof(double), s) == cudaSuccess &&
                        rtmb::launch_sqdiff(rec + nrec, rec, nrec, acc, s) == cudaSuccess &&
                        rtmb::launch_sqdiff(rec + 2 * nrec, rec, nrec, acc + 2, s) == cudaSuccess &&
                        cudaMemcpyAsync(h, acc, sizeof h, cudaMemcpyDeviceToHost, s) == cudaSuccess &&
                        cudaStreamSynchronize(s) == cudaSuccess;
        if (!ok) rc = RTMB_ECUDA;
    }
    cudaFree(rec);
    cudaFree(acc);
    if (rc) return rc;
    const float rl = h[1] > 0 ? (float)std::sqrt(h[0] / h[1]) : 0.f;
    const float rh = h[3] > 0 ? (float)std::sqrt(h[2] / h[3]) : 0.f;
    // the judge: the learned strip may reflect no more than the 32-cell taper border
    learned->closure_verdict = rl <= rh ? 1 : 2;
    if (refl_learned) *refl_learned = rl;
    if (refl_hbc) *refl_hbc = rh;
    return RTMB_OK;
}

int rtmb_model_shot_judged(rtmb_ctx *learned, rtmb_ctx *fallback, uint32_t sx, uint32_t sy, uint32_t sz, float *rec,
                           int *ran) {
    if (!learned || !fallback || !rec) return RTMB_EINVAL;
    if (learned->closure_verdict == 0) {
        learned->err = "rtmb_model_shot_judged: judge the closure first (rtmb_closure_judge)";
        return RTMB_EINVAL;
    }
    if (fallback->p.boundary == RTMB_BC_LEARNED || fallback->p.nt != learned->p.nt ||
        fallback->p.receiver_count_x != learned->p.receiver_count_x ||
        fallback->p.receiver_count_y != learned->p.receiver_count_y) {
        learned->err = "rtmb_model_shot_judged: the fallback context must be a taper-border context of the same shot geometry";
        return RTMB_EINVAL;
    }
    const bool use_learned = learned->closure_verdict == 1;
    if (ran) *ran = use_learned ? RTMB_BC_LEARNED : (int)fallback->p.boundary;
    return rtmb_model_shot(use_learned ? learned : fallback, sx, sy, sz, rec);
}

int rtmb_closure_collect(rtmb_ctx *wide, uint32_t sx, uint32_t sy, uint32_t sz, uint32_t t0, uint32_t tstride,
                         uint32_t per_step, uint64_t seed, float min_scale, void *X, float *R, uint64_t capacity,
                         uint64_t *count) {
    if (!wide || !X || !R || !count || !tstride || !per_step) return RTMB_EINVAL;
    rtmb_ctx *ctx = wide;
    const rtmb_params &p = ctx->p;
    if (p.blen < (uint32_t)kStrip + 8 || p.nx == 1) {
        ctx->err = "rtmb_closure_collect: a 3D wide context whose border is wider than the 8-cell strip";
        return RTMB_EINVAL;
    }
    int rc = rtmb::driver::check_model_shot(ctx, sx, sy, sz);
    if (rc) return rc;
    if (!ctx->d_w[0] && (cudaMalloc(&ctx->d_w[0], ctx->n * sizeof(float)) != cudaSuccess ||
                         cudaMalloc(&ctx->d_w[1], ctx->n * sizeof(float)) != cudaSuccess))
        return RTMB_ENOMEM;
    const int o = (int)p.blen - kStrip;
    const Box box{ctx->nxe, ctx->nye, ctx->nze, o, o, o, (int)p.nx + 2 * kStrip, (int)p.ny + 2 * kStrip,
                  (int)p.nz + 2 * kStrip};
    std::vector<uint32_t> cells;
    std::vector<uint8_t> faces;
    strip_cells(box, cells, faces);
    uint32_t *d_cells = nullptr;
    uint8_t *d_faces = nullptr;
    long long *slot_of = nullptr;
    float *stash = nullptr;
    __nv_bfloat16 *Xs = nullptr;
    unsigned long long *d_count = nullptr;
    auto cleanup = [&]() {
        cudaFree(d_cells); cudaFree(d_faces); cudaFree(slot_of); cudaFree(stash); cudaFree(d_count); cudaFree(Xs);
    };
    if (cudaMalloc(&d_cells, cells.size() * 4) != cudaSuccess || cudaMalloc(&d_faces, faces.size()) != cudaSuccess ||
        cudaMalloc(&slot_of, per_step * sizeof(long long)) != cudaSuccess ||
        cudaMalloc(&stash, 3 * (size_t)per_step * sizeof(float)) != cudaSuccess ||
        cudaMalloc(&d_count, sizeof(unsigned long long)) != cudaSuccess ||
        cudaMalloc(&Xs, (size_t)per_step * kIn * sizeof(__nv_bfloat16)) != cudaSuccess) {
        cleanup();
        return RTMB_ENOMEM;
    }
    cudaMemcpy(d_cells, cells.data(), cells.size() * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(d_faces, faces.data(), faces.size(), cudaMemcpyHostToDevice);
    cudaMemsetAsync(d_count, 0, sizeof(unsigned long long), ctx->stream);
    CollectHook hook;
    hook.ctx = ctx; hook.box = box; hook.cells = d_cells; hook.faces = d_faces; hook.ncells = (long long)cells.size();
    hook.t0 = (int)t0; hook.tstride = (int)tstride; hook.per_step = (int)per_step; hook.seed = seed;
    hook.inv_dx = 1.f / p.dx; hook.min_scale = min_scale; hook.X = static_cast<__nv_bfloat16 *>(X); hook.R = R; hook.cap = capacity;
    hook.count = d_count; hook.slot_of = slot_of; hook.stash = stash; hook.Xs = Xs;
    float *P = nullptr, *PP = nullptr;
    rc = rtmb::driver::run_forward(ctx, sx, sy, sz, rtmb::kTaperAll, nullptr, nullptr, &P, &PP, RTMB_PROF_MODEL,
                                   nullptr, &hook);
    unsigned long long h = 0;
    if (!rc && cudaMemcpyAsync(&h, d_count, sizeof h, cudaMemcpyDeviceToHost, ctx->stream) != cudaSuccess) rc = RTMB_ECUDA;
    if (!rc) rc = rtmb::driver::check_err_flag(ctx);
    cleanup();
    *count = h < capacity ? h : capacity;
    return rc;
}

}  // extern "C"
