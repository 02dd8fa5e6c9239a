// closure.cuh -- the learned absorbing-boundary closure: a per-cell MLP (55 -> 32 -> 32 -> 1, tanh)
// that advances the cells of an 8-cell boundary strip one time step.
//
// Inputs of a strip cell (55, padded to 64 with zeros): the 3x3x3 neighbourhood of p(t) (27) and of
// p(t-1) (27), both divided by s = max |value| over those 54, and the local Courant number
// v dt / dx = sqrt(v2dt2) / dx.  The neighbourhood is read in the cell's canonical frame: axis u is
// the inward normal of the strip face nearest to the cell (feature index (u+1)*9 + (v+1)*3 + (w+1),
// v and w along the other two axes in x, y, z order), and neighbours outside the domain read 0.
// Output: r, the correction to the first-order one-way (upwind) update of an outgoing wave,
//     p(t+1) = p + C (p_in - p) + s * clamp(r, -0.5, 0.5)
// with p_in the inward neighbour at t and C the Courant number.  The map is scale-equivariant by
// construction.  The network advances the outer 4 cells of the strip (the stencil, half width 4,
// advances the inner 4, which only it can do exactly); each new value is damped by
// 1 - damp ((4 - depth)/4)^2 and kept within [-s, s], so the network cannot amplify what reaches the
// strip.  Training pairs come from a run of the plain method on a domain padded so widely that no
// boundary reflection returns in the time window: r = (p_wide(t+1) - upwind update) / s.
//
// The two hidden layers run on the 5th-generation tensor cores (tcgen05.mma, BF16 operands, FP32
// accumulation in TMEM), M = 128 cells per tile.
#pragma once
#include <cstdint>
#include <vector>

#include <cuda_runtime.h>

namespace rtmb {
namespace closure {

constexpr int kStrip = 8;     // strip width (cells): the padded border of a learned-closure grid
constexpr int kNet = 4;       // outer cells of the strip the network advances; the stencil (half
                              // width 4) advances the inner ones, which only it can do exactly
constexpr int kIn = 64;       // input features per cell (55 used)
constexpr int kUsed = 55;
constexpr int kHid = 32;
// parameter layout (floats): W1 [32][64], b1 [32], W2 [32][32], b2 [32], w3 [32], b3
constexpr int kOffW1 = 0, kOffB1 = kHid * kIn, kOffW2 = kOffB1 + kHid, kOffB2 = kOffW2 + kHid * kHid,
              kOffW3 = kOffB2 + kHid, kOffB3 = kOffW3 + kHid, kNParam = kOffB3 + 1;

// The cells of the strip of a box [o, o+n) per axis inside an array of extents (ax, ay, az):
// linear offsets in the array and the face code (axis * 2 + side) of each cell.
struct Box {
    int ax, ay, az;      // array extents (x, y, z)
    int ox, oy, oz;      // box origin
    int nx, ny, nz;      // box extents
};

// Strip cells of box b, ordered by array offset, with their face codes (host).
void strip_cells(const Box &b, std::vector<uint32_t> &cells, std::vector<uint8_t> &faces);
// side[i] = p(t+1) of strip cell i from P = p(t), PP = p(t-1) and V = v2dt2 (the MLP on tensor cores).
// Cells whose neighbourhood max |p| is below min_scale are set to zero; the others are multiplied
// by 1 - damp * ((4 - depth) / 4)^2 (depth 0 at the outer face).
cudaError_t launch_strip_step(const float *prm, const float *P, const float *PP, const float *V, const Box &b,
                              const uint32_t *cells, const uint8_t *faces, long long ncells, float inv_dx,
                              float min_scale, float damp, float *side, unsigned *err, cudaStream_t s);
// PP[cells[i]] = side[i].
cudaError_t launch_strip_scatter(float *PP, const uint32_t *cells, const float *side, long long ncells,
                                 cudaStream_t s);

}  // namespace closure
}  // namespace rtmb
