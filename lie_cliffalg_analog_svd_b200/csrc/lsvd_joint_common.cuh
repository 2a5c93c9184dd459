// lsvd_joint_common.cuh -- constants and helpers shared by the blocked joint
// kernels (Phase-JADE, lsvd_jade.cu; two-sided joint SVD, lsvd_jsvd.cu).
#pragma once

#include <cuda_runtime.h>

namespace lsvd {
namespace joint {

constexpr int B = 8;        // block size
constexpr int B2 = 2 * B;   // indices of a block pair
// Shared sub-block layout of the solve kernels: row stride B2 + 1 and matrix
// stride B2 (B2 + 1) + 1 doubles, so that lanes walking a column, or the same
// entry of consecutive matrices, fall in different banks.
constexpr int SLD = B2 + 1, MST = B2 * SLD + 1;
constexpr int kThreads = 256;
constexpr double kPi = 3.141592653589793238462643383279502884;

__device__ __forceinline__ double warp_sum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ double wrap_quarter(double a) {  // wrap_jacobi_angle, src/lie_svd_joint.rs:506-514
    while (a > 0.25 * kPi) a -= 0.5 * kPi;
    while (a < -0.25 * kPi) a += 0.5 * kPi;
    return a;
}

__device__ __forceinline__ double wrap_half(double a) {  // wrap to (-pi/2, pi/2], src/lie_svd_joint.rs:293-301
    while (a > 0.5 * kPi) a -= kPi;
    while (a <= -0.5 * kPi) a += kPi;
    return a;
}

// Pair k of round-robin layer `layer` over m (even) items: the circle method
// of layer_pairs, src/lie_svd_joint.rs:524-539.
__device__ __forceinline__ void rr_pair(int m, int layer, int k, int& a, int& b) {
    const int ring = m - 1;
    if (k == 0) {
        a = m - 1;
        b = layer % ring;
    } else {
        a = (layer + k) % ring;
        b = (layer + ring - k) % ring;
    }
}

// Global index of position `pos` (0 .. 2B-1) of the block pair (blk_lo,
// blk_hi); -1 past the limit n.
__device__ __forceinline__ int block_pos(int blk_lo, int blk_hi, int pos, int n) {
    const int g = (pos < B ? blk_lo : blk_hi) * B + (pos % B);
    return g < n ? g : -1;
}

}  // namespace joint
}  // namespace lsvd
