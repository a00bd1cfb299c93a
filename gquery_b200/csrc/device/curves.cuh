// Space-filling-curve keys of grid cells, used to order queries so that the 32 queries of
// a warp lie close together: Morton codes (bit interleaving) and Hilbert indices.
// Consecutive Hilbert indices are face-adjacent cells, so a run of sorted points spans a
// more compact region than along a Morton curve, whose runs jump between distant
// quadrants / octants.  Hilbert indices by Skilling's method (J. Skilling, "Programming
// the Hilbert curve", AIP Conf. Proc. 707, 2004): the axes are turned into the transposed
// index by the inverse undo and Gray encoding, whose bits are then interleaved like a
// Morton code.
#pragma once

#include <cstdint>

namespace gqd {

__device__ __forceinline__ uint32_t spread3(uint32_t v) {  // 10 bits -> every third bit
    v &= 0x3ffu;
    v = (v | (v << 16)) & 0x030000ffu;
    v = (v | (v << 8)) & 0x0300f00fu;
    v = (v | (v << 4)) & 0x030c30c3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}

__device__ __forceinline__ uint32_t spread2(uint32_t v) {  // 15 bits -> every second bit
    v &= 0x7fffu;
    v = (v | (v << 8)) & 0x00ff00ffu;
    v = (v | (v << 4)) & 0x0f0f0f0fu;
    v = (v | (v << 2)) & 0x33333333u;
    v = (v | (v << 1)) & 0x55555555u;
    return v;
}

// Hilbert index of cell x[0..N) on a grid of 2^B cells per axis (N * B <= 32 bits).
template <int N, int B>
__device__ __forceinline__ uint32_t hilbert(uint32_t (&x)[N]) {
#pragma unroll
    for (uint32_t q = 1u << (B - 1); q > 1; q >>= 1) {
        const uint32_t p = q - 1;
#pragma unroll
        for (int i = 0; i < N; ++i) {
            if (x[i] & q) {
                x[0] ^= p;
            } else {
                const uint32_t t = (x[0] ^ x[i]) & p;
                x[0] ^= t;
                x[i] ^= t;
            }
        }
    }
#pragma unroll
    for (int i = 1; i < N; ++i) x[i] ^= x[i - 1];
    uint32_t t = 0;
#pragma unroll
    for (uint32_t q = 1u << (B - 1); q > 1; q >>= 1)
        if (x[N - 1] & q) t ^= q - 1;
#pragma unroll
    for (int i = 0; i < N; ++i) x[i] ^= t;
    if (N == 3) return (spread3(x[0]) << 2) | (spread3(x[1]) << 1) | spread3(x[N - 1]);
    return (spread2(x[0]) << 1) | spread2(x[N - 1]);
}

// 3D: 1024 cells per axis; 2D: 32768 cells per axis (30-bit indices)
__device__ __forceinline__ uint32_t hilbert3(uint32_t x0, uint32_t x1, uint32_t x2) {
    uint32_t x[3] = {x0, x1, x2};
    return hilbert<3, 10>(x);
}
__device__ __forceinline__ uint32_t hilbert2(uint32_t x0, uint32_t x1) {
    uint32_t x[2] = {x0, x1};
    return hilbert<2, 15>(x);
}

}  // namespace gqd
