// dssim_tile_map.h -- geometry of the DSSIM tile pass (dssim_kernels.cu) and
// the thread-to-item mapping of its blur stages, for the device and for the
// host-side check of that mapping (tests/dssim_map_check.cu).
#pragma once

#include <cuda_runtime.h>

namespace s2 {

constexpr int kDsT = 32;             // output tile edge
constexpr int kDsThreads = 256;
constexpr int kDsR = kDsT + 8;       // raw a/b region (halo 4)
constexpr int kDsP = kDsT + 6;       // first a/b pre-blur (halo 3)
constexpr int kDsX = kDsT + 4;       // blur input x, y (halo 2)
constexpr int kDsB = kDsT + 2;       // first statistics blur (halo 1)

// Row segments (S) and rows per run (L) of the three stage blurs: the first
// and second a/b pre-blurs (2 planes each) and the first statistics blur (5
// planes); each stage's planes x (n / 2) column pairs x S items fit the block.
constexpr int kDsPre1S = 6, kDsPre1L = 7;
constexpr int kDsPre2S = 6, kDsPre2L = 6;
constexpr int kDsStatS = 3, kDsStatL = 12;

// Thread t's item of a blur stage: plane p, row segment seg, column pair
// c (even).  The first 16 column pairs of every (plane, segment) go to one
// aligned half-warp, whose 16 lanes read 32 consecutive floats of a row (no
// shared-memory bank conflicts); the remaining half - 16 pairs of every
// (plane, segment) go to the threads after those.  Returns false for a
// thread without an item.
template <int half, int S, int planes>
__host__ __device__ __forceinline__ bool ds_item(int t, int &p, int &seg, int &c) {
    static_assert(half >= 16, "a half-warp of column pairs per row segment");
    constexpr int G = planes * S, extra = half - 16;
    if (t < 16 * G) {
        const int g = t >> 4;
        p = g / S;
        seg = g - p * S;
        c = 2 * (t & 15);
        return true;
    }
    if (extra == 0) return false;
    const int u = t - 16 * G;
    if (u >= G * extra) return false;
    const int g = u / extra;
    p = g / S;
    seg = g - p * S;
    c = 2 * (16 + (u - g * extra));
    return true;
}

}  // namespace s2
