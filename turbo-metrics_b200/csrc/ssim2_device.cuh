// ssim2_device.cuh -- device-side data structures and per-pixel math of the
// B200 SSIMULACRA2 engine.  Shared by the kernels in ssim2_kernels.cu.
//
// Arithmetic is written with explicit fmaf() and the translation unit is
// compiled with -fmad=false, so every rounding step is the one written here
// (the CPU restatement of the same arithmetic reproduces it).
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <stdint.h>

namespace s2 {

constexpr int kScales = 6;
constexpr int kTileW = 56;           // output columns per fused tile
constexpr int kCols = kTileW + 8;    // columns incl. the 4-px halo on each side
constexpr int kBand = 63;            // rows per shift band (tiles never straddle one; 7 x 9)
constexpr int kRowsPerBlk = 9;       // output rows per horizontal step (= window length)
constexpr int kSegs = 7;             // horizontal segments per row
constexpr int kSegW = 8;             // output pixels per segment (kSegs * kSegW == kTileW)
constexpr int kChunk = 4;            // pixels per f32 partial sum
constexpr int kPyrBlk = 32;          // scale-0 block edge of the pyramid kernel
constexpr float kC2 = 0.0009f;

enum Format { FMT_LINEAR_F32 = 0, FMT_SRGB8 = 1, FMT_NV12 = 2, FMT_RGB16 = 3 };
enum Storage { ST_F32 = 0, ST_F16 = 1, ST_BF16 = 2 };

// FIR taps of the exact form of the recursive Gaussian (sigma 1.5, N = 5),
// |k| = 0..4, rounded to f32.  The engine re-derives them in double at start
// (ssim2_engine.cpp) and refuses to run if they differ.
#define S2_T0 0x1.0ef8d6p-2f
#define S2_T1 0x1.b413e8p-3f
#define S2_T2 0x1.bfd672p-4f
#define S2_T3 0x1.2700c8p-5f
#define S2_T4 0x1.347d7p-7f

// One pair as the kernels see it.
struct DevPair {
    const void *in[2];       // scale-0 input: ref, dis (NV12: Y plane)
    const void *in_uv[2];    // NV12 CbCr planes
    long long pitch[2];      // bytes
    int fmt, bits;
    int w[kScales], h[kScales];
    int nscales;             // scored scales (>= 1)
    int lp[kScales];         // element pitch of the XYB planes of scale s
    void *lvl[2][kScales];   // planar XYB of scales 0..nscales-1 (3 planes each)
    int tile_base[kScales];  // first global tile of each scale
    int tile_cnt[kScales];
    int blk_base;            // first pyramid block
    int blk_x, blk_y;        // pyramid blocks of this pair
    int status;
};

// A run of tiles of one (pair, scale); tiles are numbered across segments.
struct Seg {
    int first_tile;
    int pair;
    int scale;
    int tiles_x;
    int strip_rows;
};

struct DevResult {
    double score;
    double stats[108];
    double sums[108];
    int n_scales;
    int status;
};

// ---------------------------------------------------------------------------
// colour math
// ---------------------------------------------------------------------------

// Opsin absorbance (crates/ssimulacra2-cuda-kernel/src/xyb.rs:3-36).
#define S2_M00 0.30f
#define S2_M02 0.078f
#define S2_M10 0.23f
#define S2_M12 0.078f
#define S2_M20 0.24342269f
#define S2_M21 0.20476745f
#define S2_B0 0.0037930734f
#define S2_B0_ROOT 0.1559542025327239180319220163705f

// Cube root of x >= 0 (0 for x <= 0 or NaN).  Newton iteration on the
// reciprocal cube root, r <- r + r (1 - x r^3) / 3, which needs no division,
// from the exponent-thirds bit-manipulation seed of W. Kahan ("Computing a
// real cube root", 1991); then y = x r^2 and one Newton correction of y.
// Only IEEE multiplies and fused multiply-adds, so every platform rounds the
// same way.  Two iterations from the ~3% seed leave ~1e-5, which the final
// correction squares away: <= 1 ulp over [1e-30, 1e30] (checked in the tests).
__device__ __forceinline__ float s2_cbrtf(float x) {
    if (!(x > 0.0f)) return 0.0f;
    float sc = 1.0f;
    if (x < 0x1p-100f) {
        x *= 0x1p102f;
        sc = 0x1p-34f;
    }
    float r = __uint_as_float(0x54a2fa8cu - __float_as_uint(x) / 3u);
    const float third = 0x1.555556p-2f;
#pragma unroll
    for (int k = 0; k < 2; k++) {
        float t = x * r;
        t = t * r;
        t = t * r;
        r = fmaf(r * third, 1.0f - t, r);
    }
    float y = x * r;
    y = y * r;
    const float e = fmaf(y * y, y, -x);
    const float c = (r * r) * third;
    y = fmaf(-e, c, y);
    return y * sc;
}

// p^(20/9) for p >= 0 (the BT.709 inverse OETF exponent 1/0.45 = 20/9),
// as p^2 * (p^(1/9))^2 with p^(1/9) = cbrt(cbrt(p)).  <= 5 ulp.
__device__ __forceinline__ float s2_pow_20_9(float p) {
    const float q = s2_cbrtf(s2_cbrtf(p));
    return (p * p) * (q * q);
}

__device__ __forceinline__ float opsin_row(int g, float r, float gg, float b) {
    const float m01 = 1.0f - S2_M02 - S2_M00;
    const float m11 = 1.0f - S2_M12 - S2_M10;
    const float m22 = 1.0f - S2_M20 - S2_M21;
    float v;
    if (g == 0)
        v = fmaf(S2_M00, r, fmaf(m01, gg, fmaf(S2_M02, b, S2_B0)));
    else if (g == 1)
        v = fmaf(S2_M10, r, fmaf(m11, gg, fmaf(S2_M12, b, S2_B0)));
    else
        v = fmaf(S2_M20, r, fmaf(S2_M21, gg, fmaf(m22, b, S2_B0)));
    return s2_cbrtf(fmaxf(v, 0.0f)) - S2_B0_ROOT;
}

// XYB channel g from the three opsin cube roots (xyb.rs:42-78).
__device__ __forceinline__ float xyb_from_opsin(int g, float rg, float gr, float bb) {
    float y = 0.5f * (rg + gr);
    if (g == 0) return fmaf(0.5f * (rg - gr), 14.0f, 0.42f);
    if (g == 1) return y + 0.01f;
    return (bb - y) + 0.55f;
}

// BT.709 inverse OETF (crates/cuda-colorspace-kernel/src/lib.rs:223-238).
__device__ __forceinline__ float bt709_eotf(float v) {
    const float beta = 0.018053968510807f;
    const float alpha = 1.0f + 5.5f * beta;
    const float thr = 0.08124285829863521110029445797874f;
    if (v >= thr) return s2_pow_20_9((v + (alpha - 1.0f)) / alpha);
    return v / 4.5f;
}

struct ColorConsts {
    // NV12 BT.709 limited range: y_coeff, r_coeff, b_coeff, g_coeff1, g_coeff2
    float nv12[5];
    // BT.2020 -> BT.709 linear matrix (row-major)
    float m2020[9];
};

template <typename T> __device__ __forceinline__ float ld_store(const T *p);
template <> __device__ __forceinline__ float ld_store<float>(const float *p) { return __ldg(p); }
template <> __device__ __forceinline__ float ld_store<__half>(const __half *p) { return __half2float(*p); }
template <> __device__ __forceinline__ float ld_store<__nv_bfloat16>(const __nv_bfloat16 *p) {
    return __bfloat162float(*p);
}
template <typename T> __device__ __forceinline__ T to_store(float v);
template <> __device__ __forceinline__ float to_store<float>(float v) { return v; }
template <> __device__ __forceinline__ __half to_store<__half>(float v) { return __float2half_rn(v); }
template <> __device__ __forceinline__ __nv_bfloat16 to_store<__nv_bfloat16>(float v) {
    return __float2bfloat16_rn(v);
}

// "Pre-linear" value of channel g of image img at scale-0 pixel (x, y): the
// final linear value for every format except RGB16, where it is the EOTF of
// channel g before the BT.2020 -> BT.709 matrix.  (x, y) must be inside.
__device__ __forceinline__ float pre_lin0(const DevPair &P, int img, int x, int y, int g,
                                          const float *lut, const ColorConsts &cc) {
    const char *base = (const char *)P.in[img] + (long long)y * P.pitch[img];
    switch (P.fmt) {
    case FMT_LINEAR_F32:
        return __ldg((const float *)base + 3 * x + g);
    case FMT_SRGB8:
        return lut[__ldg((const uint8_t *)base + 3 * x + g)];
    case FMT_NV12: {
        int Y = __ldg((const uint8_t *)base + x);
        const uint8_t *uv = (const uint8_t *)P.in_uv[img] + (long long)(y >> 1) * P.pitch[img] + 2 * (x >> 1);
        float cb = (float)((int)__ldg(uv) - 128);
        float cr = (float)((int)__ldg(uv + 1) - 128);
        float luma = (float)(max(Y, 16) - 16) * cc.nv12[0];
        float add;
        if (g == 0) add = cc.nv12[1] * cr;
        else if (g == 1) add = fmaf(cc.nv12[3], cb, cc.nv12[4] * cr);
        else add = cc.nv12[2] * cb;
        return fminf(fmaxf(bt709_eotf(luma + add), 0.0f), 1.0f);
    }
    default: { // FMT_RGB16
        float inv = 1.0f / (float)((1 << P.bits) - 1);
        return bt709_eotf((float)__ldg((const uint16_t *)base + 3 * x + g) * inv);
    }
    }
}

// Final linear channel g from the three pre-linear values.
__device__ __forceinline__ float fin_lin0(int fmt, int g, float p0, float p1, float p2,
                                          const ColorConsts &cc) {
    if (fmt != FMT_RGB16) return g == 0 ? p0 : (g == 1 ? p1 : p2);
    const float *m = cc.m2020 + 3 * g;
    float v = fmaf(m[0], p0, fmaf(m[1], p1, m[2] * p2));
    return fmaxf(v, 0.0f);
}

// Sum of the exact-form FIR taps over the valid positions around x in
// [0, n) (the blur's response to a constant 1 under zero padding), rounded
// to f32: exactly 1.0f in the interior, where all nine taps are inside.
// Prefix sums S[m] = t0 + ... + tm of the double-precision taps.
__device__ __forceinline__ float border_gain(int x, int n) {
    int lo = min(x, 4), hi = min(n - 1 - x, 4);
    if (lo == 4 && hi == 4) return 1.0f;
    const double S[5] = {0x1.0ef8d5c79cdafp-2, 0x1.e902c9b3e2946p-2, 0x1.2c7c332eb15f4p-1,
                         0x1.3eec3fae31770p-1, 0x1.43be3571e736ap-1};
    double s = S[lo] + S[hi];
    return (float)(s - S[0]);
}

}  // namespace s2
