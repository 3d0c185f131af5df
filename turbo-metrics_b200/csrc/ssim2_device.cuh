// ssim2_device.cuh -- device-side data structures and per-pixel math of the
// B200 SSIMULACRA2 engine.  Shared by the kernels in ssim2_kernels.cu.
//
// Arithmetic is written with explicit fmaf() and the translation unit is
// compiled with -fmad=false, so every rounding step is the one written here
// (the CPU restatement of the same arithmetic reproduces it).
#pragma once
#include <type_traits>

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <stdint.h>

namespace s2 {

constexpr int kScales = 6;
constexpr int kTileW = 120;          // output columns per fused tile (1920 = 16 tiles)
constexpr int kCols = kTileW + 8;    // columns incl. the 4-px halo on each side (one thread each)
constexpr int kBand = 64;            // rows per shift band (tiles never straddle one)
constexpr int kStep = 8;             // output rows per vertical / horizontal step
constexpr int kSegW = 8;             // output pixels per horizontal task (one f32 partial sum)
constexpr int kSegs = kTileW / kSegW;  // horizontal tasks per row (15)
constexpr int kStripMin = 16, kStripMid = 32, kStripMax = 64;  // tile heights (divide kBand)
constexpr int kPyrBlk = 64;          // scale-0 block edge of the prep kernel
constexpr float kC2 = 0.0009f;
constexpr int kDsLevels = 5;         // DSSIM scales (dssim-cuda/src/lib.rs:73)

enum Format { FMT_LINEAR_F32 = 0, FMT_SRGB8 = 1, FMT_NV12 = 2, FMT_RGB16 = 3, FMT_P016 = 4 };
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
    int prep_mask;           // images the prep pass converts: bit 0 reference, bit 1 distorted
    // 4:2:0 YUV (NV12 / P016): y_coeff, r_coeff, b_coeff, g_coeff1, g_coeff2
    // of the pair's matrix, range and depth, the luma minimum and the chroma
    // neutral value (cuda-colorspace-kernel/src/lib.rs:46-203)
    float yuv[5];
    int yuv_min, yuv_neutral;
    int lvl_ext;             // images whose XYB planes live outside the submission (bit per image)
    // DSSIM, the sibling metric sharing this pyramid: the prep pass also
    // converts levels 0..lab_levels-1 to dssim-core's scaled Lab (3 f32
    // planes per level, pitch lp[s]) and, when DSSIM's later levels are
    // clamped to 8 pixels, keeps the linear RGB of level lab_levels-1 in
    // `keep` (3 planes, pitch lp[s]) for the clamp pass.
    float *lab[2][kDsLevels];
    float *keep[2];
    int lab_levels;          // 0: no Lab output
    int prep_levels;         // levels the prep pass builds (XYB and Lab)
};

// One pair as the DSSIM kernels see it.  Level sizes follow dssim-cuda
// (halved rounding up, never below 8: dssim-cuda/src/lib.rs:184-205).
struct DsPair {
    float *lab[2][kDsLevels];    // 3 planes (L, a, b) per level, `pitch` floats per row
    float *map[kDsLevels];       // SSIM map per level, same pitch
    float *keep[2];              // clamp pass source: linear RGB of level clamp_from - 1
    float *scratch[2];           // clamp pass: two linear-RGB levels, 3 planes each
    long long splane;            // floats per plane of one scratch level
    int w[kDsLevels], h[kDsLevels], pitch[kDsLevels];
    int tile_base[kDsLevels], tile_cnt[kDsLevels];
    int kw, kh, kpitch;          // keep geometry
    int clamp_from;              // first level the clamp pass builds (kDsLevels: none)
    int prep_mask;
    int status;
};

// A run of DSSIM tiles (32 x 32 outputs) of one (pair, level).
struct DsSeg {
    int first_tile;
    int pair;
    int level;
    int tiles_x;
};

// A run of tiles of one (pair, scale); tiles are numbered across segments.
struct Seg {
    int first_tile;
    int pair;
    int scale;
    int tiles_x;
    int strip_rows;
};

// A run of S2_BLUR_IIR_REF work items of one (pair, scale): columns x planes
// for the vertical walk, rows x channels for the horizontal walk.
struct IirSeg {
    int first;     // first work item
    int pair;
    int scale;
    int rec_base;  // first row record of this (pair, scale) in the partial sums
    float *v;      // the 15 vertical-walk output planes of this (pair, scale)
};

struct DevResult {
    double score;
    double stats[108];
    double sums[108];
    int n_scales;
    int status;
    double dssim;                // DSSIM of the pair (NaN when not scored)
    double dssim_scale[kDsLevels];  // per-level 1 - mean |avg - ssim|
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
// Only IEEE multiplies and fused multiply-adds, and no branches, so every
// platform rounds the same way.  Two iterations from the ~3% seed leave
// ~1e-5, which the final correction squares away: <= 1 ulp over
// [1e-30, 1e30] (checked in the tests).
// i / 3 for i < 2^31 (the bits of a non-negative float) as one high multiply:
// 0x55555556 = (2^32 + 2) / 3, so the high word of i * 0x55555556 is
// floor(i / 3 + 2 i / (3 * 2^32)), and the added fraction is below 1/3.
__device__ __forceinline__ unsigned s2_div3(unsigned i) { return __umulhi(i, 0x55555556u); }

__device__ __forceinline__ float s2_cbrtf(float x) {
    const bool pos = x > 0.0f, tiny = x < 0x1p-100f;
    float xs = tiny ? x * 0x1p102f : x;
    xs = pos ? xs : 1.0f;
    float r = __uint_as_float(0x54a2fa8cu - s2_div3(__float_as_uint(xs)));
    const float third = 0x1.555556p-2f;
#pragma unroll
    for (int k = 0; k < 2; k++) {
        float t = xs * r;
        t = t * r;
        t = t * r;
        r = fmaf(r * third, 1.0f - t, r);
    }
    float y = xs * r;
    y = y * r;
    const float e = fmaf(y * y, y, -xs);
    const float c = (r * r) * third;
    y = fmaf(-e, c, y);
    y = y * (tiny ? 0x1p-34f : 1.0f);
    return pos ? y : 0.0f;
}

// ---- the XYB cube root --------------------------------------------------
// Correctly rounded in all but a few cases per 10^5 (<= 1 ulp always): a
// seed r ~ x^(-1/3) from the SFU, 2^(-log2(x) / 3) (lg2.approx / ex2.approx,
// about 4e-7 relative), y = x r^2, and one Newton step for y^3 = x whose
// residual y^3 - x is formed with y^2 split exactly into hi + lo (the
// FMA-based TwoProduct of Ogita, Rump and Oishi, "Accurate sum and dot
// product", 2005), so the step's error is second order in the seed's: the
// result then no longer depends on how the seed was found, and a CPU can
// check it against the correctly rounded cube root.  (s2_cbrtf above, with a
// plain residual, is within an ulp but its last bit follows its seed.)
__device__ __forceinline__ float s2_rcbrt_sfu(float x) {
    float l, r;
    asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(l) : "f"(x));
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(l * -0x1.555556p-2f));
    return r;
}

__device__ __forceinline__ float s2_cbrt_step(float x, float r) {
    float y = x * r;
    y = y * r;
    const float hi = y * y;
    const float lo = fmaf(y, y, -hi);  // y^2 = hi + lo exactly
    float e = fmaf(hi, y, -x);
    e = fmaf(lo, y, e);  // y^3 - x
    const float c = (r * r) * 0x1.555556p-2f;  // 1 / (3 y^2)
    return fmaf(-e, c, y);
}

// x in [2^-100, 2^100] (the opsin values of non-negative linear RGB, which
// are >= the bias 0.0038)
__device__ __forceinline__ float s2_cbrtf_unit(float x) { return s2_cbrt_step(x, s2_rcbrt_sfu(x)); }

// any x: 0 for x <= 0 or NaN; tiny x scaled by 2^102 and the root by 2^-34
__device__ __forceinline__ float s2_cbrtf_xyb(float x) {
    const bool pos = x > 0.0f, tiny = x < 0x1p-100f;
    float xs = tiny ? x * 0x1p102f : x;
    xs = pos ? xs : 1.0f;
    const float y = s2_cbrt_step(xs, s2_rcbrt_sfu(xs)) * (tiny ? 0x1p-34f : 1.0f);
    return pos ? y : 0.0f;
}

// dssim-core's scaled Lab of one linear-RGB pixel, with the reference GPU's
// f32 operations: fused multiply-adds where dssim-cuda-kernel/src/lab.rs:42-86
// uses mul_add, IEEE divisions, a cube root above the CIE threshold and the
// linear segment below it (lab.rs:37-44).  The cube root is s2_cbrtf (within
// an ulp, like the math library's the reference calls), whose IEEE-only
// operations the CPU restatement reproduces bit for bit: the SSIM map's
// variance terms amplify ulp-level differences of the Lab values.
__device__ __forceinline__ float ds_lab_f(float t) {
    return t > 216.0f / 24389.0f ? s2_cbrtf(t) : fmaf(24389.0f / (27.0f * 116.0f), t, 16.0f / 116.0f);
}

__device__ __forceinline__ void ds_lab(float r, float g, float b, float o[3]) {
    const float x = fmaf(0.4124f, r, fmaf(0.3576f, g, 0.1805f * b)) / 0.9505f;
    const float y = fmaf(0.2126f, r, fmaf(0.7152f, g, 0.0722f * b)) / 1.0f;
    const float z = fmaf(0.0193f, r, fmaf(0.1192f, g, 0.9505f * b)) / 1.089f;
    const float fx = ds_lab_f(x), fy = ds_lab_f(y), fz = ds_lab_f(z);
    o[0] = (fy - 16.0f / 116.0f) * 1.05f;
    o[1] = fmaf(fx - fy, 500.0f / 220.0f, 86.2f / 220.0f);
    o[2] = fmaf(fy - fz, 200.0f / 220.0f, 107.9f / 220.0f);
}

// a / b for b > 0 normal (the error-map denominators: >= 9e-4 and >= 1).
// The reciprocal comes from the SFU approximation (PTX rcp.approx.ftz.f32,
// at most 1 ulp from 1/b); the quotient q = a r then gets one residual
// correction q + (a - b q) r, the final step of Markstein's division
// (P. Markstein, "IA-64 and Elementary Functions", 2000): the residual
// a - b q is exact under FMA, so the corrected quotient is within
// 0.5 ulp + 2^-23 of the residual's weight -- the IEEE quotient except in
// rare near-halfway cases.  4 instructions instead of a division's
// multi-instruction sequence with its slow path.
__device__ __forceinline__ float s2_div(float a, float b) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(b));
    const float q = a * r;
    const float e = fmaf(-b, q, a);
    return fmaf(e, r, q);
}

// 2^(r/9), r = 0..8, rounded to f32
__device__ __forceinline__ float s2_pow2_r9(int r) {
    const float lo = r < 2 ? (r == 0 ? 0x1p+0f : 0x1.147eccp+0f) : (r == 2 ? 0x1.2aa1a6p+0f : 0x1.428a3p+0f);
    const float mid = r < 6 ? (r == 4 ? 0x1.5c5cbcp+0f : 0x1.784086p+0f) : (r == 6 ? 0x1.965feap+0f : 0x1.b6e8aep+0f);
    return r < 4 ? lo : (r < 8 ? mid : 0x1.da0c4p+0f);
}

// p^(20/9) for normal p > 0 (the BT.709 inverse OETF exponent 1/0.45 =
// 20/9), 0 for p <= 0.  With p = m 2^e, m in [1, 2): m^(20/9) is a degree-7
// polynomial in t = m - 1.5 (Chebyshev interpolation at 8 nodes, converted
// to monomials and rounded to f32; Horner with fmaf), times 2^(20e/9) =
// 2^(2e + k) 2^(r/9) with 2e = 9k + r, 0 <= r < 9.  Branch-free; <= 3.3 ulp
// on [0.1, 2].
__device__ __forceinline__ float s2_pow_20_9(float p) {
    const bool pos = p > 0.0f;
    const unsigned b = __float_as_uint(pos ? p : 1.0f);
    const int e = (int)((b >> 23) & 0xffu) - 127;
    const float t = __uint_as_float((b & 0x7fffffu) | 0x3f800000u) - 1.5f;
    float y = 0x1.1eb37ap-12f;
    y = fmaf(y, t, -0x1.88e318p-11f);
    y = fmaf(y, t, 0x1.2713a6p-9f);
    y = fmaf(y, t, -0x1.37717ep-7f);
    y = fmaf(y, t, 0x1.2c9724p-4f);
    y = fmaf(y, t, 0x1.7c6f02p+0f);
    y = fmaf(y, t, 0x1.d2e55cp+1f);
    y = fmaf(y, t, 0x1.3b279ep+1f);
    const int n = 2 * e;
    const int k = (n + 261) / 9 - 29;  // floor(n / 9) for n >= -261
    const int r = n - 9 * k;
    y = y * s2_pow2_r9(r);
    y = y * __uint_as_float((unsigned)(2 * e + k + 127) << 23);
    return pos ? y : 0.0f;
}

// s2_pow_20_9 for p in [1/8, 2): there the exponent e is -3..0 and the
// product of 2^(r/9) and 2^(2e + k) is one f32 constant 2^(20e/9) (a power
// of two times the rounded 2^(r/9), so multiplying by it rounds exactly as
// the two multiplications do): the same result from 4 selects instead of
// the exponent arithmetic.
__device__ __forceinline__ float s2_pow_20_9_unit(float p) {
    const unsigned b = __float_as_uint(p);
    const int e = (int)(b >> 23) - 127;
    const float t = __uint_as_float((b & 0x7fffffu) | 0x3f800000u) - 1.5f;
    float y = 0x1.1eb37ap-12f;
    y = fmaf(y, t, -0x1.88e318p-11f);
    y = fmaf(y, t, 0x1.2713a6p-9f);
    y = fmaf(y, t, -0x1.37717ep-7f);
    y = fmaf(y, t, 0x1.2c9724p-4f);
    y = fmaf(y, t, 0x1.7c6f02p+0f);
    y = fmaf(y, t, 0x1.d2e55cp+1f);
    y = fmaf(y, t, 0x1.3b279ep+1f);
    const float s = e == 0 ? 1.0f : (e == -1 ? 0x1.b6e8aep-3f : (e == -2 ? 0x1.784086p-5f : 0x1.428a3p-7f));
    return y * s;
}

// KUNIT: the argument is known >= 0.0038 (non-negative linear RGB).
template <bool KUNIT>
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
    if (KUNIT) return s2_cbrtf_unit(v) - S2_B0_ROOT;
    return s2_cbrtf_xyb(v) - S2_B0_ROOT;
}

// XYB channel g from the three opsin cube roots (xyb.rs:42-78).
__device__ __forceinline__ float xyb_from_opsin(int g, float rg, float gr, float bb) {
    float y = 0.5f * (rg + gr);
    if (g == 0) return fmaf(0.5f * (rg - gr), 14.0f, 0.42f);
    if (g == 1) return y + 0.01f;
    return (bb - y) + 0.55f;
}

// BT.709 inverse OETF (crates/cuda-colorspace-kernel/src/lib.rs:223-238):
// ((v + (alpha - 1)) / alpha)^(1/0.45) above the threshold, v / 4.5 below.
// The two divisions are multiplications by the f32 reciprocals 1/alpha and
// 2/9 (<= 1 ulp from dividing); both branches are evaluated and selected.
// The power's base is clamped to [1/8, 1.5]: the selected branch has
// base >= 0.164, and a base above 1.5 (v > 1.55, possible only for NV12,
// whose caller clamps the result to 1) gives a result above 1 either way.
__device__ __forceinline__ float bt709_eotf(float v) {
    const float alpha_m1 = 0x1.96b84p-4f;    // alpha - 1, alpha = 1 + 5.5 * 0.018053968510807
    const float inv_alpha = 0x1.d1c096p-1f;  // 1 / alpha in f32
    const float thr = 0.08124285829863521110029445797874f;
    const float hi = s2_pow_20_9_unit(fminf(fmaxf((v + alpha_m1) * inv_alpha, 0.125f), 1.5f));
    const float lo = v * 0x1.c71c72p-3f;     // v / 4.5
    return v >= thr ? hi : lo;
}

// ---- two pixels at once (sm_100 f32x2 operations; each lane rounds exactly
// as the scalar operation, so these return the scalar functions' results) --
__device__ __forceinline__ float2 s2_f2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 s2_neg2(float2 a) { return make_float2(-a.x, -a.y); }

// s2_cbrtf of two values at once (f32x2 where both lanes do the same
// operation; each lane rounds as the scalar steps).  The product that
// 1 - t subtracts is formed by two scalar multiplies: a packed product
// feeding a packed add would be fused into one rounding.
__device__ __forceinline__ float2 s2_cbrtf2(float2 x) {
    const bool p0 = x.x > 0.0f, p1 = x.y > 0.0f, t0 = x.x < 0x1p-100f, t1 = x.y < 0x1p-100f;
    float2 xs = make_float2(t0 ? x.x * 0x1p102f : x.x, t1 ? x.y * 0x1p102f : x.y);
    xs = make_float2(p0 ? xs.x : 1.0f, p1 ? xs.y : 1.0f);
    float2 r = make_float2(__uint_as_float(0x54a2fa8cu - s2_div3(__float_as_uint(xs.x))),
                           __uint_as_float(0x54a2fa8cu - s2_div3(__float_as_uint(xs.y))));
    const float2 third = s2_f2(0x1.555556p-2f);
#pragma unroll
    for (int k = 0; k < 2; k++) {
        float2 t = __fmul2_rn(xs, r);
        t = __fmul2_rn(t, r);
        t = make_float2(t.x * r.x, t.y * r.y);
        r = __ffma2_rn(__fmul2_rn(r, third), __fadd2_rn(s2_f2(1.0f), s2_neg2(t)), r);
    }
    float2 y = __fmul2_rn(xs, r);
    y = __fmul2_rn(y, r);
    const float2 e = __ffma2_rn(__fmul2_rn(y, y), y, s2_neg2(xs));
    const float2 c = __fmul2_rn(__fmul2_rn(r, r), third);
    y = __ffma2_rn(s2_neg2(e), c, y);
    y = __fmul2_rn(y, make_float2(t0 ? 0x1p-34f : 1.0f, t1 ? 0x1p-34f : 1.0f));
    return make_float2(p0 ? y.x : 0.0f, p1 ? y.y : 0.0f);
}

__device__ __forceinline__ float2 ds_lab_f2(float2 t) {
    const float thr = 216.0f / 24389.0f;
    const float2 c = s2_cbrtf2(t);
    const float2 l = __ffma2_rn(s2_f2(24389.0f / (27.0f * 116.0f)), t, s2_f2(16.0f / 116.0f));
    return make_float2(t.x > thr ? c.x : l.x, t.y > thr ? c.y : l.y);
}

// ds_lab of two pixels (lanes), each lane rounding as ds_lab: the products
// of the colour matrix feed the addends of FMAs, never a packed add.
__device__ __forceinline__ void ds_lab2(float2 r, float2 g, float2 b, float2 o[3]) {
    const float2 xn = __ffma2_rn(s2_f2(0.4124f), r, __ffma2_rn(s2_f2(0.3576f), g, __fmul2_rn(s2_f2(0.1805f), b)));
    const float2 y = __ffma2_rn(s2_f2(0.2126f), r, __ffma2_rn(s2_f2(0.7152f), g, __fmul2_rn(s2_f2(0.0722f), b)));
    const float2 zn = __ffma2_rn(s2_f2(0.0193f), r, __ffma2_rn(s2_f2(0.1192f), g, __fmul2_rn(s2_f2(0.9505f), b)));
    const float2 fx = ds_lab_f2(make_float2(xn.x / 0.9505f, xn.y / 0.9505f));
    const float2 fy = ds_lab_f2(y);
    const float2 fz = ds_lab_f2(make_float2(zn.x / 1.089f, zn.y / 1.089f));
    o[0] = __fmul2_rn(__fadd2_rn(fy, s2_f2(-(16.0f / 116.0f))), s2_f2(1.05f));
    o[1] = __ffma2_rn(__fadd2_rn(fx, s2_neg2(fy)), s2_f2(500.0f / 220.0f), s2_f2(86.2f / 220.0f));
    o[2] = __ffma2_rn(__fadd2_rn(fy, s2_neg2(fz)), s2_f2(200.0f / 220.0f), s2_f2(107.9f / 220.0f));
}


__device__ __forceinline__ float s2_pow_scale_unit(unsigned b) {
    const int e = (int)(b >> 23) - 127;
    return e == 0 ? 1.0f : (e == -1 ? 0x1.b6e8aep-3f : (e == -2 ? 0x1.784086p-5f : 0x1.428a3p-7f));
}

// Packed f32x2 arithmetic (__fmul2_rn, __fadd2_rn, __ffma2_rn): each lane
// rounds as the scalar operation, but the compiler contracts a packed
// multiply whose result feeds a packed add into one fused multiply-add (one
// rounding instead of two), even in a -fmad=false build (measured on sm_100a
// with CUDA 12.9).  So no packed product here feeds a packed sum: products
// that are summed are formed by scalar multiplies (never contracted under
// -fmad=false), or the sum is the addend of a packed FMA, or the product is
// exact (a multiplication by 0.5).
// The same operations as inline PTX (add / mul / fma .rn.f32x2).  Each lane
// rounds as the scalar operation -- but the assembler, too, was measured to
// fuse a packed multiply whose result feeds a packed add into one fused
// multiply-add (a probe over 1.7e7 operand triples on sm_100a, CUDA 12.9:
// every case where the two roundings differ from one came out fused).  So
// here as well no packed product feeds a packed sum: the fused tile pass
// feeds products to the multiplicand or addend of an explicit FMA, or sums
// the two lanes of a product with a scalar add.
__device__ __forceinline__ float2 s2_padd(float2 a, float2 b) {
    float2 d;
    asm("{.reg .b64 ra, rb, rd;\n\tmov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
        "add.rn.f32x2 rd, ra, rb;\n\tmov.b64 {%0, %1}, rd;}"
        : "=f"(d.x), "=f"(d.y) : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return d;
}
__device__ __forceinline__ float2 s2_pmul(float2 a, float2 b) {
    float2 d;
    asm("{.reg .b64 ra, rb, rd;\n\tmov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
        "mul.rn.f32x2 rd, ra, rb;\n\tmov.b64 {%0, %1}, rd;}"
        : "=f"(d.x), "=f"(d.y) : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return d;
}
__device__ __forceinline__ float2 s2_pfma(float2 a, float2 b, float2 c) {
    float2 d;
    asm("{.reg .b64 ra, rb, rc, rd;\n\tmov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
        "mov.b64 rc, {%6, %7};\n\tfma.rn.f32x2 rd, ra, rb, rc;\n\tmov.b64 {%0, %1}, rd;}"
        : "=f"(d.x), "=f"(d.y) : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y), "f"(c.x), "f"(c.y));
    return d;
}

__device__ __forceinline__ float2 s2_mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 s2_add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 s2_mul2s(float2 a, float2 b) { return make_float2(a.x * b.x, a.y * b.y); }

// The negated quotients -(a.x / b.x, a.y / b.y) by s2_div's steps on both
// lanes, with the reciprocals of -b: r' = -r, q' = a r' = -q, e = b q' + a =
// a - b q, e r' + q' = -(e r + q); each step rounds to the negation of the
// scalar step's result (round-to-nearest is symmetric, and so is the
// hardware reciprocal), so -n is s2_div of each lane.
__device__ __forceinline__ float2 s2_div2_neg(float2 a, float2 b) {
    float2 r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r.x) : "f"(-b.x));
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r.y) : "f"(-b.y));
    const float2 q = s2_pmul(a, r);
    const float2 e = s2_pfma(b, q, a);
    return s2_pfma(e, r, q);
}

// The factors 2^(20e/9) of s2_pow_20_9_unit for e = -3..0, indexed by the
// exponent field minus 124 (the caller keeps them in shared memory: one
// shared load per lane instead of three compares and selects).
#define S2_POW_TAB_INIT {0x1.428a3p-7f, 0x1.784086p-5f, 0x1.b6e8aep-3f, 0x1p+0f}

// s2_pow_20_9_unit of both lanes; pw = the S2_POW_TAB_INIT table
__device__ __forceinline__ float2 s2_pow_20_9_unit2(float2 p, const float *pw) {
    const unsigned bx = __float_as_uint(p.x), by = __float_as_uint(p.y);
    const float2 m = make_float2(__uint_as_float((bx & 0x7fffffu) | 0x3f800000u),
                                 __uint_as_float((by & 0x7fffffu) | 0x3f800000u));
    const float2 t = s2_add2(m, s2_f2(-1.5f));
    float2 y = __ffma2_rn(s2_f2(0x1.1eb37ap-12f), t, s2_f2(-0x1.88e318p-11f));
    y = __ffma2_rn(y, t, s2_f2(0x1.2713a6p-9f));
    y = __ffma2_rn(y, t, s2_f2(-0x1.37717ep-7f));
    y = __ffma2_rn(y, t, s2_f2(0x1.2c9724p-4f));
    y = __ffma2_rn(y, t, s2_f2(0x1.7c6f02p+0f));
    y = __ffma2_rn(y, t, s2_f2(0x1.d2e55cp+1f));
    y = __ffma2_rn(y, t, s2_f2(0x1.3b279ep+1f));
    return s2_mul2(y, make_float2(pw[(bx >> 23) - 124u], pw[(by >> 23) - 124u]));
}

// bt709_eotf of both lanes; pw = the S2_POW_TAB_INIT table
__device__ __forceinline__ float2 bt709_eotf2(float2 v, const float *pw) {
    const float thr = 0.08124285829863521110029445797874f;
    const float2 q = s2_mul2(s2_add2(v, s2_f2(0x1.96b84p-4f)), s2_f2(0x1.d1c096p-1f));
    const float2 hi =
        s2_pow_20_9_unit2(make_float2(fminf(fmaxf(q.x, 0.125f), 1.5f), fminf(fmaxf(q.y, 0.125f), 1.5f)), pw);
    const float2 lo = s2_mul2(v, s2_f2(0x1.c71c72p-3f));
    return make_float2(v.x >= thr ? hi.x : lo.x, v.y >= thr ? hi.y : lo.y);
}

// s2_cbrtf_unit of both lanes (each lane rounds as the scalar steps: no
// packed product feeds a packed sum)
__device__ __forceinline__ float2 s2_cbrtf_unit2(float2 x) {
    const float2 r = make_float2(s2_rcbrt_sfu(x.x), s2_rcbrt_sfu(x.y));
    float2 y = s2_mul2(x, r);
    y = s2_mul2(y, r);
    const float2 hi = s2_mul2(y, y);
    const float2 lo = __ffma2_rn(y, y, s2_neg2(hi));
    float2 e = __ffma2_rn(hi, y, s2_neg2(x));
    e = __ffma2_rn(lo, y, e);
    const float2 c = s2_mul2(s2_mul2(r, r), s2_f2(0x1.555556p-2f));
    return __ffma2_rn(s2_neg2(e), c, y);
}

// XYB of two pixels of non-negative linear RGB (opsin_row<true> and
// xyb_from_opsin per lane): out[c] = (pixel a, pixel b) of channel c.
__device__ __forceinline__ void xyb_pair_unit(float2 r, float2 g, float2 b, float2 out[3]) {
    const float m01 = 1.0f - S2_M02 - S2_M00;
    const float m11 = 1.0f - S2_M12 - S2_M10;
    const float m22 = 1.0f - S2_M20 - S2_M21;
    const float2 v0 = __ffma2_rn(s2_f2(S2_M00), r, __ffma2_rn(s2_f2(m01), g, __ffma2_rn(s2_f2(S2_M02), b, s2_f2(S2_B0))));
    const float2 v1 = __ffma2_rn(s2_f2(S2_M10), r, __ffma2_rn(s2_f2(m11), g, __ffma2_rn(s2_f2(S2_M12), b, s2_f2(S2_B0))));
    const float2 v2 = __ffma2_rn(s2_f2(S2_M20), r, __ffma2_rn(s2_f2(S2_M21), g, __ffma2_rn(s2_f2(m22), b, s2_f2(S2_B0))));
    const float2 nroot = s2_f2(-S2_B0_ROOT);
    const float2 rg = s2_add2(s2_cbrtf_unit2(v0), nroot);
    const float2 gr = s2_add2(s2_cbrtf_unit2(v1), nroot);
    const float2 bb = s2_add2(s2_cbrtf_unit2(v2), nroot);
    const float2 y = s2_mul2(s2_f2(0.5f), s2_add2(rg, gr));
    out[0] = __ffma2_rn(s2_mul2(s2_f2(0.5f), s2_add2(rg, s2_neg2(gr))), s2_f2(14.0f), s2_f2(0.42f));
    out[1] = s2_add2(y, s2_f2(0.01f));
    out[2] = s2_add2(s2_add2(bb, s2_neg2(y)), s2_f2(0.55f));
}

struct ColorConsts {
    // BT.2020 -> BT.709 linear matrix (row-major)
    float m2020[9];
};

__device__ __forceinline__ void rgb16_linear(unsigned r, unsigned g, unsigned b, float inv, const ColorConsts &cc,
                                             float o[3]) {
    const float p0 = bt709_eotf((float)r * inv);
    const float p1 = bt709_eotf((float)g * inv);
    const float p2 = bt709_eotf((float)b * inv);
#pragma unroll
    for (int k = 0; k < 3; k++) {
        const float *m = cc.m2020 + 3 * k;
        o[k] = fmaxf(fmaf(m[0], p0, fmaf(m[1], p1, m[2] * p2)), 0.0f);
    }
}

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

// RGB16: samples of `bits` bits, BT.709/BT.2020 inverse OETF, then BT.2020 ->
// BT.709 primaries, clamped >= 0.  inv = 1 / (2^bits - 1) in f32.
struct ColorConsts;
__device__ __forceinline__ void rgb16_linear(unsigned r, unsigned g, unsigned b, float inv, const ColorConsts &cc,
                                             float o[3]);

// Linear RGB of scale-0 pixel (x, y) of image img (inside the image), for
// input format FMT (the packed formats; 4:2:0 YUV goes by whole quads,
// yuv_load_quad / yuv_quad_linear).  sRGB8: the reference table; RGB16:
// BT.709/BT.2020 inverse OETF, then BT.2020 -> BT.709 primaries, clamped >= 0.
template <int FMT>
__device__ __forceinline__ void lin_pixel(const DevPair &P, int img, int x, int y, const float *lut,
                                          const ColorConsts &cc, float o[3]) {
    const char *base = (const char *)P.in[img] + (long long)y * P.pitch[img];
    if (FMT == FMT_LINEAR_F32) {
        const float *q = (const float *)base + 3 * x;
        o[0] = __ldg(q);
        o[1] = __ldg(q + 1);
        o[2] = __ldg(q + 2);
    } else if (FMT == FMT_SRGB8) {
        const uint8_t *q = (const uint8_t *)base + 3 * x;
        o[0] = lut[__ldg(q)];
        o[1] = lut[__ldg(q + 1)];
        o[2] = lut[__ldg(q + 2)];
    } else {
        const uint16_t *q = (const uint16_t *)base + 3 * x;
        rgb16_linear(__ldg(q), __ldg(q + 1), __ldg(q + 2), 1.0f / (float)((1 << P.bits) - 1), cc, o);
    }
}

// The six samples of a 4:2:0 quad (x, y even): luma of rows y and y + 1 and
// the shared CbCr pair, two samples per word (low half = left sample / Cb).
// ES = bytes per sample (1 NV12, 2 P016); read as one word per pair when the
// plane bases and the pitch are aligned to it (always for the engine's own
// staging), else sample by sample.
struct Nv12Quad {
    unsigned y0, y1, uv;
};
template <int ES>
__device__ __forceinline__ Nv12Quad yuv_load_quad(const DevPair &P, int img, int x, int y) {
    using W = typename std::conditional<ES == 1, unsigned short, unsigned>::type;
    using S = typename std::conditional<ES == 1, uint8_t, uint16_t>::type;
    const char *yp = (const char *)P.in[img] + (long long)y * P.pitch[img] + ES * x;
    const char *uv = (const char *)P.in_uv[img] + (long long)(y >> 1) * P.pitch[img] + ES * x;
    Nv12Quad q;
    if ((((unsigned long long)P.in[img] | (unsigned long long)P.in_uv[img] | (unsigned long long)P.pitch[img]) &
         (2 * ES - 1)) == 0) {
        q.y0 = __ldg((const W *)yp);
        q.y1 = __ldg((const W *)(yp + P.pitch[img]));
        q.uv = __ldg((const W *)uv);
    } else {
        const S *a = (const S *)yp, *b = (const S *)(yp + P.pitch[img]), *c = (const S *)uv;
        q.y0 = (unsigned)__ldg(a) | ((unsigned)__ldg(a + 1) << (8 * ES));
        q.y1 = (unsigned)__ldg(b) | ((unsigned)__ldg(b + 1) << (8 * ES));
        q.uv = (unsigned)__ldg(c) | ((unsigned)__ldg(c + 1) << (8 * ES));
    }
    return q;
}

// Limited / full range YUV of the pair's matrix (cuda-colorspace-kernel/src/
// biplanar.rs:8-70: nearest chroma, luma floored at the range minimum, BT.709
// inverse OETF, clamp to [0, 1]) of a loaded quad: pixels (0, 1) and (2, 3)
// as f32x2 lanes.
template <int ES>
__device__ __forceinline__ void yuv_quad_linear(const Nv12Quad &q, const DevPair &P, const float *pw, float o[4][3]) {
    constexpr unsigned kMask = ES == 1 ? 0xffu : 0xffffu;
    constexpr int kShift = 8 * ES;
    const float cb = (float)((int)(q.uv & kMask) - P.yuv_neutral);
    const float cr = (float)((int)(q.uv >> kShift) - P.yuv_neutral);
    const float ar = P.yuv[1] * cr;
    const float ag = fmaf(P.yuv[3], cb, P.yuv[4] * cr);
    const float ab = P.yuv[2] * cb;
    const int ymin = P.yuv_min;
    const float yc = P.yuv[0];
#pragma unroll
    for (int row = 0; row < 2; row++) {
        const unsigned w = row ? q.y1 : q.y0;
        const int Y0 = (int)(w & kMask), Y1 = (int)(w >> kShift);
        // scalar products: luma is summed with the chroma terms below
        const float2 luma = make_float2((float)(max(Y0, ymin) - ymin) * yc, (float)(max(Y1, ymin) - ymin) * yc);
        const float2 r = bt709_eotf2(s2_add2(luma, s2_f2(ar)), pw);
        const float2 g = bt709_eotf2(s2_add2(luma, s2_f2(ag)), pw);
        const float2 b = bt709_eotf2(s2_add2(luma, s2_f2(ab)), pw);
        float *p0 = o[2 * row], *p1 = o[2 * row + 1];
        p0[0] = fminf(fmaxf(r.x, 0.0f), 1.0f);
        p0[1] = fminf(fmaxf(g.x, 0.0f), 1.0f);
        p0[2] = fminf(fmaxf(b.x, 0.0f), 1.0f);
        p1[0] = fminf(fmaxf(r.y, 0.0f), 1.0f);
        p1[1] = fminf(fmaxf(g.y, 0.0f), 1.0f);
        p1[2] = fminf(fmaxf(b.y, 0.0f), 1.0f);
    }
}

// Linear RGB of the 2x2 quad whose top-left pixel is (x, y) (inside the
// image); px 0..3 = (x,y), (x+1,y), (x,y+1), (x+1,y+1); pixels outside the
// image (vx / vy false) are not read.  NV12 chroma is one sample per quad.
// lut: the sRGB8 table (256 entries) followed by the S2_POW_TAB_INIT table.
template <int FMT>
__device__ __forceinline__ void lin_quad(const DevPair &P, int img, int x, int y, bool vx, bool vy,
                                         const float *lut, const ColorConsts &cc, float o[4][3]) {
    if (FMT == FMT_NV12 || FMT == FMT_P016) {
        // 4:2:0 input has even width and height: the quad is complete
        constexpr int ES = FMT == FMT_NV12 ? 1 : 2;
        yuv_quad_linear<ES>(yuv_load_quad<ES>(P, img, x, y), P, lut + 256, o);
    } else {
        // a complete quad whose rows are aligned for the format's word size is
        // read as three words per row: sRGB8 16-bit, RGB16 32-bit, linear f32
        // 64-bit (x is even: the row pair starts 6, 12 or 24 bytes x/2 in)
        constexpr int kAlign = FMT == FMT_SRGB8 ? 2 : (FMT == FMT_RGB16 ? 4 : 8);
        if (vx && vy && ((((unsigned long long)P.in[img]) | (unsigned long long)P.pitch[img]) & (kAlign - 1)) == 0) {
            const float inv = FMT == FMT_RGB16 ? 1.0f / (float)((1 << P.bits) - 1) : 0.0f;
#pragma unroll
            for (int row = 0; row < 2; row++) {
                const char *rp = (const char *)P.in[img] + (long long)(y + row) * P.pitch[img];
                float *p0 = o[2 * row], *p1 = o[2 * row + 1];
                if (FMT == FMT_SRGB8) {
                    const unsigned short *q = (const unsigned short *)(rp + 3 * x);
                    const unsigned w0 = __ldg(q), w1 = __ldg(q + 1), w2 = __ldg(q + 2);
                    p0[0] = lut[w0 & 0xffu];
                    p0[1] = lut[w0 >> 8];
                    p0[2] = lut[w1 & 0xffu];
                    p1[0] = lut[w1 >> 8];
                    p1[1] = lut[w2 & 0xffu];
                    p1[2] = lut[w2 >> 8];
                } else if (FMT == FMT_RGB16) {
                    const unsigned *q = (const unsigned *)(rp + 6 * x);
                    const unsigned w0 = __ldg(q), w1 = __ldg(q + 1), w2 = __ldg(q + 2);
                    rgb16_linear(w0 & 0xffffu, w0 >> 16, w1 & 0xffffu, inv, cc, p0);
                    rgb16_linear(w1 >> 16, w2 & 0xffffu, w2 >> 16, inv, cc, p1);
                } else {
                    const float2 *q = (const float2 *)(rp + 12 * x);
                    const float2 a = __ldg(q), b = __ldg(q + 1), c = __ldg(q + 2);
                    p0[0] = a.x;
                    p0[1] = a.y;
                    p0[2] = b.x;
                    p1[0] = b.y;
                    p1[1] = c.x;
                    p1[2] = c.y;
                }
            }
        } else {
#pragma unroll
            for (int k = 0; k < 4; k++) {
                const bool in = (k & 1 ? vx : true) && (k & 2 ? vy : true);
                if (in) lin_pixel<FMT>(P, img, x + (k & 1), y + (k >> 1), lut, cc, o[k]);
            }
        }
    }
}

// Sum of the exact-form FIR taps over the valid positions around x in
// [0, n) (the blur's response to a constant 1 under zero padding), rounded
// to f32: exactly 1.0f in the interior, where all nine taps are inside.
// Prefix sums S[m] = t0 + ... + tm of the double-precision taps.
// (The prefix sums are picked by selects: an indexed local array would be
// built in local memory on every call.)
__device__ __forceinline__ double border_prefix(int k) {
    return k == 0 ? 0x1.0ef8d5c79cdafp-2
                  : (k == 1 ? 0x1.e902c9b3e2946p-2
                            : (k == 2 ? 0x1.2c7c332eb15f4p-1 : (k == 3 ? 0x1.3eec3fae31770p-1 : 0x1.43be3571e736ap-1)));
}
__device__ __forceinline__ float border_gain(int x, int n) {
    int lo = min(x, 4), hi = min(n - 1 - x, 4);
    if (lo == 4 && hi == 4) return 1.0f;
    double s = border_prefix(lo) + border_prefix(hi);
    return (float)(s - 0x1.0ef8d5c79cdafp-2);
}

}  // namespace s2
