// ssim2_kernels.cu -- sm_100a kernels of the B200 SSIMULACRA2 engine.
//
// One pair (or a batch of pairs of any sizes) is scored by three launches:
//
//   prep_kernel      reads each pair's scale-0 input once (any input format,
//                    converted to linear RGB on the fly), builds the 2x2 box
//                    pyramid in linear RGB and writes the XYB planes of all
//                    six scales (planar, f32/f16/bf16).
//                    (ssimulacra2-cuda-kernel/src/downscale.rs:4-35, srgb.rs,
//                    xyb.rs)
//   fused_kernel     persistent; each work item is one channel of a tile of
//                    120 columns x `strip_rows` rows at one scale of one pair.
//                    Walking down the tile 8 rows per step it forms the four
//                    blurred inputs on band-shifted values, runs the vertical
//                    9-tap FIR in registers, then the horizontal FIR, the
//                    SSIM / artifact / detail-loss maps and their L1/L4 sums
//                    from shared memory.  Only 6 pooled sums per item leave
//                    the SM.  (blur.rs, error_maps.rs, lib.rs:862-1016)
//   finalize_kernel  per pair: fixed-order f64 reduction of the tile sums,
//                    the 108 statistics and the score (lib.rs:1018-1192).
//
// The blur is the exact closed form of the reference's recursive Gaussian:
// the truncated-cosine recursion of blur.rs equals, in exact arithmetic, a
// symmetric 9-tap FIR with zero padding.  Moments are taken of values shifted
// by one reference XYB sample per (120-column tile, 64-row band), and the
// SSIM error is formed from the blurred difference of the two images, which
// removes the f32 cancellation in sigma - mu^2; the shift is undone
// algebraically (including at image borders, where the blur of a constant is
// not the constant).
#include "../../include/ssim2b200.h"
#include "ssim2_device.cuh"
#include "ssim2_launch.h"

namespace s2 {

// Shared memory of fused_kernel (one CTA = one channel of a tile): the step
// buffer, three float2 planes of kStep rows x kRS columns -- plane 0 and 1
// the vertical FIRs, plane 2 the raw (x', e) of the output rows -- then two
// stages of input rows (filled by bulk copies) and the threads' f64 sums.  A horizontal task reads 16-byte words of one row; the 8
// lanes of a load phase take the same segment of rows 0..7, whose starts are
// kRS * 8 = 1040 bytes apart: 65 16-byte groups, odd, so the 8 rows fall in
// distinct bank groups.
constexpr int kRS = kCols + 2;                        // float2 per row
constexpr int kPlaneF2 = kStep * kRS;                 // float2 per plane
constexpr int kBufF2 = 3 * kPlaneF2;                  // float2 per buffer
constexpr int kFusedThreads = kCols;                  // one vertical column each
constexpr int kTasks = kStep * kSegs;                 // horizontal tasks per step (120)
static_assert((kRS / 2) % 2 == 1, "odd 16-byte stride between rows");
static_assert(kTasks <= kFusedThreads, "one horizontal task per thread");
static_assert(kBand % kStripMax == 0 && kStripMax % kStep == 0 && kStripMid % kStep == 0 &&
                  kStripMin % kStep == 0, "tiles never straddle a band; whole steps");

// 9-tap symmetric FIR of two planes at once (f32x2 lanes; each lane rounds as
// acc = t4 (a0 + a8); acc = fma(t3, a1 + a7, acc); ...; fma(t0, a4, acc)).
// f32x2 operations take registers only, so the five tap pairs are the same
// five register pairs for every FIR of the pass.
__device__ __forceinline__ float2 fir9p(float2 a0, float2 a1, float2 a2, float2 a3, float2 a4, float2 a5,
                                        float2 a6, float2 a7, float2 a8) {
    float2 acc = s2_pmul(s2_f2(S2_T4), s2_padd(a0, a8));
    acc = s2_pfma(s2_f2(S2_T3), s2_padd(a1, a7), acc);
    acc = s2_pfma(s2_f2(S2_T2), s2_padd(a2, a6), acc);
    acc = s2_pfma(s2_f2(S2_T1), s2_padd(a3, a5), acc);
    return s2_pfma(s2_f2(S2_T0), a4, acc);
}

template <bool KUNIT>
__device__ __forceinline__ void xyb3(const float l[3], float o[3]) {
    const float a = opsin_row<KUNIT>(0, l[0], l[1], l[2]);
    const float b = opsin_row<KUNIT>(1, l[0], l[1], l[2]);
    const float c = opsin_row<KUNIT>(2, l[0], l[1], l[2]);
    o[0] = xyb_from_opsin(0, a, b, c);
    o[1] = xyb_from_opsin(1, a, b, c);
    o[2] = xyb_from_opsin(2, a, b, c);
}

__device__ __forceinline__ int find_seg(const Seg *segs, int nseg, int tile) {
    int lo = 0, hi = nseg - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (segs[mid].first_tile <= tile) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// ---------------------------------------------------------------------------
// prep: input -> linear -> XYB of every scale (2x2 box pyramid in linear RGB)
//
// Block = 64x64 scale-0 pixels of one pair, 256 threads, each thread a 2x2
// quad at a time: it converts the quad's four pixels, stores their XYB, and
// averages them (downscale.rs:4-35, source clamped at the far edge) into the
// scale-1 pixel, whose XYB it stores too and whose linear RGB goes to shared
// memory for scales 2..5.
// ---------------------------------------------------------------------------
// KUNIT: linear RGB known non-negative (every input format but linear f32).
template <typename ST, bool KUNIT>
__device__ __forceinline__ void store_xyb(const DevPair &P, int img, int s, int x, int y, const float lin[3]) {
    float o[3];
    xyb3<KUNIT>(lin, o);
    ST *dst = (ST *)P.lvl[img][s];
    const long long plane = (long long)P.lp[s] * P.h[s];
    const long long off = (long long)y * P.lp[s] + x;
#pragma unroll
    for (int c = 0; c < 3; c++) dst[c * plane + off] = to_store<ST>(o[c]);
}

// XYB of two horizontally adjacent pixels, stored as one 2-element write
// (x even: the planes' pitch is a multiple of 64 elements).
template <typename ST, bool KUNIT>
__device__ __forceinline__ void store_xyb_pair(ST *dst, long long plane, long long off, const float a[3],
                                               const float b[3]) {
    float2 o[3];
    if (KUNIT) {
        xyb_pair_unit(make_float2(a[0], b[0]), make_float2(a[1], b[1]), make_float2(a[2], b[2]), o);
    } else {
        float oa[3], ob[3];
        xyb3<KUNIT>(a, oa);
        xyb3<KUNIT>(b, ob);
#pragma unroll
        for (int c = 0; c < 3; c++) o[c] = make_float2(oa[c], ob[c]);
    }
#pragma unroll
    for (int c = 0; c < 3; c++) {
        if constexpr (sizeof(ST) == 4) {
            *(float2 *)(dst + c * plane + off) = o[c];
        } else {
            ST two[2] = {to_store<ST>(o[c].x), to_store<ST>(o[c].y)};
            *(unsigned *)(dst + c * plane + off) = *(const unsigned *)two;
        }
    }
}

constexpr int kLv1 = kPyrBlk / 2;  // scale-1 block edge (32)

// DSSIM outputs of one level's pixel: its Lab (levels below lab_levels) and,
// for the clamp pass, its linear RGB (level lab_levels - 1, when kept).
__device__ __forceinline__ void store_lab(const DevPair &P, int img, int s, int x, int y, const float lin[3]) {
    const long long plane = (long long)P.lp[s] * P.h[s];
    const long long off = (long long)y * P.lp[s] + x;
    if (s < P.lab_levels) {
        float o[3];
        ds_lab(lin[0], lin[1], lin[2], o);
        float *dst = P.lab[img][s];
#pragma unroll
        for (int c = 0; c < 3; c++) dst[c * plane + off] = o[c];
    }
    if (s == P.lab_levels - 1 && P.keep[img]) {
        float *dst = P.keep[img];
#pragma unroll
        for (int c = 0; c < 3; c++) dst[c * plane + off] = lin[c];
    }
}

// The same for pixels (x, y) and, when `two`, (x + 1, y) of one row, their
// Lab formed two at a time (ds_lab2, each lane as ds_lab).
__device__ __forceinline__ void store_lab_pair(const DevPair &P, int img, int s, int x, int y, const float a[3],
                                               const float b[3], bool two) {
    const long long plane = (long long)P.lp[s] * P.h[s];
    const long long off = (long long)y * P.lp[s] + x;
    if (s < P.lab_levels) {
        float2 o[3];
        ds_lab2(make_float2(a[0], two ? b[0] : a[0]), make_float2(a[1], two ? b[1] : a[1]),
                make_float2(a[2], two ? b[2] : a[2]), o);
        float *dst = P.lab[img][s];
#pragma unroll
        for (int c = 0; c < 3; c++) {
            dst[c * plane + off] = o[c].x;
            if (two) dst[c * plane + off + 1] = o[c].y;
        }
    }
    if (s == P.lab_levels - 1 && P.keep[img]) {
        float *dst = P.keep[img];
#pragma unroll
        for (int c = 0; c < 3; c++) {
            dst[c * plane + off] = a[c];
            if (two) dst[c * plane + off + 1] = b[c];
        }
    }
}

// OUT: bit 0 SSIMULACRA2's XYB planes, bit 1 DSSIM's Lab planes (both from
// the same linear pyramid).  OUT == 1 is the SSIMULACRA2-only pass.
//
// A thread takes two horizontally adjacent 2x2 quads at a time (4 x 2
// scale-0 pixels): the scale-0 XYB goes out as pixel pairs, and the two
// quads' scale-1 pixels form one pair for the f32x2 XYB conversion too.
template <int FMT, typename ST, int OUT>
__device__ __forceinline__ void prep_quads(const DevPair &P, int X0, int Y0, const float *lut, const ColorConsts &cc,
                                           float (*lv1)[3][kLv1 * kLv1]) {
    constexpr bool KU = FMT != FMT_LINEAR_F32;
    constexpr bool kX = (OUT & 1) != 0, kL = (OUT & 2) != 0;
    constexpr bool kYuv = FMT == FMT_NV12 || FMT == FMT_P016;
    constexpr int kEs = FMT == FMT_P016 ? 2 : 1;
    const int W = P.w[0], H = P.h[0];
    const bool scale1 = (kL ? P.prep_levels : P.nscales) > 1;
    for (int qq = threadIdx.x; qq < kLv1 * kLv1 / 2; qq += blockDim.x) {
        const int qx = 2 * (qq % (kLv1 / 2)), qy = qq / (kLv1 / 2);  // first quad of the two
        const int x = X0 + 2 * qx, y = Y0 + 2 * qy;
        if (x >= W || y >= H) continue;
        const bool two = x + 2 < W;  // the second quad starts inside the image
        const bool vy = y + 1 < H;
        // 4:2:0 YUV: both images' samples are loaded before either is converted
        Nv12Quad nr0{}, nr1{}, nd0{}, nd1{};  // [reference, distorted][quad]
        if (kYuv) {
            if (P.prep_mask & 1) {
                nr0 = yuv_load_quad<kEs>(P, 0, x, y);
                if (two) nr1 = yuv_load_quad<kEs>(P, 0, x + 2, y);
            }
            if (P.prep_mask & 2) {
                nd0 = yuv_load_quad<kEs>(P, 1, x, y);
                if (two) nd1 = yuv_load_quad<kEs>(P, 1, x + 2, y);
            }
        }
#pragma unroll 1
        for (int img = 0; img < 2; img++) {
            if (!((P.prep_mask >> img) & 1)) continue;
            float l1[2][3];
#pragma unroll
            for (int k = 0; k < 2; k++) {
                if (k == 1 && !two) break;
                const int xq = x + 2 * k;
                const bool vx = xq + 1 < W;
                float v[4][3];
                if (kYuv) yuv_quad_linear<kEs>(img ? (k ? nd1 : nd0) : (k ? nr1 : nr0), P, lut + 256, v);
                else lin_quad<FMT>(P, img, xq, y, vx, vy, lut, cc, v);
                if (kX && (!kL || P.nscales > 0)) {
                    ST *dst = (ST *)P.lvl[img][0];
                    const long long plane = (long long)P.lp[0] * H;
                    const long long off = (long long)y * P.lp[0] + xq;
                    if (vx) store_xyb_pair<ST, KU>(dst, plane, off, v[0], v[1]);
                    else store_xyb<ST, KU>(P, img, 0, xq, y, v[0]);
                    if (vy) {
                        if (vx) store_xyb_pair<ST, KU>(dst, plane, off + P.lp[0], v[2], v[3]);
                        else store_xyb<ST, KU>(P, img, 0, xq, y + 1, v[2]);
                    }
                }
                if (kL) {
                    store_lab_pair(P, img, 0, xq, y, v[0], v[1], vx);
                    if (vy) store_lab_pair(P, img, 0, xq, y + 1, v[2], v[3], vx);
                }
                // scale-1 pixel: 2x2 mean, far-edge clamp (a missing column
                // repeats the left pixel, a missing row the upper one)
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    const float a = v[0][c];
                    const float b = vx ? v[1][c] : a;
                    const float cc2 = vy ? v[2][c] : a;
                    const float d = vy ? (vx ? v[3][c] : cc2) : b;
                    float sum = a + b;
                    sum = sum + cc2;
                    sum = sum + d;
                    l1[k][c] = sum * 0.25f;
                }
            }
            if (!scale1) continue;
            const int x1 = (X0 >> 1) + qx, y1 = (Y0 >> 1) + qy;
#pragma unroll
            for (int c = 0; c < 3; c++) {
                lv1[img][c][qy * kLv1 + qx] = l1[0][c];
                if (two) lv1[img][c][qy * kLv1 + qx + 1] = l1[1][c];
            }
            if (kX && (!kL || P.nscales > 1)) {
                // x1 is even and the planes' pitch a multiple of 64 elements
                if (two) store_xyb_pair<ST, KU>((ST *)P.lvl[img][1], (long long)P.lp[1] * P.h[1],
                                                (long long)y1 * P.lp[1] + x1, l1[0], l1[1]);
                else store_xyb<ST, KU>(P, img, 1, x1, y1, l1[0]);
            }
            if (kL) store_lab_pair(P, img, 1, x1, y1, l1[0], l1[1], two);
        }
    }
}

// 128 threads: 4 blocks per SM (registers), whose barrier waits over the
// small scales overlap the other blocks' work.
constexpr int kPrepThreads = 128;

// FMT: the input format of every pair of the launch, or -1 for a mix (each
// block then switches on its pair's format).  A kernel compiled for one
// format carries one conversion instead of five, which the instruction
// cache notices.
template <typename ST, int OUT, int FMT>
__global__ void __launch_bounds__(kPrepThreads, 4) prep_kernel(const DevPair *__restrict__ pairs, int npairs,
                                                   const int *__restrict__ blk_first, int first_block,
                                                   int end_block,
                                                   ColorConsts cc, const float *__restrict__ lut_g) {
    __shared__ float lv1[2][3][kLv1 * kLv1];              // scale-1 linear block [img][ch][px]
    __shared__ float pp[2][2][3][(kLv1 / 2) * (kLv1 / 2)];  // scales >= 2, ping-pong
    __shared__ float lut[256 + 4];  // the sRGB8 table, then the BT.709 power's 2^(20e/9) factors
    // the block's pair descriptor: in shared memory, so the level stores
    // (global) cannot alias it and its fields need no per-thread copy
    __shared__ DevPair sP;
    static_assert(sizeof(DevPair) % 8 == 0, "DevPair copied as 8-byte words");
    for (int i = threadIdx.x; i < 256; i += blockDim.x) lut[i] = lut_g[i];
    if (threadIdx.x < 4) {
        const float pw[4] = S2_POW_TAB_INIT;
        lut[256 + threadIdx.x] = pw[threadIdx.x];
    }
    for (int item = first_block + blockIdx.x; item < end_block; item += gridDim.x) {
        int lo = 0, hi = npairs - 1;
        while (lo < hi) {
            int mid = (lo + hi + 1) >> 1;
            if (blk_first[mid] <= item) lo = mid;
            else hi = mid - 1;
        }
        __syncthreads();  // the previous item's readers of sP are done
        for (int i = threadIdx.x; i < (int)(sizeof(DevPair) / 8); i += blockDim.x)
            ((long long *)&sP)[i] = __ldg((const long long *)(pairs + lo) + i);
        __syncthreads();
        const DevPair &P = sP;
        const int b = item - blk_first[lo];
        const int bx = b % P.blk_x, by = b / P.blk_x;
        const int X0 = bx * kPyrBlk, Y0 = by * kPyrBlk;
        if constexpr (FMT >= 0) {
            prep_quads<(FMT >= 0 ? FMT : 0), ST, OUT>(P, X0, Y0, lut, cc, lv1);
        } else {
            switch (P.fmt) {
            case FMT_LINEAR_F32: prep_quads<FMT_LINEAR_F32, ST, OUT>(P, X0, Y0, lut, cc, lv1); break;
            case FMT_SRGB8: prep_quads<FMT_SRGB8, ST, OUT>(P, X0, Y0, lut, cc, lv1); break;
            case FMT_NV12: prep_quads<FMT_NV12, ST, OUT>(P, X0, Y0, lut, cc, lv1); break;
            case FMT_P016: prep_quads<FMT_P016, ST, OUT>(P, X0, Y0, lut, cc, lv1); break;
            default: prep_quads<FMT_RGB16, ST, OUT>(P, X0, Y0, lut, cc, lv1); break;
            }
        }
        __syncthreads();
        const int nlev = (OUT & 2) ? P.prep_levels : P.nscales;
        for (int s = 2; s < nlev; s++) {
            const int bs = kPyrBlk >> s, pbs = kPyrBlk >> (s - 1);
            const int ox0 = X0 >> s, oy0 = Y0 >> s;
            const int px0 = X0 >> (s - 1), py0 = Y0 >> (s - 1);
            const int wp = P.w[s - 1], hp = P.h[s - 1];
            for (int i = threadIdx.x; i < bs * bs; i += blockDim.x) {
                const int ox = ox0 + i % bs, oy = oy0 + i / bs;
                if (ox >= P.w[s] || oy >= P.h[s]) continue;
                // downscale.rs:4-35: source index clamped to the previous level
                const int xa = 2 * ox, xb = min(2 * ox + 1, wp - 1);
                const int ya = 2 * oy, yb = min(2 * oy + 1, hp - 1);
                const int ia = (ya - py0) * pbs, ib = (yb - py0) * pbs;
                const int ja = xa - px0, jb = xb - px0;
                for (int img = 0; img < 2; img++) {
                    if (!((P.prep_mask >> img) & 1)) continue;
                    float v[3];
                    for (int c = 0; c < 3; c++) {
                        const float *src = s == 2 ? lv1[img][c] : pp[(s - 1) & 1][img][c];
                        float sum = src[ia + ja] + src[ia + jb];
                        sum = sum + src[ib + ja];
                        sum = sum + src[ib + jb];
                        v[c] = sum * 0.25f;
                        pp[s & 1][img][c][i] = v[c];
                    }
                    if ((OUT & 1) && (!(OUT & 2) || s < P.nscales)) {
                        if (P.fmt == FMT_LINEAR_F32) store_xyb<ST, false>(P, img, s, ox, oy, v);
                        else store_xyb<ST, true>(P, img, s, ox, oy, v);
                    }
                    if (OUT & 2) store_lab(P, img, s, ox, oy, v);
                }
            }
            __syncthreads();
        }
    }
}

// ---------------------------------------------------------------------------
// fused per-scale tile pass
// ---------------------------------------------------------------------------
//
// Work item = one channel of a tile of kTileW (120) output columns x
// `strip_rows` rows at one scale of one pair: item = 3 * tile + channel.  A
// tile's three items write its 18 partial sums, channel-major.  128 threads
// walk down the tile in steps of kStep (8) rows; each step has two phases.
//
//   vertical    thread c owns input column x0 - 4 + c (the tile's columns and
//               a 4-column halo on each side).  The step's 8 input rows of
//               both images are already in shared memory: the bulk-copy
//               engine (cp.async.bulk, completion on an mbarrier) brought
//               them in two steps ahead.  The thread keeps the shifted inputs
//               of its column in register rings of 16 rows, where x' = ref -
//               anchor and y' = dis - anchor, and for each output row of the
//               step forms their 9-tap vertical FIRs.  The step's 8 new input
//               rows go to ring slots 8..15 on even steps and 0..7 on odd
//               steps, so every ring index is a compile-time constant.
//               Pixels outside the image read the anchor itself, which shifts
//               to exactly 0: zero padding of the shifted values, undone at
//               the borders by border_gain.
//   horizontal  thread t takes row t % 8 of the step and the 8-pixel segment
//               t / 8 (120 tasks): the horizontal FIRs give the blurred
//               moments, then the SSIM error, artifact and detail-loss maps
//               and their sums and fourth-power sums, in f32 over the
//               segment, then in f64 per thread (kept in shared memory).
//
// What is blurred: with x' = ref - anchor, y' = dis - anchor and the
// difference e = ref - dis, the four planes x', e, e^2 and x'y'.  Then
// mu1 = blur(x'), md = blur(e) = mu1 - mu2, and the SSIM error
//   d = 1 - num_m num_s / den = (Vd + md^2 num_s) / (Vd + num_s),
//   Vd = blur(e^2) - md^2 = var1 + var2 - 2 cov,  num_s = 2 cov + C2,
// is formed from the blurred difference itself: for near-identical images
// no small quantity is recovered from the difference of two large moments,
// which f32 cannot do to the metric's precision.
//
// The four planes are blurred as two f32x2 pairs: ring A = (x', e) and
// ring B = (e^2, x'y').  A barrier follows each phase (one step buffer: a
// second one would not leave room for four blocks per SM).
//
// EXPORT (error-map export, one scale of one pair): every pixel's SSIM error,
// artifact and detail-loss values are also stored to `maps`, 9 planes
// [channel][map] of `mpitch` floats per row and `mplane` floats per plane.
struct MapOut {
    float *maps;
    long long mpitch, mplane;
};

// Register rings of one vertical column.
struct Rings {
    float2 a[16];  // (x', e)
    float2 b[16];  // (e^2, x'y')
};

// Shift one input row into ring slot `sl` (vr, vd: the reference and
// distorted samples; cg: the anchor).  Outside the image both are the anchor,
// so every plane is 0 there.
__device__ __forceinline__ void ring_in(Rings &R, int sl, float vr, float vd, float cg) {
    const float xp = vr - cg;
    const float e = vr - vd;
    const float xy = __fmul_rn(xp, vd - cg);  // products rounded on their own
    const float ee = __fmul_rn(e, e);
    R.a[sl] = make_float2(xp, e);
    R.b[sl] = make_float2(ee, xy);
}

// ---- input rows through the bulk-copy engine -------------------------------
// A stage holds 8 input rows of the tile's 128 columns of both images
// ([image][row][column] floats, 8 KB).  Each row of each image is one
// cp.async.bulk copy (global -> shared, completion counted in bytes on the
// stage's mbarrier): the columns [x0 - 4, x0 + 124) clipped to [0, pitch), so
// every copy starts 16-byte aligned (x0 is a multiple of 120, the pitch of 64
// elements, the planes 256-byte aligned) and never leaves its row.  Rows and
// columns outside the image are not copied; their stage words are stale and
// the vertical phase replaces them by the anchor.
constexpr int kStageFloats = 2 * kStep * kCols;  // 8 KB
constexpr int kStages = 2;

__device__ __forceinline__ unsigned s2_smem_addr(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

// a stage barrier: one arrival (with its byte count) per warp a phase
__device__ __forceinline__ void s2_mbar_init(uint64_t *bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 4;" ::"r"(s2_smem_addr(bar)) : "memory");
}

__device__ __forceinline__ void s2_mbar_expect(uint64_t *bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(s2_smem_addr(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void s2_bulk_g2s(void *dst, const void *src, unsigned bytes, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            s2_smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(s2_smem_addr(bar))
        : "memory");
}

// The tile pass's wait bound in SM cycles, set by each block from its
// TileCheck (in shared memory so that the spin loops hold no register for it).
__shared__ long long s2_wait_limit;

// Wait for the stage's phase `parity`, at most s2_wait_limit SM clock
// cycles; on time-out set *err and return false.
__device__ __forceinline__ bool s2_mbar_wait(uint64_t *bar, unsigned parity, int *err) {
    const unsigned a = s2_smem_addr(bar);
    const long long t0 = clock64();
    for (;;) {
        unsigned done;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, "
            "p;\n\t}"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
        if (clock64() - t0 > s2_wait_limit) {
            atomicExch(err, 1);
            return false;
        }
    }
}

// The 8 rows of a stage for this thread's column.  inner: every column of
// the tile and all 8 rows are inside the image; otherwise rows and columns
// outside read the anchor (rows beyond the tile's nr output rows are not
// used).
struct StepRows {
    float r[kStep], d[kStep];
};

__device__ __forceinline__ void v_load(StepRows &in, const float *stage, int col, bool colin, int ybase, int H,
                                       bool inner, float cg) {
    if (inner) {  // no masks: a branch of its own, so the selects are not executed
#pragma unroll
        for (int k = 0; k < kStep; k++) {
            in.r[k] = stage[k * kCols + col];
            in.d[k] = stage[(kStep + k) * kCols + col];
        }
        return;
    }
#pragma unroll
    for (int k = 0; k < kStep; k++) {
        const float vr = stage[k * kCols + col], vd = stage[(kStep + k) * kCols + col];
        const bool ok = colin && ybase + k >= 0 && ybase + k < H;
        in.r[k] = ok ? vr : cg;
        in.d[k] = ok ? vd : cg;
    }
}

// One vertical step: the step's input rows enter ring slots S0 + 8 ..
// S0 + 15 (mod 16); output row k reads slots S0 + k .. S0 + k + 8 and is
// stored to row k of the buffer: plane 0 the FIR of ring a, plane 1 that of
// ring b, plane 2 the raw (x', e) of the output row.  All 8 rows are formed
// even in an item's last, partial step (nr < 8, which happens only at the
// image's bottom edge): its rows beyond nr lie below the image, read the
// anchor (0 after the shift) and are neither read by the horizontal phase
// nor used by a later step.
template <int S0>
__device__ __forceinline__ void v_step(Rings &R, const StepRows &in, float cg, float2 *__restrict__ buf, int col) {
#pragma unroll
    for (int k = 0; k < kStep; k++) {
        ring_in(R, (S0 + 8 + k) & 15, in.r[k], in.d[k], cg);
#define S2_R(a, j) a[(S0 + k + (j)) & 15]
        buf[k * kRS + col] = fir9p(S2_R(R.a, 0), S2_R(R.a, 1), S2_R(R.a, 2), S2_R(R.a, 3), S2_R(R.a, 4),
                                   S2_R(R.a, 5), S2_R(R.a, 6), S2_R(R.a, 7), S2_R(R.a, 8));
        buf[kPlaneF2 + k * kRS + col] = fir9p(S2_R(R.b, 0), S2_R(R.b, 1), S2_R(R.b, 2), S2_R(R.b, 3),
                                              S2_R(R.b, 4), S2_R(R.b, 5), S2_R(R.b, 6), S2_R(R.b, 7),
                                              S2_R(R.b, 8));
        buf[2 * kPlaneF2 + k * kRS + col] = S2_R(R.a, 4);  // raw (x', e)
#undef S2_R
    }
}

// Horizontal FIR of 4 outputs from 12 float2 of a buffer row (16-byte loads).
__device__ __forceinline__ void h_fir4(const float2 *__restrict__ p, float2 o[4]) {
    float2 v[12];
    const float4 *q = (const float4 *)p;
#pragma unroll
    for (int j = 0; j < 6; j++) {
        const float4 t = q[j];
        v[2 * j] = make_float2(t.x, t.y);
        v[2 * j + 1] = make_float2(t.z, t.w);
    }
#pragma unroll
    for (int j = 0; j < 4; j++)
        o[j] = fir9p(v[j], v[j + 1], v[j + 2], v[j + 3], v[j + 4], v[j + 5], v[j + 6], v[j + 7], v[j + 8]);
}

// Sums of one task's maps: (d, art, det) and their 4th powers, f32.
struct TaskSums {
    float fs_d, f4_d;
    float2 fs_ad, f4_ad;  // (artifact, detail loss)
};

__device__ __forceinline__ void add_maps(TaskSums &t, float d, float art, float det) {
    t.fs_d += d;
    const float q = d * d;
    t.f4_d = fmaf(q, q, t.f4_d);
    const float2 ad = make_float2(art, det);
    t.fs_ad = s2_padd(t.fs_ad, ad);
    const float2 q2 = s2_pmul(ad, ad);
    t.f4_ad = s2_pfma(q2, q2, t.f4_ad);
}

// Error maps of one pixel.  m = (mu1, md) and s = (blur(e^2), blur(x'y')),
// r = the raw (x', e) of the pixel.  kk = anchor * (1 - border gain): the
// correction of the shifted moments at the image borders (0 inside).  With
// the anchor c and the gain g the true means are mu = m + c g and
// sigma12 - mu1 mu2 = cov + kk h, cov = blur(x'y') - mu1 mu2,
// h = (mu1 + mu2) + ce, ce = c - kk = c g; md, blur(e) and blur(e^2) need
// no correction (e is the same with and without the shift).  For identical
// images e = 0, so Vd, md and the SSIM error are exactly 0.
template <bool BORDER>
__device__ __forceinline__ void maps_px(float2 m, float2 s, float2 r, float kk, float ce, float &d, float &art,
                                        float &det) {
    const float m1 = m.x, md = m.y;
    const float m2 = m1 - md;
    float cov = fmaf(-m1, m2, s.y);
    if (BORDER) cov = fmaf(kk, (m1 + m2) + ce, cov);
    const float num_s = fmaf(2.0f, cov, kC2);
    const float vd = fmaf(-md, md, s.x);
    const float den = vd + num_s;
    const float nn = fmaf(md * md, num_s, vd);
    const float2 t = s2_pfma(m, s2_f2(-1.0f), r);  // (x' - mu1, e - md)
    float t1 = t.x, t2 = t.x - t.y;              // x' - mu1, y' - mu2
    if (BORDER) {
        t1 = t1 + kk;
        t2 = t2 + kk;
    }
    const float aa = fabsf(t1), bb = fabsf(t2);
    if (BORDER) {
        d = fmaxf(s2_div(nn, den), 0.0f);
        const float d1 = s2_div(bb - aa, 1.0f + aa);
        art = fmaxf(d1, 0.0f);
        det = fmaxf(-d1, 0.0f);
    } else {
        // both quotients at once: n = -(nn / den, (bb - aa) / (1 + aa))
        const float2 n = s2_div2_neg(make_float2(nn, bb - aa), make_float2(den, 1.0f + aa));
        d = fmaxf(-n.x, 0.0f);
        art = fmaxf(-n.y, 0.0f);
        det = fmaxf(n.y, 0.0f);
    }
}


// What a horizontal task needs of its work item.
struct ItemGeo {
    int x0, y0, W, H, g;
    float cg;
    int lp;  // row pitch of the planes (elements)
};


__device__ __forceinline__ void add_task(double *a, const TaskSums &ts) {
    a[0] += (double)ts.fs_d;
    a[kFusedThreads] += (double)ts.fs_ad.x;
    a[2 * kFusedThreads] += (double)ts.fs_ad.y;
    a[3 * kFusedThreads] += (double)ts.f4_d;
    a[4 * kFusedThreads] += (double)ts.f4_ad.x;
    a[5 * kFusedThreads] += (double)ts.f4_ad.y;
}

// Horizontal phase of one step (output rows r0 .. r0 + nr - 1 of the tile):
// this thread's task, row t_r, segment t_s; its sums are added to acc.
template <bool EXPORT, typename ACC>
__device__ __forceinline__ void h_step(const float2 *__restrict__ buf, int r0, int nr, int t_r, int t_s, bool t_on,
                                       const ItemGeo &G, ACC &&acc, const MapOut &mo) {
    if (!t_on || t_r >= nr) return;
    const int c0 = t_s * kSegW;  // first output column of the task (tile coordinates)
    const int xc = G.x0 + c0;
    if (xc >= G.W) return;
    const int y = G.y0 + r0 + t_r;
    const float bv = border_gain(y, G.H);
    const bool interior = bv == 1.0f && xc >= 4 && xc + kSegW + 4 <= G.W;
    TaskSums ts{0.0f, 0.0f, make_float2(0.0f, 0.0f), make_float2(0.0f, 0.0f)};
#pragma unroll 1
    for (int half = 0; half < kSegW / 4; half++) {
        const int cc = c0 + 4 * half;
        const float2 *pa = buf + t_r * kRS + cc;
        float2 mA[4], mB[4], rw[4];
        h_fir4(pa, mA);             // (mu1, md)
        h_fir4(pa + kPlaneF2, mB);  // (blur(e^2), blur(x'y'))
        {
            const float4 *q = (const float4 *)(pa + 2 * kPlaneF2 + 4);
            const float4 t0 = q[0], t1 = q[1];
            rw[0] = make_float2(t0.x, t0.y);
            rw[1] = make_float2(t0.z, t0.w);
            rw[2] = make_float2(t1.x, t1.y);
            rw[3] = make_float2(t1.z, t1.w);
        }
        if (interior) {
#pragma unroll
            for (int j = 0; j < 4; j++) {
                float d, art, det;
                maps_px<false>(mA[j], mB[j], rw[j], 0.0f, 0.0f, d, art, det);
                if (EXPORT) {
                    float *m = mo.maps + (long long)(3 * G.g) * mo.mplane + (long long)y * mo.mpitch + G.x0 + cc + j;
                    m[0] = d;
                    m[mo.mplane] = art;
                    m[2 * mo.mplane] = det;
                }
                add_maps(ts, d, art, det);
            }
        } else {
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const int xx = G.x0 + cc + j;
                if (xx < G.W) {
                    const float bh = border_gain(xx, G.W);
                    const float corr = (bh == 1.0f && bv == 1.0f) ? 0.0f : (float)(1.0 - (double)bh * (double)bv);
                    const float kk = G.cg * corr;
                    float d, art, det;
                    maps_px<true>(mA[j], mB[j], rw[j], kk, G.cg - kk, d, art, det);
                    if (EXPORT) {
                        float *m = mo.maps + (long long)(3 * G.g) * mo.mplane + (long long)y * mo.mpitch + xx;
                        m[0] = d;
                        m[mo.mplane] = art;
                        m[2 * mo.mplane] = det;
                    }
                    add_maps(ts, d, art, det);
                }
            }
        }
    }
    add_task(acc, ts);
}

// The geometry of one work item.
template <typename ST>
struct Item {
    ItemGeo G;
    int rows_out, nsteps;
    const ST *xr, *xd;
};

template <typename ST>
__device__ __forceinline__ Item<ST> decode_item(const DevPair &P, const Seg &sg, int tile, int g) {
    Item<ST> it;
    const int s = sg.scale;
    ItemGeo &G = it.G;
    G.W = P.w[s];
    G.H = P.h[s];
    G.g = g;
    const int local = tile - sg.first_tile;
    const int tx = local % sg.tiles_x, ty = local / sg.tiles_x;
    G.x0 = tx * kTileW;
    G.y0 = ty * sg.strip_rows;
    it.rows_out = min(G.y0 + sg.strip_rows, G.H) - G.y0;
    it.nsteps = (it.rows_out + kStep - 1) / kStep;
    G.lp = P.lp[s];
    const long long plane = (long long)G.lp * G.H;
    it.xr = (const ST *)P.lvl[0][s] + g * plane;
    it.xd = (const ST *)P.lvl[1][s] + g * plane;
    // anchor: reference XYB of channel g at the tile's first column, band start
    G.cg = ld_store<ST>(it.xr + (long long)((G.y0 / kBand) * kBand) * G.lp + G.x0);
    return it;
}

constexpr int kTileThreads = kFusedThreads;
constexpr int kTileBlocks = 4;  // resident blocks per SM (128 registers per thread, 47 KB shared)

// Issue the copies of stage load L of the item (input rows
// y0 - 4 + 8 L .. + 7) into `stage`, completing on `bar`.  Every warp takes a
// quarter: warp w announces the bytes of rows 4 (w & 1) .. + 3 of image
// w >> 1 (lane 0; the stage barriers count 4 arrivals a phase) and lanes 0..3
// copy one row each.  Spread over the four warps, the copies' address work
// no longer makes warp 0 the last to reach every barrier (one warp issuing
// all 16 copies: 3.07 instead of 2.85 ms per 64 x 1080p pairs).
// withhold: announce the bytes but copy nothing (the failure test's way to
// make the stage's waits run out).  ok: this lane's waits so far succeeded;
// once any lane of the warp has timed out the warp issues nothing more for
// the item, so no barrier ever sees a second arrival in an unfinished phase.
template <typename ST>
__device__ __forceinline__ void issue_rows(const Item<ST> &it, int L, float *stage, uint64_t *bar, int warp,
                                           int lane, bool withhold, bool ok) {
    if (!__all_sync(0xffffffffu, ok)) return;
    const ItemGeo &G = it.G;
    const int ybase = G.y0 - 4 + kStep * L;
    const int xs = max(G.x0 - 4, 0), xe = min(G.x0 + kCols - 4, G.lp);
    const unsigned bytes = (unsigned)(xe - xs) * (unsigned)sizeof(ST);
    // warp w copies rows 4 (w & 1) .. + 3 of image w >> 1
    const int k0 = 4 * (warp & 1);
    const int rows = max(0, min(k0 + 4, G.H - ybase) - max(k0, -ybase));  // its rows inside [0, H)
    // order this CTA's earlier generic reads of the stage before the async
    // copies that overwrite it
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    if (lane == 0) s2_mbar_expect(bar, (unsigned)rows * bytes);
    __syncwarp();
    if (lane < 4 && !withhold) {
        const int img = warp >> 1, k = k0 + lane, y = ybase + k;
        if (y >= 0 && y < G.H) {
            const ST *src = (img ? it.xd : it.xr) + (long long)y * G.lp + xs;
            s2_bulk_g2s(stage + (img * kStep + k) * kCols + (xs - (G.x0 - 4)), src, bytes, bar);
        }
    }
}

// One work item.  Stage load L (L = 0: the 8 priming rows y0 - 4 .. y0 + 3;
// L = st + 1: the rows of step st) goes to stage L % 2, issued two loads
// ahead: loads 0 and 1 at the start, load 2 after the priming rows are read,
// load st + 3 right after the barrier that follows step st's vertical phase
// (every thread has then read stage (st + 1) % 2, which it overwrites).  All
// loads of an item are consumed before it ends.  `phase` holds each stage's
// expected mbarrier parity (bit s), the same in every thread.
template <typename ST, bool EXPORT>
__device__ __forceinline__ bool flat_item(const Item<ST> &it, float2 *smb, float *stages, uint64_t *bars,
                                          unsigned &phase, const TileCheck &ck, int tid, double (*s_warp)[6],
                                          double *__restrict__ partials, int item, const MapOut &mo) {
    const ItemGeo &G = it.G;
    const float cg = G.cg;
    const int x = G.x0 - 4 + tid;
    const bool colin = x >= 0 && x < G.W;
    const bool cols_in = G.x0 >= 4 && G.x0 + kCols - 4 <= G.W;  // every column of the tile
    const int t_r = tid % kStep, t_s = tid / kStep;
    const bool t_on = tid < kTasks;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    const bool withhold = item == ck.drop_item;
    bool ok = true;
    auto stage = [&](int L) { return stages + (L & 1) * kStageFloats; };
    auto wait = [&](int L) {
        const int sidx = L & 1;
        ok &= s2_mbar_wait(&bars[sidx], (phase >> sidx) & 1u, ck.err);
        phase ^= 1u << sidx;
    };
    issue_rows<ST>(it, 0, stage(0), &bars[0], warp, lane, withhold, ok);
    issue_rows<ST>(it, 1, stage(1), &bars[1], warp, lane, withhold, ok);
    Rings R;
    wait(0);
    {
        StepRows in;
        v_load(in, stage(0), tid, colin, G.y0 - 4, G.H, cols_in && G.y0 >= 4 && G.y0 + 4 <= G.H, cg);
#pragma unroll
        for (int k = 0; k < 8; k++) ring_in(R, k, in.r[k], in.d[k], cg);
    }
    __syncthreads();  // stage 0 read by every thread
    if (it.nsteps >= 2) issue_rows<ST>(it, 2, stage(2), &bars[0], warp, lane, withhold, ok);
    float2 *const buf = smb;
    double *sacc = (double *)(stages + kStages * kStageFloats) + tid;
#pragma unroll
    for (int m = 0; m < 6; m++) sacc[m * kFusedThreads] = 0.0;
    auto step = [&](int st, auto s0) {
        const int r = st * kStep, nr = min(kStep, it.rows_out - r);
        const int ybase = G.y0 + r + 4;
        wait(st + 1);
        StepRows in;
        v_load(in, stage(st + 1), tid, colin, ybase, G.H, cols_in && nr == kStep && ybase + kStep <= G.H, cg);
        v_step<decltype(s0)::value>(R, in, cg, buf, tid);
        __syncthreads();
        if (st + 3 <= it.nsteps) issue_rows<ST>(it, st + 3, stage(st + 3), &bars[(st + 3) & 1], warp, lane, withhold, ok);
        h_step<EXPORT>(buf, r, nr, t_r, t_s, t_on, G, sacc, mo);
        __syncthreads();
    };
    for (int st = 0; st < it.nsteps; st += 2) {
        step(st, std::integral_constant<int, 0>());
        if (st + 1 < it.nsteps) step(st + 1, std::integral_constant<int, 8>());
    }
#pragma unroll
    for (int m = 0; m < 6; m++) {
        double v = sacc[m * kFusedThreads];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
        if ((tid & 31) == 0) s_warp[tid >> 5][m] = v;
    }
    __syncthreads();
    if (tid < 6) {
        double v = 0.0;
#pragma unroll
        for (int w = 0; w < kFusedThreads / 32; w++) v += s_warp[w][tid];
        partials[(long long)item * 6 + tid] = v;  // = tile * 18 + channel * 6 + m
    }
    return ok;
}

// Persistent: each block claims work items from the atomic counter until
// they run out.  Dynamic shared memory: the step buffer, the two row stages,
// the threads' f64 sums.  A block whose row copies time out (err set) stops claiming.
template <typename ST, bool EXPORT = false>
__global__ void __launch_bounds__(kFusedThreads, kTileBlocks)
    fused_kernel(const DevPair *__restrict__ pairs, const Seg *__restrict__ segs, int nseg, int first_item,
                 int end_item, int *__restrict__ counter, TileCheck ck, double *__restrict__ partials,
                 MapOut mo = MapOut{nullptr, 0, 0}) {
    extern __shared__ __align__(128) float2 smb[];  // [3 planes][kStep][kRS], then the stages and sums
    float *const stages = (float *)(smb + kBufF2);
    __shared__ int s_item, s_bad;
    __shared__ double s_warp[kFusedThreads / 32][6];
    __shared__ __align__(8) uint64_t s_bar[kStages];
    const int tid = threadIdx.x;
    if (tid == 0) {
        for (int i = 0; i < kStages; i++) s2_mbar_init(&s_bar[i]);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        s_bad = 0;
        s2_wait_limit = ck.wait_cycles;
    }
    unsigned phase = 0;
    for (;;) {
        __syncthreads();  // the previous item's readers of s_item, s_warp and the buffers are done
        if (tid == 0) s_item = s_bad ? end_item : first_item + atomicAdd(counter, 1);
        __syncthreads();
        const int item = s_item;
        if (item >= end_item) break;
        const int tile = item / 3, g = item - 3 * tile;
        const Seg sg = segs[find_seg(segs, nseg, tile)];
        const Item<ST> it = decode_item<ST>(pairs[sg.pair], sg, tile, g);
        if (!flat_item<ST, EXPORT>(it, smb, stages, s_bar, phase, ck, tid, s_warp, partials, item, mo))
            s_bad = 1;
    }
    // after a time-out, give copies still in flight a bounded wait before the
    // block's shared memory goes away
    if (s_bad)
        for (int i = 0; i < kStages; i++) s2_mbar_wait(&s_bar[i], (phase >> i) & 1u, ck.err);
}

// ---------------------------------------------------------------------------
// finalize: tile sums -> 108 statistics -> score
// ---------------------------------------------------------------------------
__constant__ double c_weight[108];

// The tile records of a scale are contiguous ([tile_base, tile_base + cnt),
// 18 doubles each).  They are staged in shared memory kFinChunk at a time by
// coalesced loads of the whole block; then the 18 threads of that scale add
// their column in tile order (the fixed order that makes a pair's result
// independent of the rest of the batch).
constexpr int kFinThreads = 256, kFinChunk = 128;

// err: set by a tile pass whose row copies timed out; every pair of the
// submission then reports S2_ERR_TIMEOUT.
__global__ void __launch_bounds__(kFinThreads) finalize_kernel(const DevPair *__restrict__ pairs, int npairs,
                                                               const double *__restrict__ partials,
                                                               const int *__restrict__ err,
                                                               DevResult *__restrict__ out) {
    __shared__ double st[108];
    __shared__ double rec[kFinChunk * 18];
    const int p = blockIdx.x;
    const DevPair &P = pairs[p];
    const int t = threadIdx.x;
    const int c = t / 36, sc_t = (t % 36) / 6, k = t % 6;
    double sum = 0.0;
    const int ns = P.status == 0 ? P.nscales : 0;
    for (int s = 0; s < ns; s++) {
        const int base = P.tile_base[s], cnt = P.tile_cnt[s];
        for (int i0 = 0; i0 < cnt; i0 += kFinChunk) {
            const int n = min(kFinChunk, cnt - i0);
            const double *src = partials + (long long)(base + i0) * 18;
            for (int j = t; j < n * 18; j += kFinThreads) rec[j] = src[j];
            __syncthreads();
            if (t < 108 && sc_t == s)
                for (int i = 0; i < n; i++) sum += rec[i * 18 + c * 6 + k];
            __syncthreads();
        }
    }
    if (t < 108) {
        double v = 0.0;
        if (sc_t < ns) {
            const double inv = 1.0 / ((double)P.w[sc_t] * (double)P.h[sc_t]);
            v = k < 3 ? sum * inv : sqrt(sqrt(sum * inv));
        }
        st[t] = v;
        out[p].stats[t] = v;
        out[p].sums[t] = sum;
    }
    __syncthreads();
    if (t == 0) {
        double sc = 0.0;
        for (int i = 0; i < 108; i++) sc = fma(c_weight[i], fabs(st[i]), sc);
        sc *= 0.9562382616834844;
        sc = fma(6.248496625763138e-5 * sc * sc, sc, fma(2.326765642916932, sc, -0.020884521182843837 * sc * sc));
        sc = sc > 0.0 ? fma(pow(sc, 0.6276336467831387), -10.0, 100.0) : 100.0;
        out[p].score = P.status == 0 ? sc : 0.0;
        out[p].n_scales = P.status == 0 ? P.nscales : 0;
        out[p].status = (P.status == 0 && err && *err) ? (int)S2_ERR_TIMEOUT : P.status;
    }
}

}  // namespace s2

// ---------------------------------------------------------------------------
// launch wrappers (C++ linkage, used by ssim2_engine.cpp)
// ---------------------------------------------------------------------------
#include "ssim2_launch.h"

namespace s2 {

static const double kWeights[108] = {
    0.0, 0.0007376606707406586, 0.0, 0.0, 0.0007793481682867309, 0.0,
    0.0, 0.0004371155730107379, 0.0, 1.1041726426657346, 0.00066284834129271, 0.00015231632783718752,
    0.0, 0.0016406437456599754, 0.0, 1.8422455520539298, 11.441172603757666, 0.0,
    0.0007989109436015163, 0.000176816438078653, 0.0, 1.8787594979546387, 10.94906990605142, 0.0,
    0.0007289346991508072, 0.9677937080626833, 0.0, 0.00014003424285435884, 0.9981766977854967, 0.00031949755934435053,
    0.0004550992113792063, 0.0, 0.0, 0.0013648766163243398, 0.0, 0.0,
    0.0, 0.0, 0.0, 7.466890328078848, 0.0, 17.445833984131262,
    0.0006235601634041466, 0.0, 0.0, 6.683678146179332, 0.00037724407979611296, 1.027889937768264,
    225.20515300849274, 0.0, 0.0, 19.213238186143016, 0.0011401524586618361, 0.001237755635509985,
    176.39317598450694, 0.0, 0.0, 24.43300999870476, 0.28520802612117757, 0.0004485436923833408,
    0.0, 0.0, 0.0, 34.77906344483772, 44.835625328877896, 0.0,
    0.0, 0.0, 0.0, 0.0, 0.0, 0.0,
    0.0, 0.0008680556573291698, 0.0, 0.0, 0.0, 0.0,
    0.0, 0.0005313191874358747, 0.0, 0.00016533814161379112, 0.0, 0.0,
    0.0, 0.0, 0.0, 0.0004179171803251336, 0.0017290828234722833, 0.0,
    0.0020827005846636437, 0.0, 0.0, 8.826982764996862, 23.19243343998926, 0.0,
    95.1080498811086, 0.9863978034400682, 0.9834382792465353, 0.0012286405048278493, 171.2667255897307, 0.9807858872435379,
    0.0, 0.0, 0.0, 0.0005130064588990679, 0.0, 0.00010854057858411537,
};

const double *host_weights() { return kWeights; }

cudaError_t upload_weights() { return cudaMemcpyToSymbol(c_weight, kWeights, sizeof kWeights); }

size_t fused_smem_bytes() { return (size_t)kBufF2 * sizeof(float2) + (size_t)kStages * kStageFloats * sizeof(float) + 6 * kFusedThreads * sizeof(double); }
int fused_threads() { return kTileThreads; }

template <bool EXPORT>
static cudaError_t fused_attrs() {
    const void *f = (const void *)fused_kernel<float, EXPORT>;
    // the tile pass is limited by registers and shared memory together: ask
    // for the largest shared-memory carveout so that 4 blocks fit per SM
    cudaError_t e = cudaFuncSetAttribute(f, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fused_smem_bytes());
}

cudaError_t configure_kernels() {
    cudaError_t e;
    if ((e = fused_attrs<false>()) != cudaSuccess) return e;
    if ((e = fused_attrs<true>()) != cudaSuccess) return e;
    return configure_dssim_kernels();
}

// The XYB planes are f32 (S2_STORAGE_F32, the only storage type offered).
int fused_blocks_per_sm(int storage) {
    (void)storage;
    int n = 0;
    const void *f = (const void *)fused_kernel<float, false>;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, f, kTileThreads, fused_smem_bytes()) != cudaSuccess) return 1;
    return n > 0 ? n : 1;
}

template <int OUT, int FMT>
static void prep_launch_f(const DevPair *pairs, int npairs, const int *blk_first, int first_block, int end_block,
                          const ColorConsts &cc, const float *lut, int grid, cudaStream_t st) {
    prep_kernel<float, OUT, FMT>
        <<<grid, kPrepThreads, 0, st>>>(pairs, npairs, blk_first, first_block, end_block, cc, lut);
}

template <int OUT>
static void prep_launch(const DevPair *pairs, int npairs, const int *blk_first, int first_block, int end_block,
                        const ColorConsts &cc, const float *lut, int grid, cudaStream_t st, int fmt) {
    switch (fmt) {
    case FMT_LINEAR_F32:
        prep_launch_f<OUT, FMT_LINEAR_F32>(pairs, npairs, blk_first, first_block, end_block, cc, lut, grid, st);
        break;
    case FMT_SRGB8:
        prep_launch_f<OUT, FMT_SRGB8>(pairs, npairs, blk_first, first_block, end_block, cc, lut, grid, st);
        break;
    case FMT_NV12:
        prep_launch_f<OUT, FMT_NV12>(pairs, npairs, blk_first, first_block, end_block, cc, lut, grid, st);
        break;
    case FMT_P016:
        prep_launch_f<OUT, FMT_P016>(pairs, npairs, blk_first, first_block, end_block, cc, lut, grid, st);
        break;
    case FMT_RGB16:
        prep_launch_f<OUT, FMT_RGB16>(pairs, npairs, blk_first, first_block, end_block, cc, lut, grid, st);
        break;
    default: prep_launch_f<OUT, -1>(pairs, npairs, blk_first, first_block, end_block, cc, lut, grid, st); break;
    }
}

cudaError_t launch_pyramid(int storage, const DevPair *pairs, int npairs, const int *blk_first, int first_block,
                           int end_block, const ColorConsts &cc, const float *lut, int grid, cudaStream_t st,
                           int out, int fmt) {
    const int nb = end_block - first_block;
    if (nb <= 0) return cudaSuccess;
    grid = grid > nb ? nb : grid;
    (void)storage;
    if (out == 3) prep_launch<3>(pairs, npairs, blk_first, first_block, end_block, cc, lut, grid, st, fmt);
    else if (out == 2) prep_launch<2>(pairs, npairs, blk_first, first_block, end_block, cc, lut, grid, st, fmt);
    else prep_launch<1>(pairs, npairs, blk_first, first_block, end_block, cc, lut, grid, st, fmt);
    return cudaGetLastError();
}

cudaError_t launch_fused(int storage, const DevPair *pairs, const Seg *segs, int nseg, int first_tile, int end_tile,
                         int *counter, const TileCheck &ck, double *partials, int grid, cudaStream_t st) {
    const int fi = 3 * first_tile, ei = 3 * end_tile;  // work items: (tile, channel)
    const int nt = ei - fi;
    if (nt <= 0) return cudaSuccess;
    grid = grid > nt ? nt : grid;
    (void)storage;
    fused_kernel<float, false><<<grid, kTileThreads, fused_smem_bytes(), st>>>(pairs, segs, nseg, fi, ei, counter,
                                                                              ck, partials, MapOut{nullptr, 0, 0});
    return cudaGetLastError();
}

cudaError_t launch_fused_export(int storage, const DevPair *pairs, const Seg *segs, int nseg, int first_tile,
                                int end_tile, int *counter, const TileCheck &ck, double *partials, float *maps,
                                long long mpitch, long long mplane, int grid, cudaStream_t st) {
    const int fi = 3 * first_tile, ei = 3 * end_tile;
    const int nt = ei - fi;
    if (nt <= 0) return cudaSuccess;
    grid = grid > nt ? nt : grid;
    (void)storage;
    fused_kernel<float, true><<<grid, kTileThreads, fused_smem_bytes(), st>>>(pairs, segs, nseg, fi, ei, counter,
                                                                             ck, partials, MapOut{maps, mpitch, mplane});
    return cudaGetLastError();
}

// Device copy of the submission descriptors from page-locked host memory
// (read through the host mapping), 16 bytes per thread.
__global__ void __launch_bounds__(256) desc_copy_kernel(uint4 *__restrict__ dst, const uint4 *__restrict__ src, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) dst[i] = src[i];
}

cudaError_t launch_desc_copy(void *dst, const void *src_host_mapped, size_t bytes, cudaStream_t st) {
    const int n = (int)(bytes / 16);
    if (n <= 0) return cudaSuccess;
    const int grid = n < 256 * 64 ? (n + 255) / 256 : 64;
    desc_copy_kernel<<<grid, 256, 0, st>>>((uint4 *)dst, (const uint4 *)src_host_mapped, n);
    return cudaGetLastError();
}

cudaError_t launch_finalize(const DevPair *pairs, int npairs, const double *partials, const int *err,
                            DevResult *out, cudaStream_t st) {
    if (npairs <= 0) return cudaSuccess;
    finalize_kernel<<<npairs, kFinThreads, 0, st>>>(pairs, npairs, partials, err, out);
    return cudaGetLastError();
}

}  // namespace s2
