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
//                    56 columns x `strip_rows` rows at one scale of one pair.
//                    Walking down the tile it forms the five blurred inputs on
//                    band-shifted values, runs the vertical 9-tap FIR in
//                    registers, then every 9 rows the horizontal FIR, the
//                    SSIM / artifact / detail-loss maps and their L1/L4 sums
//                    from shared memory.  Only 6 pooled sums per item leave
//                    the SM.  (blur.rs, error_maps.rs, lib.rs:862-1016)
//   finalize_kernel  per pair: fixed-order f64 reduction of the tile sums,
//                    the 108 statistics and the score (lib.rs:1018-1192).
//
// The blur is the exact closed form of the reference's recursive Gaussian:
// the truncated-cosine recursion of blur.rs equals, in exact arithmetic, a
// symmetric 9-tap FIR with zero padding.  Moments are taken of values shifted
// by one reference XYB sample per (56-column tile, 63-row band), which removes
// most of the f32 cancellation in sigma - mu^2; the shift is undone
// algebraically (including at image borders, where the blur of a constant is
// not the constant).
#include "ssim2_device.cuh"

namespace s2 {

// Shared memory layout of fused_kernel (one CTA = one channel of a tile).
// Rows ("rb" = output row of the 9-row block) of the float2 arrays are
// kRowStride2 float2 apart and rows of the float array kRowStride1 floats
// apart.  The horizontal tasks read them with 16-byte loads, lane t taking
// block row t % 9 and segment t / 9: with kRowStride2 / 2 and
// kRowStride1 / 4 odd, consecutive rows fall in distinct 16-byte bank groups
// (at most 2-way where a load phase spans two segments).  The plain
// 64-element stride gave up to 10-way conflicts.
constexpr int kRB = kRowsPerBlk;                         // rows of one block
constexpr int kRowStride2 = 74;                          // float2 elements
constexpr int kRowStride1 = 76;                          // float elements
static_assert(kRowStride2 % 2 == 0 && (kRowStride2 / 2) % 2 == 1, "16-byte aligned rows, odd 16-byte stride");
static_assert(kRowStride1 % 4 == 0 && (kRowStride1 / 4) % 2 == 1, "16-byte aligned rows, odd 16-byte stride");
constexpr int kSmVo2 = 2 * kRB * kRowStride2 * 2;        // vertical FIR of (x,y), (xx,yy) [pair][rb][col] (floats)
constexpr int kSmXo = kRB * kRowStride2 * 2;             // shifted raw XYB (x', y') of the output rows [rb][col]
constexpr int kSmVo1 = kRB * kRowStride1;                // vertical FIR of xy [rb][col]
constexpr int kFusedSmemFloats = kSmVo2 + kSmXo + kSmVo1;
constexpr int kFusedThreads = kCols;
constexpr int kTasks = kRB * kSegs;                      // horizontal tasks per 9-row block
static_assert(kSmVo2 % 4 == 0 && kSmXo % 4 == 0, "arrays start 16-byte aligned");

__device__ __forceinline__ float fir9(float a0, float a1, float a2, float a3, float a4, float a5,
                                      float a6, float a7, float a8) {
    float acc = S2_T4 * (a0 + a8);
    acc = fmaf(S2_T3, a1 + a7, acc);
    acc = fmaf(S2_T2, a2 + a6, acc);
    acc = fmaf(S2_T1, a3 + a5, acc);
    return fmaf(S2_T0, a4, acc);
}

// The same FIR on two planes at once (sm_100 packed f32x2; each lane rounds
// exactly as the scalar fir9).
__device__ __forceinline__ float2 fir9x2(float2 a0, float2 a1, float2 a2, float2 a3, float2 a4, float2 a5,
                                         float2 a6, float2 a7, float2 a8) {
    float2 acc = s2_mul2(make_float2(S2_T4, S2_T4), s2_add2(a0, a8));
    acc = __ffma2_rn(make_float2(S2_T3, S2_T3), s2_add2(a1, a7), acc);
    acc = __ffma2_rn(make_float2(S2_T2, S2_T2), s2_add2(a2, a6), acc);
    acc = __ffma2_rn(make_float2(S2_T1, S2_T1), s2_add2(a3, a5), acc);
    return __ffma2_rn(make_float2(S2_T0, S2_T0), a4, acc);
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

// OUT: bit 0 SSIMULACRA2's XYB planes, bit 1 DSSIM's Lab planes (both from
// the same linear pyramid).  OUT == 1 is the SSIMULACRA2-only pass.
template <int FMT, typename ST, int OUT>
__device__ __forceinline__ void prep_quads(const DevPair &P, int X0, int Y0, const float *lut, const ColorConsts &cc,
                                           float (*lv1)[3][kLv1 * kLv1]) {
    constexpr bool KU = FMT != FMT_LINEAR_F32;
    constexpr bool kX = (OUT & 1) != 0, kL = (OUT & 2) != 0;
    const int W = P.w[0], H = P.h[0];
    const bool scale1 = (kL ? P.prep_levels : P.nscales) > 1;
    for (int q = threadIdx.x; q < kLv1 * kLv1; q += blockDim.x) {
        const int qx = q % kLv1, qy = q / kLv1;
        const int x = X0 + 2 * qx, y = Y0 + 2 * qy;
        if (x >= W || y >= H) continue;
        const bool vx = x + 1 < W, vy = y + 1 < H;
        // 4:2:0 YUV: both images' samples are loaded before either is converted
        constexpr bool kYuv = FMT == FMT_NV12 || FMT == FMT_P016;
        constexpr int kEs = FMT == FMT_P016 ? 2 : 1;
        Nv12Quad nq0{}, nq1{};
        if (kYuv) {
            if (P.prep_mask & 1) nq0 = yuv_load_quad<kEs>(P, 0, x, y);
            if (P.prep_mask & 2) nq1 = yuv_load_quad<kEs>(P, 1, x, y);
        }
#pragma unroll 1
        for (int img = 0; img < 2; img++) {
            if (!((P.prep_mask >> img) & 1)) continue;
            float v[4][3];
            if (kYuv) yuv_quad_linear<kEs>(img ? nq1 : nq0, P, v);
            else lin_quad<FMT>(P, img, x, y, vx, vy, lut, cc, v);
            if (kX && (!kL || P.nscales > 0)) {
                ST *dst = (ST *)P.lvl[img][0];
                const long long plane = (long long)P.lp[0] * H;
                const long long off = (long long)y * P.lp[0] + x;
                if (vx) store_xyb_pair<ST, KU>(dst, plane, off, v[0], v[1]);
                else store_xyb<ST, KU>(P, img, 0, x, y, v[0]);
                if (vy) {
                    if (vx) store_xyb_pair<ST, KU>(dst, plane, off + P.lp[0], v[2], v[3]);
                    else store_xyb<ST, KU>(P, img, 0, x, y + 1, v[2]);
                }
            }
            if (kL) {
                store_lab(P, img, 0, x, y, v[0]);
                if (vx) store_lab(P, img, 0, x + 1, y, v[1]);
                if (vy) store_lab(P, img, 0, x, y + 1, v[2]);
                if (vx && vy) store_lab(P, img, 0, x + 1, y + 1, v[3]);
            }
            if (!scale1) continue;
            // far-edge clamp: a missing column repeats the left pixel, a
            // missing row the upper one
            float l1[3];
#pragma unroll
            for (int c = 0; c < 3; c++) {
                const float a = v[0][c];
                const float b = vx ? v[1][c] : a;
                const float cc2 = vy ? v[2][c] : a;
                const float d = vy ? (vx ? v[3][c] : cc2) : b;
                float sum = a + b;
                sum = sum + cc2;
                sum = sum + d;
                l1[c] = sum * 0.25f;
                lv1[img][c][q] = l1[c];
            }
            if (kX && (!kL || P.nscales > 1)) store_xyb<ST, KU>(P, img, 1, (X0 >> 1) + qx, (Y0 >> 1) + qy, l1);
            if (kL) store_lab(P, img, 1, (X0 >> 1) + qx, (Y0 >> 1) + qy, l1);
        }
    }
}

template <typename ST, int OUT>
__global__ void __launch_bounds__(256, 3) prep_kernel(const DevPair *__restrict__ pairs, int npairs,
                                                   const int *__restrict__ blk_first, int first_block,
                                                   int end_block,
                                                   ColorConsts cc, const float *__restrict__ lut_g) {
    __shared__ float lv1[2][3][kLv1 * kLv1];              // scale-1 linear block [img][ch][px]
    __shared__ float pp[2][2][3][(kLv1 / 2) * (kLv1 / 2)];  // scales >= 2, ping-pong
    __shared__ float lut[256];
    // the block's pair descriptor: in shared memory, so the level stores
    // (global) cannot alias it and its fields need no per-thread copy
    __shared__ DevPair sP;
    static_assert(sizeof(DevPair) % 8 == 0, "DevPair copied as 8-byte words");
    for (int i = threadIdx.x; i < 256; i += blockDim.x) lut[i] = lut_g[i];
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
        switch (P.fmt) {
        case FMT_LINEAR_F32: prep_quads<FMT_LINEAR_F32, ST, OUT>(P, X0, Y0, lut, cc, lv1); break;
        case FMT_SRGB8: prep_quads<FMT_SRGB8, ST, OUT>(P, X0, Y0, lut, cc, lv1); break;
        case FMT_NV12: prep_quads<FMT_NV12, ST, OUT>(P, X0, Y0, lut, cc, lv1); break;
        case FMT_P016: prep_quads<FMT_P016, ST, OUT>(P, X0, Y0, lut, cc, lv1); break;
        default: prep_quads<FMT_RGB16, ST, OUT>(P, X0, Y0, lut, cc, lv1); break;
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
// Work item = (tile, channel): item = 3 * tile + channel, 64 threads (two
// warps) per CTA, so that a block barrier waits for two warps only and up to
// ten CTAs share an SM.  A tile's three items write the tile's 18 partial
// sums (channel-major) and are summed in the same order as one CTA per tile
// over all channels would.
//
// EXPORT (error-map export, one scale of one pair): every pixel's SSIM error,
// artifact and detail-loss values are also stored to `maps`, 9 planes
// [channel][map] of `mpitch` floats per row and `mplane` floats per plane.
struct MapOut {
    float *maps;
    long long mpitch, mplane;
};

template <typename ST, bool EXPORT = false>
__global__ void __maxnreg__(96)
    fused_kernel(const DevPair *__restrict__ pairs, const Seg *__restrict__ segs, int nseg,
                 int first_item, int end_item, int *__restrict__ counter, double *__restrict__ partials,
                 MapOut mo = MapOut{nullptr, 0, 0}) {
    extern __shared__ float sm[];
    float2 *s_vo2 = (float2 *)sm;                  // [pair][rb][col]
    float2 *s_xo = (float2 *)(sm + kSmVo2);        // [rb][col]
    float *s_vo1 = sm + kSmVo2 + kSmXo;            // [rb][col]
    __shared__ int s_item;
    __shared__ double s_red[kFusedThreads][6];

    const int col = threadIdx.x;
    const int tid = col;
    // horizontal task of this thread: segment-major over the 9 block rows
    const int t_r = tid % kRB, t_s = tid / kRB;
    const bool t_on = tid < kTasks;

    for (;;) {
        __syncthreads();
        if (tid == 0) s_item = first_item + atomicAdd(counter, 1);
        __syncthreads();
        const int item = s_item;
        if (item >= end_item) break;
        const int tile = item / 3, g = item - 3 * tile;
        const Seg sg = segs[find_seg(segs, nseg, tile)];
        const DevPair &P = pairs[sg.pair];
        const int s = sg.scale;
        const int W = P.w[s], H = P.h[s];
        const int local = tile - sg.first_tile;
        const int tx = local % sg.tiles_x, ty = local / sg.tiles_x;
        const int x0 = tx * kTileW, y0 = ty * sg.strip_rows;
        const int y1 = min(y0 + sg.strip_rows, H);
        const long long plane = (long long)P.lp[s] * H;
        const ST *xr = (const ST *)P.lvl[0][s] + g * plane;
        const ST *xd = (const ST *)P.lvl[1][s] + g * plane;
        const int lp = P.lp[s];
        // shift: reference XYB of channel g at the tile's first column, band start
        const float cg = ld_store<ST>(xr + (long long)((y0 / kBand) * kBand) * lp + x0);

        const int x = x0 - 4 + col;
        const bool colin = (x >= 0) && (x < W);
        float2 w2a[9], w2b[9];  // windows of (x', y') and (x'^2, y'^2)
        float w1[9];            // window of x' y'
#pragma unroll
        for (int m = 0; m < 6; m++) s_red[tid][m] = 0.0;

        auto shifted = [&](float vr, float vd, bool in, float2 &a, float2 &b, float &c) {
            if (in) {
                const float px = vr - cg, py = vd - cg;
                a = make_float2(px, py);
                b = s2_mul2s(a, a);  // scalar squares: the FIR sums them
                c = px * py;
            } else {
                a = make_float2(0.f, 0.f);
                b = make_float2(0.f, 0.f);
                c = 0.f;
            }
        };

        // prime with input rows y0-4 .. y0+3 (window slots 0..7)
        {
            float lr[8], ld[8];
#pragma unroll
            for (int k = 0; k < 8; k++) {
                const int y = y0 - 4 + k;
                const bool in = colin && y >= 0 && y < H;
                lr[k] = in ? ld_store<ST>(xr + (long long)y * lp + x) : 0.f;
                ld[k] = in ? ld_store<ST>(xd + (long long)y * lp + x) : 0.f;
            }
#pragma unroll
            for (int k = 0; k < 8; k++) {
                const int y = y0 - 4 + k;
                shifted(lr[k], ld[k], colin && y >= 0 && y < H, w2a[k], w2b[k], w1[k]);
            }
        }

        const int rows_out = y1 - y0;
        for (int r0 = 0; r0 < rows_out; r0 += kRowsPerBlk) {
            const int nr = min(kRowsPerBlk, rows_out - r0);
            float lr[kRowsPerBlk], ld[kRowsPerBlk];
#pragma unroll
            for (int k = 0; k < kRowsPerBlk; k++) {
                const int y = y0 + r0 + k + 4;
                const bool in = k < nr && colin && y < H;
                lr[k] = in ? ld_store<ST>(xr + (long long)y * lp + x) : 0.f;
                ld[k] = in ? ld_store<ST>(xd + (long long)y * lp + x) : 0.f;
            }
#pragma unroll
            for (int k = 0; k < kRowsPerBlk; k++) {
                if (k < nr) {
                    const int sl = (8 + k) % 9;
                    const int y = y0 + r0 + k + 4;
                    shifted(lr[k], ld[k], colin && y < H, w2a[sl], w2b[sl], w1[sl]);
#define S2_W(a, j) a[(sl + 1 + (j)) % 9]
                    const float2 va = fir9x2(S2_W(w2a, 0), S2_W(w2a, 1), S2_W(w2a, 2), S2_W(w2a, 3), S2_W(w2a, 4),
                                             S2_W(w2a, 5), S2_W(w2a, 6), S2_W(w2a, 7), S2_W(w2a, 8));
                    const float2 vb = fir9x2(S2_W(w2b, 0), S2_W(w2b, 1), S2_W(w2b, 2), S2_W(w2b, 3), S2_W(w2b, 4),
                                             S2_W(w2b, 5), S2_W(w2b, 6), S2_W(w2b, 7), S2_W(w2b, 8));
                    const float vc = fir9(S2_W(w1, 0), S2_W(w1, 1), S2_W(w1, 2), S2_W(w1, 3), S2_W(w1, 4),
                                          S2_W(w1, 5), S2_W(w1, 6), S2_W(w1, 7), S2_W(w1, 8));
                    const int rb = k;
                    s_vo2[rb * kRowStride2 + col] = va;
                    s_vo2[(kRB + rb) * kRowStride2 + col] = vb;
                    s_vo1[rb * kRowStride1 + col] = vc;
                    s_xo[rb * kRowStride2 + col] = S2_W(w2a, 4);
#undef S2_W
                }
            }
            __syncthreads();
            // horizontal FIR + error maps: task = (row, channel, 8-px segment)
            if (t_on && t_r < nr) {
                const int y = y0 + r0 + t_r;
                const int xs = t_s * kSegW;
                if (x0 + xs < W) {
                    const int rb = t_r;
                    const float2 *pa = s_vo2 + rb * kRowStride2;
                    const float2 *pb = s_vo2 + (kRB + rb) * kRowStride2;
                    const float *pc = s_vo1 + rb * kRowStride1;
                    const float2 *px = s_xo + rb * kRowStride2;
                    // shift of the task's channel (same anchor as the vertical pass)
                    const float cv = ld_store<ST>((const ST *)P.lvl[0][s] + g * plane +
                                                  (long long)((y0 / kBand) * kBand) * lp + x0);
                    const float bv = border_gain(y, H);
#pragma unroll 1
                    for (int half = 0; half < kSegW / kChunk; half++) {
                        const int c0 = xs + half * kChunk;  // first output (tile coords), a multiple of 4
                        float2 ma[kChunk], mb[kChunk];
                        float mc[kChunk];
                        {
                            float2 v[kChunk + 8];
                            const float4 *q = (const float4 *)(pa + c0);
#pragma unroll
                            for (int j = 0; j < (kChunk + 8) / 2; j++) {
                                const float4 t4 = q[j];
                                v[2 * j] = make_float2(t4.x, t4.y);
                                v[2 * j + 1] = make_float2(t4.z, t4.w);
                            }
#pragma unroll
                            for (int j = 0; j < kChunk; j++)
                                ma[j] = fir9x2(v[j], v[j + 1], v[j + 2], v[j + 3], v[j + 4], v[j + 5], v[j + 6], v[j + 7], v[j + 8]);
                        }
                        {
                            float2 v[kChunk + 8];
                            const float4 *q = (const float4 *)(pb + c0);
#pragma unroll
                            for (int j = 0; j < (kChunk + 8) / 2; j++) {
                                const float4 t4 = q[j];
                                v[2 * j] = make_float2(t4.x, t4.y);
                                v[2 * j + 1] = make_float2(t4.z, t4.w);
                            }
#pragma unroll
                            for (int j = 0; j < kChunk; j++)
                                mb[j] = fir9x2(v[j], v[j + 1], v[j + 2], v[j + 3], v[j + 4], v[j + 5], v[j + 6], v[j + 7], v[j + 8]);
                        }
                        {
                            float v[kChunk + 8];
                            const float4 *q = (const float4 *)(pc + c0);
#pragma unroll
                            for (int j = 0; j < (kChunk + 8) / 4; j++) {
                                const float4 t4 = q[j];
                                v[4 * j] = t4.x;
                                v[4 * j + 1] = t4.y;
                                v[4 * j + 2] = t4.z;
                                v[4 * j + 3] = t4.w;
                            }
#pragma unroll
                            for (int j = 0; j < kChunk; j++)
                                mc[j] = fir9(v[j], v[j + 1], v[j + 2], v[j + 3], v[j + 4], v[j + 5], v[j + 6], v[j + 7], v[j + 8]);
                        }
                        float2 xyv[kChunk];
                        {
                            const float4 *q = (const float4 *)(px + c0 + 4);
#pragma unroll
                            for (int j = 0; j < kChunk / 2; j++) {
                                const float4 t4 = q[j];
                                xyv[2 * j] = make_float2(t4.x, t4.y);
                                xyv[2 * j + 1] = make_float2(t4.z, t4.w);
                            }
                        }
                        float fs[3] = {0.f, 0.f, 0.f}, f4[3] = {0.f, 0.f, 0.f};
                        const int xc = x0 + c0;
                        if (bv == 1.0f && xc >= 4 && xc + kChunk + 4 <= W) {
                            // every pixel of the chunk is interior: border gain
                            // 1, so the correction term kk of the general form
                            // below is zero and drops out; all pixels inside
                            // the image.  The (mu1, mu2) and (art, det) pairs
                            // go through f32x2 operations (each lane rounds as
                            // the scalar operation).
                            float2 fs12 = make_float2(0.f, 0.f), f412 = make_float2(0.f, 0.f);
#pragma unroll
                            for (int j = 0; j < kChunk; j++) {
                                const float2 mu = ma[j];
                                const float2 nmu = make_float2(-mu.x, -mu.y);
                                const float2 var = __ffma2_rn(nmu, mu, mb[j]);  // (sigma11 - mu1^2, sigma22 - mu2^2)
                                const float cov = fmaf(nmu.x, mu.y, mc[j]);
                                const float md = mu.x - mu.y;
                                const float num_m = fmaf(-md, md, 1.0f);
                                const float num_s = fmaf(2.0f, cov, kC2);
                                const float den = (var.x + var.y) + kC2;
                                const float d = fmaxf(s2_div(fmaf(-num_m, num_s, den), den), 0.0f);
                                const float2 t = s2_add2(xyv[j], nmu);
                                const float aa = fabsf(t.x), bb = fabsf(t.y);
                                const float d1 = s2_div(bb - aa, 1.0f + aa);
                                const float2 ad = make_float2(fmaxf(d1, 0.0f), fmaxf(-d1, 0.0f));
                                if (EXPORT) {
                                    float *m = mo.maps + (long long)(3 * g) * mo.mplane + (long long)y * mo.mpitch + xc + j;
                                    m[0] = d;
                                    m[mo.mplane] = ad.x;
                                    m[2 * mo.mplane] = ad.y;
                                }
                                const float q = d * d;
                                fs[0] += d;
                                f4[0] += q * q;
                                const float2 q2 = s2_mul2(ad, ad);
                                fs12 = s2_add2(fs12, ad);
                                f412 = s2_add2(f412, s2_mul2s(q2, q2));  // scalar: summed
                            }
                            fs[1] = fs12.x;
                            fs[2] = fs12.y;
                            f4[1] = f412.x;
                            f4[2] = f412.y;
                        } else {
#pragma unroll
                        for (int j = 0; j < kChunk; j++) {
                            const int xx = x0 + c0 + j;
                            if (xx < W) {
                                const float m1 = ma[j].x, m2 = ma[j].y, s11 = mb[j].x, s22 = mb[j].y, s12 = mc[j];
                                const float2 xy = xyv[j];
                                const float bh = border_gain(xx, W);
                                const float corr =
                                    (bh == 1.0f && bv == 1.0f) ? 0.0f : (float)(1.0 - (double)bh * (double)bv);
                                const float kk = cv * corr;
                                const float e = cv - kk;
                                const float v1 = fmaf(kk, fmaf(2.0f, m1, e), fmaf(-m1, m1, s11));
                                const float v2 = fmaf(kk, fmaf(2.0f, m2, e), fmaf(-m2, m2, s22));
                                const float cov = fmaf(kk, (m1 + m2) + e, fmaf(-m1, m2, s12));
                                const float md = m1 - m2;
                                const float num_m = fmaf(-md, md, 1.0f);
                                const float num_s = fmaf(2.0f, cov, kC2);
                                const float den = (v1 + v2) + kC2;
                                float d = s2_div(fmaf(-num_m, num_s, den), den);
                                d = fmaxf(d, 0.0f);
                                const float aa = fabsf((xy.x - m1) + kk);
                                const float bb = fabsf((xy.y - m2) + kk);
                                const float d1 = s2_div(bb - aa, 1.0f + aa);
                                const float art = fmaxf(d1, 0.0f), det = fmaxf(-d1, 0.0f);
                                if (EXPORT) {
                                    float *m = mo.maps + (long long)(3 * g) * mo.mplane + (long long)y * mo.mpitch + xx;
                                    m[0] = d;
                                    m[mo.mplane] = art;
                                    m[2 * mo.mplane] = det;
                                }
                                float q;
                                fs[0] += d;   q = d * d;     f4[0] += q * q;
                                fs[1] += art; q = art * art; f4[1] += q * q;
                                fs[2] += det; q = det * det; f4[2] += q * q;
                            }
                        }
                        }
#pragma unroll
                        for (int m = 0; m < 3; m++) {
                            s_red[tid][m] += (double)fs[m];
                            s_red[tid][3 + m] += (double)f4[m];
                        }
                    }
                }
            }
            __syncthreads();
        }

        // channel reduction, fixed order: the tasks segment-major
        __syncthreads();
        if (tid < 6) {
            double v = 0.0;
            for (int t = 0; t < kTasks; t++) v += s_red[t][tid];
            partials[(long long)item * 6 + tid] = v;  // = tile * 18 + channel * 6 + m
        }
    }
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

__global__ void __launch_bounds__(kFinThreads) finalize_kernel(const DevPair *__restrict__ pairs, int npairs,
                                                               const double *__restrict__ partials,
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
        out[p].status = P.status;
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

size_t fused_smem_bytes() { return (size_t)kFusedSmemFloats * sizeof(float); }
int fused_threads() { return kFusedThreads; }

template <typename ST> static const void *fused_fn() { return (const void *)fused_kernel<ST>; }

cudaError_t configure_kernels() {
    cudaError_t e;
    // the fused pass is limited by registers and shared memory together: ask
    // for the largest shared-memory carveout so that 3 blocks fit per SM
    e = cudaFuncSetAttribute(fused_kernel<float>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(fused_kernel<__half>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(fused_kernel<__nv_bfloat16>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(fused_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fused_smem_bytes());
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(fused_kernel<__half>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fused_smem_bytes());
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(fused_kernel<__nv_bfloat16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fused_smem_bytes());
    if (e != cudaSuccess) return e;
    return configure_dssim_kernels();
}

int fused_blocks_per_sm(int storage) {
    int n = 0;
    const void *f = storage == ST_F16 ? fused_fn<__half>() : storage == ST_BF16 ? fused_fn<__nv_bfloat16>() : fused_fn<float>();
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, f, kFusedThreads, fused_smem_bytes()) != cudaSuccess) return 1;
    return n > 0 ? n : 1;
}

template <int OUT>
static void prep_launch(int storage, const DevPair *pairs, int npairs, const int *blk_first, int first_block,
                        int end_block, const ColorConsts &cc, const float *lut, int grid, cudaStream_t st) {
    // Lab planes are f32 whatever the storage type; XYB-less passes need one instance
    if constexpr (OUT != 2) {
        if (storage == ST_F16) {
            prep_kernel<__half, OUT><<<grid, 256, 0, st>>>(pairs, npairs, blk_first, first_block, end_block, cc, lut);
            return;
        }
        if (storage == ST_BF16) {
            prep_kernel<__nv_bfloat16, OUT>
                <<<grid, 256, 0, st>>>(pairs, npairs, blk_first, first_block, end_block, cc, lut);
            return;
        }
    }
    prep_kernel<float, OUT><<<grid, 256, 0, st>>>(pairs, npairs, blk_first, first_block, end_block, cc, lut);
}

cudaError_t launch_pyramid(int storage, const DevPair *pairs, int npairs, const int *blk_first, int first_block,
                           int end_block, const ColorConsts &cc, const float *lut, int grid, cudaStream_t st,
                           int out) {
    const int nb = end_block - first_block;
    if (nb <= 0) return cudaSuccess;
    grid = grid > nb ? nb : grid;
    if (out == 3) prep_launch<3>(storage, pairs, npairs, blk_first, first_block, end_block, cc, lut, grid, st);
    else if (out == 2) prep_launch<2>(storage, pairs, npairs, blk_first, first_block, end_block, cc, lut, grid, st);
    else prep_launch<1>(storage, pairs, npairs, blk_first, first_block, end_block, cc, lut, grid, st);
    return cudaGetLastError();
}

cudaError_t launch_fused(int storage, const DevPair *pairs, const Seg *segs, int nseg, int first_tile, int end_tile,
                         int *counter, double *partials, int grid, cudaStream_t st) {
    const int fi = 3 * first_tile, ei = 3 * end_tile;  // work items: (tile, channel)
    const int nt = ei - fi;
    if (nt <= 0) return cudaSuccess;
    grid = grid > nt ? nt : grid;
    dim3 block(kFusedThreads);
    size_t sm = fused_smem_bytes();
    if (storage == ST_F16)
        fused_kernel<__half><<<grid, block, sm, st>>>(pairs, segs, nseg, fi, ei, counter, partials);
    else if (storage == ST_BF16)
        fused_kernel<__nv_bfloat16><<<grid, block, sm, st>>>(pairs, segs, nseg, fi, ei, counter, partials);
    else
        fused_kernel<float><<<grid, block, sm, st>>>(pairs, segs, nseg, fi, ei, counter, partials);
    return cudaGetLastError();
}

cudaError_t launch_fused_export(int storage, const DevPair *pairs, const Seg *segs, int nseg, int first_tile,
                                int end_tile, int *counter, double *partials, float *maps, long long mpitch,
                                long long mplane, int grid, cudaStream_t st) {
    const int fi = 3 * first_tile, ei = 3 * end_tile;
    const int nt = ei - fi;
    if (nt <= 0) return cudaSuccess;
    grid = grid > nt ? nt : grid;
    dim3 block(kFusedThreads);
    size_t sm = fused_smem_bytes();
    const MapOut mo{maps, mpitch, mplane};
    cudaError_t e;
    if (storage == ST_F16) {
        e = cudaFuncSetAttribute(fused_kernel<__half, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        if (e != cudaSuccess) return e;
        fused_kernel<__half, true><<<grid, block, sm, st>>>(pairs, segs, nseg, fi, ei, counter, partials, mo);
    } else if (storage == ST_BF16) {
        e = cudaFuncSetAttribute(fused_kernel<__nv_bfloat16, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)sm);
        if (e != cudaSuccess) return e;
        fused_kernel<__nv_bfloat16, true><<<grid, block, sm, st>>>(pairs, segs, nseg, fi, ei, counter, partials, mo);
    } else {
        e = cudaFuncSetAttribute(fused_kernel<float, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        if (e != cudaSuccess) return e;
        fused_kernel<float, true><<<grid, block, sm, st>>>(pairs, segs, nseg, fi, ei, counter, partials, mo);
    }
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

cudaError_t launch_finalize(const DevPair *pairs, int npairs, const double *partials, DevResult *out,
                            cudaStream_t st) {
    if (npairs <= 0) return cudaSuccess;
    finalize_kernel<<<npairs, kFinThreads, 0, st>>>(pairs, npairs, partials, out);
    return cudaGetLastError();
}

}  // namespace s2
