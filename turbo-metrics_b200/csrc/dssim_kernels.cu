// dssim_kernels.cu -- DSSIM (the metric of crates/dssim-cuda) over the Lab
// planes that the prep pass writes beside SSIMULACRA2's XYB planes, from the
// same linear-RGB pyramid.
//
//   dssim_clamp_kernel  levels that dssim-cuda clamps to 8 pixels
//                       (dssim-cuda/src/lib.rs:184-205) for small images:
//                       2x2 downscale of the kept linear level, then Lab
//   dssim_tile_kernel   per 32 x 32 output tile of one (pair, level): the
//                       a/b pre-blur (lib.rs:296-316), the two-pass blurs of
//                       x, y, x^2, y^2, xy for L, a, b (lib.rs:336-391), the
//                       channel-averaged SSIM (dssim-cuda-kernel/src/ssim.rs:
//                       152-236), stored to the level's SSIM map, and the
//                       tile's sum of SSIM in f64
//   dssim_mean_kernel   per (pair, level): mean SSIM, avg = mean^(0.5^s)
//                       (lib.rs:404-411)
//   dssim_mad_kernel    per tile: sum of |avg - ssim| (ssim.rs:240-262)
//   dssim_final_kernel  per pair: 1 - MAD per level, weighted mean, 1/ssim - 1
//                       (lib.rs:320-333, :457-460)
//
// The blurs are dssim-cuda's 3x3 kernel (blur.rs:13-17) with replicated
// borders, evaluated in shared memory one stage at a time: every stage's
// buffer holds, at each position, the stage's value at the position clamped
// into the level, which is what the next stage's clamped reads see in the
// reference.  Taps run row-major with a separate multiply and add (this unit
// is compiled with -fmad=false), so the SSIM map is the reference's f32
// arithmetic operation for operation.  Sums are f64 in a fixed order: a
// pair's DSSIM does not depend on the rest of its batch.
#include <cfloat>

#include "dssim_tile_map.h"
#include "ssim2_launch.h"

namespace s2 {

// dssim-cuda-kernel/src/blur.rs:13-17
__device__ __forceinline__ float ds_k(int i) {
    return (i == 4) ? 0.146293f : ((i & 1) ? 0.118095f : 0.095332f);
}

__device__ __forceinline__ int ds_clamp(int v, int hi) { return v < 0 ? 0 : (v > hi ? hi : v); }

// Fixed-order sum of n doubles by the whole block (kDsThreads threads):
// strided per-thread sums, then a tree; every caller gets the same value for
// the same array.
__device__ double ds_block_sum(const double *p, int n, double *red) {
    const int t = threadIdx.x;
    double s = 0.0;
    for (int i = t; i < n; i += kDsThreads) s += p[i];
    __syncthreads();
    red[t] = s;
    __syncthreads();
    for (int w = kDsThreads / 2; w > 0; w >>= 1) {
        if (t < w) red[t] += red[t + w];
        __syncthreads();
    }
    const double r = red[0];
    __syncthreads();
    return r;
}

__device__ double ds_block_reduce(double v, double *red) {
    const int t = threadIdx.x;
    __syncthreads();
    red[t] = v;
    __syncthreads();
    for (int w = kDsThreads / 2; w > 0; w >>= 1) {
        if (t < w) red[t] += red[t + w];
        __syncthreads();
    }
    const double r = red[0];
    __syncthreads();
    return r;
}

__device__ __forceinline__ int ds_find_seg(const DsSeg *segs, int nseg, int tile) {
    int lo = 0, hi = nseg - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (segs[mid].first_tile <= tile) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// ---------------------------------------------------------------------------
// clamp pass: one block per pair; levels clamp_from..4, each a 2x2 downscale
// of the previous one with clamped source indexes (downscale.rs:50-83), kept
// as linear RGB for the next level and stored as Lab.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kDsThreads) dssim_clamp_kernel(const DsPair *__restrict__ pairs) {
    const DsPair &P = pairs[blockIdx.x];
    if (P.status != 0 || P.clamp_from >= kDsLevels) return;
    for (int img = 0; img < 2; img++) {
        if (!((P.prep_mask >> img) & 1)) continue;
        for (int s = P.clamp_from; s < kDsLevels; s++) {
            const bool first = s == P.clamp_from;
            const float *src = first ? P.keep[img] : P.scratch[img] + ((s - 1) & 1) * 3 * P.splane;
            const int sw = first ? P.kw : P.w[s - 1], sh = first ? P.kh : P.h[s - 1];
            const long long sp = first ? P.kpitch : P.pitch[s - 1];
            const long long splane = first ? (long long)P.kpitch * P.kh : P.splane;
            float *lin = P.scratch[img] + (s & 1) * 3 * P.splane;
            float *lab = P.lab[img][s];
            const int W = P.w[s], H = P.h[s];
            const long long dp = P.pitch[s], dplane = (long long)P.pitch[s] * H;
            for (int i = threadIdx.x; i < W * H; i += kDsThreads) {
                const int ox = i % W, oy = i / W;
                const int x0 = min(2 * ox, sw - 1), x1 = min(2 * ox + 1, sw - 1);
                const int y0 = min(2 * oy, sh - 1), y1 = min(2 * oy + 1, sh - 1);
                float v[3];
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    const float *q = src + c * splane;
                    float sum = q[y0 * sp + x0] + q[y0 * sp + x1];
                    sum = sum + q[y1 * sp + x0];
                    sum = sum + q[y1 * sp + x1];
                    v[c] = sum * 0.25f;
                    lin[c * P.splane + oy * dp + ox] = v[c];
                }
                float o[3];
                ds_lab(v[0], v[1], v[2], o);
#pragma unroll
                for (int c = 0; c < 3; c++) lab[c * dplane + oy * dp + ox] = o[c];
            }
            __syncthreads();  // level s is read by level s + 1
        }
    }
}

// ---------------------------------------------------------------------------
// tile pass
// ---------------------------------------------------------------------------
//
// Each blur stage fills an n x n buffer (n = 32 + 2 x its halo, even) from the
// (n + 2)-wide buffer of the stage before.  A thread takes two adjacent
// columns and a run of consecutive rows and slides a 3 x 4 window of the
// input down them (two 8-byte shared loads per row).  The taps' products
// are formed once per input row (ds_prod) and added, one f32x2 add for both
// columns per tap, in the reference's row-major tap order: every lane rounds
// as the scalar reference does.  The first tap initialises the sum, which equals 0 + tap
// for every tap but -0 (no Lab value or product of two is -0 where it
// matters: the sign of a zero sum does not reach the SSIM).  x^2, y^2 and xy
// are formed as the first statistics blur reads its window rows
// (ds_stat_blur).  The window is evaluated at every position; on tiles that
// touch the level's edge, positions outside the level then take the value of
// the position clamped into it (ds_fix_edges), which is what the reference's
// next stage reads there with clamped indexes.
// One input row of a thread's window: columns c .. c + 3 as two aligned
// register pairs (w0, w1), (w2, w3).
struct DsRow {
    float2 a, b;
};

__device__ __forceinline__ DsRow ds_row(const float *src) {
    return DsRow{*(const float2 *)src, *(const float2 *)(src + 2)};
}

// The products of one window row with its taps for both columns, in tap
// order kx = 0, 1, 2: (k0 w0, k0 w1), (k1 w1, k1 w2), (k0 w2, k0 w3), where
// k0 is the row's outer tap and k1 its middle one (corner / edge for the top
// and bottom rows, edge / centre for the middle row).  A product is the same
// rounded value whichever output and window position uses it, so a row's
// outer products are formed once and used by the two outputs whose top and
// bottom row it is, and its middle products once when it is the middle row
// (8 instructions per row instead of 18 multiplies).  The aligned pairs are
// packed FMAs with the addend -0 (nz): k w + (-0) rounds exactly as k w,
// signed zeros included, and an FMA cannot be fused with the add that
// follows (a packed multiply feeding a packed add is fused even under
// -fmad=false); the middle pair (w1, w2) is not an aligned register pair, so
// its two products are scalar multiplies (never fused under -fmad=false).
struct DsProd {
    float2 p0, p1, p2;
};

__device__ __forceinline__ DsProd ds_prod(const DsRow &w, float k0, float k1, float2 nz) {
    DsProd p;
    p.p0 = __ffma2_rn(make_float2(k0, k0), w.a, nz);
    p.p1 = make_float2(w.a.y * k1, w.b.x * k1);
    p.p2 = __ffma2_rn(make_float2(k0, k0), w.b, nz);
    return p;
}

// The 3 x 3 window of both columns, the nine products added in the
// reference's row-major tap order.
__device__ __forceinline__ float2 ds_sum3(const DsProd &t, const DsProd &m, const DsProd &b) {
    float2 s = t.p0;
    s = __fadd2_rn(s, t.p1);
    s = __fadd2_rn(s, t.p2);
    s = __fadd2_rn(s, m.p0);
    s = __fadd2_rn(s, m.p1);
    s = __fadd2_rn(s, m.p2);
    s = __fadd2_rn(s, b.p0);
    s = __fadd2_rn(s, b.p1);
    return __fadd2_rn(s, b.p2);
}

// L output rows of one column pair from input rows row(0) .. row(L + 1)
template <int L, typename R, typename F>
__device__ __forceinline__ void ds_blur_rows(R &&row, float2 nz, F &&emit) {
    const float kc = ds_k(0), ke = ds_k(1), km = ds_k(4);
    DsProd top = ds_prod(row(0), kc, ke, nz);
    DsRow mid = row(1);
    DsProd mid_outer = ds_prod(mid, kc, ke, nz);
#pragma unroll
    for (int r = 0; r < L; r++) {
        const DsRow nw = row(r + 2);
        const DsProd bot = ds_prod(nw, kc, ke, nz);
        emit(r, ds_sum3(top, ds_prod(mid, ke, km, nz), bot));
        top = mid_outer;
        mid = nw;
        mid_outer = bot;
    }
}

// the same from rows src[0 .. L + 1] of pitch m
template <int L, int m, typename F>
__device__ __forceinline__ void ds_blur_run(const float *src, float2 nz, F &&emit) {
    ds_blur_rows<L>([&](int i) { return ds_row(src + i * m); }, nz, emit);
}

// `planes` planes: out[p] (n x n) = 3x3 blur of in[p] (pitch n + 2, plane
// (n + 2)^2).  Thread t takes one column pair of one plane and a run of L
// rows (ds_item): the plane's n / 2 column pairs times S row segments, at
// most one item per thread; segment k starts at row min(k L, n - L), so the last run
// may overlap the one before it (those rows are written twice, with the same
// values).  Every size is a compile-time constant: the item's plane, columns
// and rows are found once, and the run is unrolled without row checks.
template <int n, int planes, int S, int L>
__device__ __forceinline__ void ds_stage_blur(const float *in, float *out, float2 nz) {
    constexpr int m = n + 2, half = n / 2, items = planes * half * S;
    static_assert(items <= kDsThreads && S * L >= n && L <= n && n % 2 == 0, "one run per thread");
    int p, seg, c;
    if (!ds_item<half, S, planes>(threadIdx.x, p, seg, c)) return;
    const int j0 = min(seg * L, n - L);
    const float *src = in + p * m * m + j0 * m + c;
    float *dst = out + p * n * n + j0 * n + c;
    ds_blur_run<L, m>(src, nz, [&](int r, float2 v) { *(float2 *)(dst + r * n) = v; });
}

// The first statistics blur: the five planes x, y, x^2, y^2, xy (n = 34
// outputs, pitch 36) from the two input planes x and y.  Each plane is read
// as the product a b of two rows: x = x * 1, y = y * 1 (b read from four 1s
// at pitch 0), x^2, y^2, xy, each a packed FMA with the addend -0, so every
// input is the reference's separately rounded product (or the value
// itself); the products are not stored, which keeps the block's shared
// memory within four blocks per SM.  Every thread runs the same code for
// every plane (no divergence where a warp straddles two planes).
template <int S, int L>
__device__ __forceinline__ void ds_stat_blur(const float *in, const float *ones, float *out, float2 nz) {
    constexpr int n = kDsB, m = n + 2, mm = m * m, half = n / 2, items = 5 * half * S;
    static_assert(items <= kDsThreads && S * L >= n && L <= n && n % 2 == 0, "one run per thread");
    int p, seg, c;
    if (!ds_item<half, S, 5>(threadIdx.x, p, seg, c)) return;
    const int j0 = min(seg * L, n - L);
    const int pa = (p == 1 || p == 3) ? 1 : 0;           // x, y, x, y, x
    const int pb = p == 2 ? 0 : (p >= 3 ? 1 : -1);       // 1, 1, x, y, y
    const float *srcA = in + pa * mm + j0 * m + c;
    const float *srcB = pb < 0 ? ones : in + pb * mm + j0 * m + c;
    const int mB = pb < 0 ? 0 : m;
    float *dst = out + p * n * n + j0 * n + c;
    ds_blur_rows<L>(
        [&](int i) {
            const DsRow a = ds_row(srcA + i * m), b = ds_row(srcB + i * mB);
            return DsRow{__ffma2_rn(a.a, b.a, nz), __ffma2_rn(a.b, b.b, nz)};
        },
        nz, [&](int r, float2 v) { *(float2 *)(dst + r * n) = v; });
}

// L's blur inputs x and y: the raw region (2 planes of nn floats) copied out
// of R, which then takes the next channel's prefetch
__device__ __forceinline__ void ds_copy2(const float *in, float *out, int nn) {
    const float4 *s = (const float4 *)in;
    float4 *d = (float4 *)out;
    for (int i = threadIdx.x; i < 2 * nn / 4; i += kDsThreads) d[i] = s[i];
}

// Asynchronous global -> shared copies (cp.async) of 4, 8 or 16 bytes: the
// next channel's raw Lab region is fetched while the current channel
// computes.
template <int BYTES>
__device__ __forceinline__ void ds_cp(float *dst, const float *src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(d), "l"(src), "n"(BYTES) : "memory");
}

// Issue the copies of channel c's raw region of `tile` (halo HALO: 2 for L,
// 4 for a and b; clamped into the level) into R, pitch 32 + 2 x halo, both
// images.  The region's edge is a compile-time constant, so the element
// index splits into row and column without a division.
template <int HALO>
__device__ __forceinline__ void ds_prefetch_h(const DsPair *__restrict__ pairs, const DsSeg *__restrict__ segs,
                                              int nseg, int tile, int c, float *R) {
    constexpr int n = kDsT + 2 * HALO;
    const DsSeg sg = segs[ds_find_seg(segs, nseg, tile)];
    const DsPair &P = pairs[sg.pair];
    const int s = sg.level, W = P.w[s], H = P.h[s];
    const long long pitch = P.pitch[s], plane = pitch * H;
    const int tl = tile - sg.first_tile;
    const int X0 = (tl % sg.tiles_x) * kDsT, Y0 = (tl / sg.tiles_x) * kDsT;
    const float *xr = P.lab[0][s] + c * plane, *yr = P.lab[1][s] + c * plane;
    if (X0 >= HALO && X0 - HALO + n <= W && Y0 >= HALO && Y0 - HALO + n <= H) {
        // the region lies inside the level: whole rows in 16-byte (halo 4:
        // X0 - 4 is a multiple of 4 floats) or 8-byte (halo 2) pieces; the
        // Lab planes' pitch is a multiple of 64 floats and the planes are
        // 256-byte aligned
        constexpr int kCh = HALO % 4 == 0 ? 16 : 8, kPer = n * 4 / kCh, kF = kCh / 4;
        static_assert((n * 4) % kCh == 0 && (kDsT - HALO) * 4 % kCh == 0, "aligned pieces");
        for (int i = threadIdx.x; i < 2 * n * kPer; i += kDsThreads) {
            const int img = i >= n * kPer, r = img ? i - n * kPer : i;
            const int row = r / kPer, ch = r - row * kPer;
            ds_cp<kCh>(R + img * n * n + row * n + ch * kF,
                       (img ? yr : xr) + (long long)(Y0 - HALO + row) * pitch + (X0 - HALO) + ch * kF);
        }
    } else {
        for (int i = threadIdx.x; i < 2 * n * n; i += kDsThreads) {
            const int img = i >= n * n, r = img ? i - n * n : i;
            const int row = r / n, col = r - row * n;
            const int gx = ds_clamp(X0 - HALO + col, W - 1), gy = ds_clamp(Y0 - HALO + row, H - 1);
            ds_cp<4>(R + i, (img ? yr : xr) + gy * pitch + gx);
        }
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
}

__device__ __forceinline__ void ds_prefetch(const DsPair *__restrict__ pairs, const DsSeg *__restrict__ segs,
                                            int nseg, int tile, int c, float *R) {
    if (c == 0) ds_prefetch_h<2>(pairs, segs, nseg, tile, c, R);
    else ds_prefetch_h<4>(pairs, segs, nseg, tile, c, R);
}

// positions of an n x n stage buffer (origin X0 - h, Y0 - h) outside the
// level take the value at the position clamped into the level
template <int n, int h>
__device__ __forceinline__ void ds_fix_edges(float *buf, int planes, int X0, int Y0, int W, int H) {
    for (int i = threadIdx.x; i < n * n; i += kDsThreads) {
        const int x = X0 - h + i % n, y = Y0 - h + i / n;
        if (x >= 0 && x < W && y >= 0 && y < H) continue;
        const int src = (ds_clamp(y, H - 1) - (Y0 - h)) * n + ds_clamp(x, W - 1) - (X0 - h);
        for (int p = 0; p < planes; p++) buf[p * n * n + i] = buf[p * n * n + src];
    }
}

// Fixed-order block sum: each warp by shuffles, then the warps in order.
__device__ double ds_block_reduce_w(double v, double *wsum) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) wsum[threadIdx.x >> 5] = v;
    __syncthreads();
    double r = 0.0;
    for (int w = 0; w < kDsThreads / 32; w++) r += wsum[w];
    return r;
}

constexpr int kDsOutCols = kDsT / 2;             // column pairs of a tile
constexpr int kDsOutRows = 2;                    // output rows per thread
static_assert(kDsThreads == kDsOutCols * (kDsT / kDsOutRows), "one 2 x 2 output block per thread");

// dynamic shared memory: A (2 planes of 36^2: the blur inputs x and y, for
// a and b the second pre-blur), B (5 planes of 34^2: the first blurs, and the
// first a/b pre-blur), R (the raw region being fetched: 2 planes of up to
// 40^2), four 1s (the b rows of the x and y planes in ds_stat_blur)
constexpr int kDsSmemFloats = 2 * kDsX * kDsX + 5 * kDsB * kDsB + 2 * kDsR * kDsR + 4;
constexpr int kDsBlocks = 4;  // resident blocks per SM (46 KB shared, at most 64 registers)

__global__ void __launch_bounds__(kDsThreads, kDsBlocks) dssim_tile_kernel(const DsPair *__restrict__ pairs,
                                                                   const DsSeg *__restrict__ segs, int nseg,
                                                                   int ntiles, double *__restrict__ partials,
                                                                   float negz) {
    extern __shared__ __align__(16) float ds_smem[];
    // (-0, -0): the addend that makes the squares of the blurred means packed
    // FMAs (k w + (-0) rounds exactly as k w, signed zeros included), which the
    // compiler, not knowing the argument, cannot turn into a multiply fused
    // with the packed add that follows (a packed multiply feeding a packed add
    // is fused even under -fmad=false)
    const float2 nz = make_float2(negz, negz);
    float *const bufA = ds_smem;
    float *const bufB = bufA + 2 * kDsX * kDsX;
    float *const bufR = bufB + 5 * kDsB * kDsB;
    float *const ones = bufR + 2 * kDsR * kDsR;
    __shared__ double wsum[kDsThreads / 32];
    static_assert(2 * kDsP * kDsP <= 5 * kDsB * kDsB, "buffer reuse");
    static_assert((2 * kDsX * kDsX) % 4 == 0 && (5 * kDsB * kDsB) % 4 == 0 && (2 * kDsR * kDsR) % 4 == 0,
                  "16-byte aligned buffers");
    if (threadIdx.x < 4) ones[threadIdx.x] = 1.0f;  // first read after the loop's first barrier
    const int t = threadIdx.x;
    const int c0 = 2 * (t % kDsOutCols), r0 = (t / kDsOutCols) * kDsOutRows;
    constexpr int nnX = kDsX * kDsX, nnB = kDsB * kDsB;
    if ((int)blockIdx.x < ntiles) ds_prefetch(pairs, segs, nseg, blockIdx.x, 0, bufR);
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const DsSeg sg = segs[ds_find_seg(segs, nseg, tile)];
        const DsPair &P = pairs[sg.pair];
        const int s = sg.level;
        const int W = P.w[s], H = P.h[s];
        const long long pitch = P.pitch[s];
        const int tl = tile - sg.first_tile;
        const int X0 = (tl % sg.tiles_x) * kDsT, Y0 = (tl / sg.tiles_x) * kDsT;
        // the tile's halo reaches outside the level: stage values there are fixed up
        const bool edge = X0 == 0 || Y0 == 0 || X0 + kDsT + 4 > W || Y0 + kDsT + 4 > H;
        // per output (2 rows x 2 columns): sums over L, a, b of mu1^2, mu2^2,
        // mu1 mu2, blur(x^2), blur(y^2), blur(xy), added in channel order as
        // ssim.rs:208-215 does
        float2 acc[kDsOutRows][6];
#pragma unroll 1
        for (int c = 0; c < 3; c++) {
            // channel c's raw region has landed in R; the previous channel's
            // readers of A and B are done
            asm volatile("cp.async.wait_group 0;\n" ::: "memory");
            __syncthreads();
            if (c == 0) {
                // L: the blur input is the plane itself (halo 2, clamped loads)
                ds_copy2(bufR, bufA, nnX);
                __syncthreads();
            } else {
                // a, b: pre-blurred twice first (lib.rs:296-316)
                ds_stage_blur<kDsP, 2, kDsPre1S, kDsPre1L>(bufR, bufB, nz);
                __syncthreads();
            }
            // R is free: fetch the next channel (or the next tile's L) during
            // this channel's blurs
            if (c < 2) ds_prefetch(pairs, segs, nseg, tile, c + 1, bufR);
            else if (tile + (int)gridDim.x < ntiles) ds_prefetch(pairs, segs, nseg, tile + gridDim.x, 0, bufR);
            if (c > 0) {
                if (edge) {
                    ds_fix_edges<kDsP, 3>(bufB, 2, X0, Y0, W, H);
                    __syncthreads();
                }
                ds_stage_blur<kDsX, 2, kDsPre2S, kDsPre2L>(bufB, bufA, nz);
                __syncthreads();
                if (edge) {
                    ds_fix_edges<kDsX, 2>(bufA, 2, X0, Y0, W, H);
                    __syncthreads();
                }
            }
            ds_stat_blur<kDsStatS, kDsStatL>(bufA, ones, bufB, nz);
            __syncthreads();
            if (edge) {
                ds_fix_edges<kDsB, 1>(bufB, 5, X0, Y0, W, H);
                __syncthreads();
            }
            // second blurs at the thread's 2 x 2 outputs
            float2 q[5][kDsOutRows];
#pragma unroll
            for (int pl = 0; pl < 5; pl++) {
                ds_blur_run<kDsOutRows, kDsB>(bufB + pl * nnB + r0 * kDsB + c0, nz,
                                              [&](int r, float2 v) { q[pl][r] = v; });
            }
#pragma unroll
            for (int r = 0; r < kDsOutRows; r++) {
                const float2 m1 = q[0][r], m2 = q[1][r];
                const float2 a0 = __ffma2_rn(m1, m1, nz);
                const float2 a1 = __ffma2_rn(m2, m2, nz);
                const float2 a2 = __ffma2_rn(m1, m2, nz);
                if (c == 0) {
                    acc[r][0] = a0, acc[r][1] = a1, acc[r][2] = a2;
                    acc[r][3] = q[2][r], acc[r][4] = q[3][r], acc[r][5] = q[4][r];
                } else {
                    acc[r][0] = __fadd2_rn(acc[r][0], a0);
                    acc[r][1] = __fadd2_rn(acc[r][1], a1);
                    acc[r][2] = __fadd2_rn(acc[r][2], a2);
                    acc[r][3] = __fadd2_rn(acc[r][3], q[2][r]);
                    acc[r][4] = __fadd2_rn(acc[r][4], q[3][r]);
                    acc[r][5] = __fadd2_rn(acc[r][5], q[4][r]);
                }
            }
        }
        // SSIM (ssim.rs:208-233), stored to the map and summed for the tile
        const float third = 1.0f / 3.0f, c1 = 0.0001f, c2 = 0.0009f;
        float *map = P.map[s];
        double tsum = 0.0;
#pragma unroll
        for (int r = 0; r < kDsOutRows; r++)
#pragma unroll
            for (int l = 0; l < 2; l++) {
                const int ox = X0 + c0 + l, oy = Y0 + r0 + r;
                if (ox >= W || oy >= H) continue;
                const float *a = (const float *)acc[r];
                const float mu1_sq = a[0 * 2 + l] * third, mu2_sq = a[1 * 2 + l] * third;
                const float mu1_mu2 = a[2 * 2 + l] * third;
                const float sigma1_sq = a[3 * 2 + l] * third - mu1_sq;
                const float sigma2_sq = a[4 * 2 + l] * third - mu2_sq;
                const float sigma12 = a[5 * 2 + l] * third - mu1_mu2;
                const float num = fmaf(2.0f, mu1_mu2, c1) * fmaf(2.0f, sigma12, c2);
                const float den = (mu1_sq + mu2_sq + c1) * (sigma1_sq + sigma2_sq + c2);
                const float val = num / den;
                map[oy * pitch + ox] = val;
                tsum += (double)val;
            }
        const double r = ds_block_reduce_w(tsum, wsum);
        if (t == 0) partials[tile] = r;
    }
}

// per (pair, level): mean SSIM and avg = max(mean, 0)^(0.5^s) as f32
// (lib.rs:404-411; the reference casts avg to f32 for the |avg - ssim| pass)
__global__ void __launch_bounds__(kDsThreads) dssim_mean_kernel(const DsPair *__restrict__ pairs,
                                                                const double *__restrict__ partials,
                                                                float *__restrict__ avg) {
    __shared__ double red[kDsThreads];
    const int p = blockIdx.x / kDsLevels, s = blockIdx.x % kDsLevels;
    const DsPair &P = pairs[p];
    if (P.status != 0) return;
    const double sum = ds_block_sum(partials + P.tile_base[s], P.tile_cnt[s], red);
    if (threadIdx.x == 0) {
        const double mean = sum / ((double)P.w[s] * (double)P.h[s]);
        avg[p * kDsLevels + s] = (float)pow(mean > 0.0 ? mean : 0.0, ldexp(1.0, -s));
    }
}

// One warp per tile: lane l sums |avg - ssim| down column l of the tile in
// row order (f64), then the warp adds the lanes by a fixed shuffle tree.  No
// block barriers, and each lane has its column's rows in flight at once.
constexpr int kMadWarps = kDsThreads / 32;
static_assert(kDsT == 32, "one lane per tile column");

__global__ void __launch_bounds__(kDsThreads) dssim_mad_kernel(const DsPair *__restrict__ pairs,
                                                               const DsSeg *__restrict__ segs, int nseg, int ntiles,
                                                               const float *__restrict__ avg,
                                                               double *__restrict__ mad) {
    const int lane = threadIdx.x & 31;
    const int nwarps = gridDim.x * kMadWarps;
    for (int tile = blockIdx.x * kMadWarps + (threadIdx.x >> 5); tile < ntiles; tile += nwarps) {
        const DsSeg sg = segs[ds_find_seg(segs, nseg, tile)];
        const DsPair &P = pairs[sg.pair];
        const int s = sg.level;
        const int tl = tile - sg.first_tile;
        const int X0 = (tl % sg.tiles_x) * kDsT, Y0 = (tl / sg.tiles_x) * kDsT;
        const float a = avg[sg.pair * kDsLevels + s];
        const long long pitch = P.pitch[s];
        const int ox = X0 + lane;
        const int rows = min(kDsT, P.h[s] - Y0);
        double acc = 0.0;
        if (ox < P.w[s]) {
            const float *col = P.map[s] + (long long)Y0 * pitch + ox;
            if (rows == kDsT) {
                float v[kDsT];
#pragma unroll
                for (int k = 0; k < kDsT; k++) v[k] = col[k * pitch];
#pragma unroll
                for (int k = 0; k < kDsT; k++) acc += (double)fabsf(a - v[k]);
            } else {
                for (int k = 0; k < rows; k++) acc += (double)fabsf(a - col[k * pitch]);
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
        if (lane == 0) mad[tile] = acc;
    }
}

__global__ void __launch_bounds__(kDsThreads) dssim_final_kernel(const DsPair *__restrict__ pairs,
                                                                 const double *__restrict__ mad,
                                                                 DevResult *__restrict__ out, int write_all) {
    __shared__ double red[kDsThreads];
    const int p = blockIdx.x;
    const DsPair &P = pairs[p];
    const double nan = __longlong_as_double(0x7ff8000000000000LL);
    if (write_all) {
        for (int i = threadIdx.x; i < 108; i += kDsThreads) out[p].stats[i] = 0.0, out[p].sums[i] = 0.0;
        if (threadIdx.x == 0) {
            out[p].score = nan;
            out[p].n_scales = 0;
            out[p].status = P.status;
        }
    }
    if (P.status != 0) {
        if (threadIdx.x == 0) {
            out[p].dssim = nan;
            for (int s = 0; s < kDsLevels; s++) out[p].dssim_scale[s] = nan;
        }
        return;
    }
    // dssim-cuda/src/lib.rs:77 and :320-333
    const double weights[kDsLevels] = {0.028, 0.197, 0.322, 0.298, 0.155};
    double wsum = 0.0, wtot = 0.0;
    for (int s = 0; s < kDsLevels; s++) {
        const double m = ds_block_sum(mad + P.tile_base[s], P.tile_cnt[s], red);
        const double score = 1.0 - m / ((double)P.w[s] * (double)P.h[s]);
        if (threadIdx.x == 0) out[p].dssim_scale[s] = score;
        wsum += score * weights[s];
        wtot += weights[s];
    }
    if (threadIdx.x == 0) {
        const double ssim = wsum / wtot;
        out[p].dssim = 1.0 / (ssim > DBL_EPSILON ? ssim : DBL_EPSILON) - 1.0;
    }
}

cudaError_t configure_dssim_kernels() {
    return cudaFuncSetAttribute(dssim_tile_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)(kDsSmemFloats * sizeof(float)));
}

cudaError_t launch_dssim(const DsPair *pairs, int npairs, const DsSeg *segs, int nseg, int ntiles, bool clamp,
                         double *partials, float *avg, DevResult *out, bool write_all, int num_sms,
                         cudaStream_t st) {
    if (npairs <= 0) return cudaSuccess;
    if (clamp) dssim_clamp_kernel<<<npairs, kDsThreads, 0, st>>>(pairs);
    if (ntiles > 0) {
        // persistent: the resident blocks of the tile kernel (4 per SM), each
        // striding over the tiles
        const int grid = ntiles < num_sms * kDsBlocks ? ntiles : num_sms * kDsBlocks;
        dssim_tile_kernel<<<grid, kDsThreads, kDsSmemFloats * sizeof(float), st>>>(pairs, segs, nseg, ntiles,
                                                                                  partials, -0.0f);
        dssim_mean_kernel<<<npairs * kDsLevels, kDsThreads, 0, st>>>(pairs, partials, avg);
        const int mgrid = (ntiles + kMadWarps - 1) / kMadWarps < num_sms * 8 ? (ntiles + kMadWarps - 1) / kMadWarps
                                                                               : num_sms * 8;
        dssim_mad_kernel<<<mgrid, kDsThreads, 0, st>>>(pairs, segs, nseg, ntiles, avg, partials + ntiles);
    }
    dssim_final_kernel<<<npairs, kDsThreads, 0, st>>>(pairs, partials + ntiles, out, write_all ? 1 : 0);
    return cudaGetLastError();
}

}  // namespace s2
