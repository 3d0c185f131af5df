// ssim2_kernels.cu -- sm_100a kernels of the B200 SSIMULACRA2 engine.
//
// One pair (or a batch of pairs of any sizes) is scored by three launches:
//
//   pyramid_kernel   reads each pair's scale-0 input once (any input format,
//                    converted to linear RGB on the fly) and writes the 2x2
//                    box pyramid levels 1..5 (planar, f32/f16/bf16).
//                    (ssimulacra2-cuda-kernel/src/downscale.rs:4-35)
//   fused_kernel     persistent; each work item is a tile of 120 columns x
//                    `strip_rows` rows at one scale of one pair.  Walking down
//                    the tile it converts to XYB, forms the five blurred
//                    inputs of each channel on block-shifted values, runs the
//                    vertical 9-tap FIR in registers, then every 9 rows the
//                    horizontal FIR, the SSIM / artifact / detail-loss maps and
//                    their L1/L4 sums from shared memory.  Only the 18 pooled
//                    sums of the tile leave the SM.
//                    (srgb.rs, xyb.rs, blur.rs, error_maps.rs, lib.rs:862-1016)
//   finalize_kernel  per pair: fixed-order f64 reduction of the tile sums,
//                    the 108 statistics and the score (lib.rs:1018-1192).
//
// The blur is the exact closed form of the reference's recursive Gaussian:
// the truncated-cosine recursion of blur.rs equals, in exact arithmetic, a
// symmetric 9-tap FIR with zero padding.  Moments are taken of values shifted
// by one reference XYB sample per (120-column, 64-row) block, which removes
// most of the f32 cancellation in sigma - mu^2; the shift is undone
// algebraically (including at image borders, where the blur of a constant is
// not the constant).
#include "ssim2_device.cuh"

namespace s2 {

// Shared memory layout of fused_kernel (floats).
constexpr int kSmLin = 2 * 3 * kCols;                 // pre-linear exchange
constexpr int kSmOp = 2 * 3 * kCols;                  // opsin cube-root exchange
constexpr int kSmVo = kRowsPerBlk * 3 * 5 * kCols;    // vertical FIR outputs
constexpr int kSmXo = kRowsPerBlk * 3 * 2 * kCols;    // shifted raw XYB of output rows
constexpr int kSmLut = 256;
constexpr int kFusedSmemFloats = kSmLin + kSmOp + kSmVo + kSmXo + kSmLut;
constexpr int kFusedThreads = kCols * 3;

__device__ __forceinline__ float fir9(float a0, float a1, float a2, float a3, float a4, float a5,
                                      float a6, float a7, float a8) {
    float acc = S2_T4 * (a0 + a8);
    acc = fmaf(S2_T3, a1 + a7, acc);
    acc = fmaf(S2_T2, a2 + a6, acc);
    acc = fmaf(S2_T1, a3 + a5, acc);
    return fmaf(S2_T0, a4, acc);
}

// Linear value of channel g at (x, y) of scale s (inside the image).
template <typename ST>
__device__ __forceinline__ float load_pre(const DevPair &P, int img, int s, int x, int y, int g,
                                          const float *lut, const ColorConsts &cc) {
    if (s == 0) return pre_lin0(P, img, x, y, g, lut, cc);
    const ST *pl = (const ST *)P.lvl[img][s] + (long long)g * P.lp[s] * P.h[s];
    return ld_store<ST>(pl + (long long)y * P.lp[s] + x);
}

// Full linear RGB of a pixel (used for the shift anchor).
template <typename ST>
__device__ void load_lin3(const DevPair &P, int img, int s, int x, int y, const float *lut,
                          const ColorConsts &cc, float out[3]) {
    float p0 = load_pre<ST>(P, img, s, x, y, 0, lut, cc);
    float p1 = load_pre<ST>(P, img, s, x, y, 1, lut, cc);
    float p2 = load_pre<ST>(P, img, s, x, y, 2, lut, cc);
    int fmt = s == 0 ? P.fmt : FMT_LINEAR_F32;
    for (int g = 0; g < 3; g++) out[g] = fin_lin0(fmt, g, p0, p1, p2, cc);
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
// pyramid
// ---------------------------------------------------------------------------
template <typename ST>
__global__ void __launch_bounds__(256) pyramid_kernel(const DevPair *__restrict__ pairs, int npairs,
                                                      const int *__restrict__ blk_first,
                                                      int total_blocks, ColorConsts cc,
                                                      const float *__restrict__ lut_g) {
    __shared__ float l0[2][3][kPyrBlk * kPyrBlk];                  // level-0 block [img][ch][px]
    __shared__ float pp[2][2][3][(kPyrBlk / 2) * (kPyrBlk / 2)];  // levels >= 1, ping-pong
    __shared__ float lut[256];
    for (int i = threadIdx.x; i < 256; i += blockDim.x) lut[i] = lut_g[i];
    __syncthreads();
    for (int item = blockIdx.x; item < total_blocks; item += gridDim.x) {
        int lo = 0, hi = npairs - 1;
        while (lo < hi) {
            int mid = (lo + hi + 1) >> 1;
            if (blk_first[mid] <= item) lo = mid;
            else hi = mid - 1;
        }
        const DevPair &P = pairs[lo];
        const int b = item - blk_first[lo];
        const int bx = b % P.blk_x, by = b / P.blk_x;
        const int X0 = bx * kPyrBlk, Y0 = by * kPyrBlk;
        for (int i = threadIdx.x; i < kPyrBlk * kPyrBlk; i += blockDim.x) {
            const int x = X0 + i % kPyrBlk, y = Y0 + i / kPyrBlk;
            for (int img = 0; img < 2; img++) {
                float v[3] = {0.f, 0.f, 0.f};
                if (x < P.w[0] && y < P.h[0]) load_lin3<ST>(P, img, 0, x, y, lut, cc, v);
                for (int c = 0; c < 3; c++) l0[img][c][i] = v[c];
            }
        }
        __syncthreads();
        for (int s = 1; s < P.nscales; s++) {
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
                    ST *dst = (ST *)P.lvl[img][s];
                    for (int c = 0; c < 3; c++) {
                        const float *src = s == 1 ? l0[img][c] : pp[(s - 1) & 1][img][c];
                        float sum = src[ia + ja] + src[ia + jb];
                        sum = sum + src[ib + ja];
                        sum = sum + src[ib + jb];
                        const float v = sum * 0.25f;
                        pp[s & 1][img][c][i] = v;
                        dst[(long long)c * P.lp[s] * P.h[s] + (long long)oy * P.lp[s] + ox] = to_store<ST>(v);
                    }
                }
            }
            __syncthreads();
        }
    }
}

// ---------------------------------------------------------------------------
// fused per-scale tile pass
// ---------------------------------------------------------------------------
template <typename ST>
__global__ void __launch_bounds__(kFusedThreads, 1)
    fused_kernel(const DevPair *__restrict__ pairs, const Seg *__restrict__ segs, int nseg,
                 int total_tiles, int *__restrict__ counter, double *__restrict__ partials,
                 ColorConsts cc, const float *__restrict__ lut_g) {
    extern __shared__ float sm[];
    float *s_lin = sm;                 // [img][g][col]
    float *s_op = s_lin + kSmLin;      // [img][g][col]
    float *s_vo = s_op + kSmOp;        // [row][g][plane][col]
    float *s_xo = s_vo + kSmVo;        // [row][g][2][col]
    float *s_lut = s_xo + kSmXo;
    __shared__ int s_item;
    __shared__ float s_c[3];
    __shared__ double s_red[4][18];

    const int col = threadIdx.x, g = threadIdx.y;
    const int tid = g * kCols + col;
    for (int i = tid; i < 256; i += kFusedThreads) s_lut[i] = lut_g[i];

    for (;;) {
        __syncthreads();
        if (tid == 0) s_item = atomicAdd(counter, 1);
        __syncthreads();
        const int item = s_item;
        if (item >= total_tiles) break;
        const Seg sg = segs[find_seg(segs, nseg, item)];
        const DevPair &P = pairs[sg.pair];
        const int s = sg.scale;
        const int W = P.w[s], H = P.h[s];
        const int local = item - sg.first_tile;
        const int tx = local % sg.tiles_x, ty = local / sg.tiles_x;
        const int x0 = tx * kTileW, y0 = ty * sg.strip_rows;
        const int y1 = min(y0 + sg.strip_rows, H);
        const int fmt = s == 0 ? P.fmt : FMT_LINEAR_F32;

        if (tid < 3) {
            // shift anchor: reference XYB at the tile's column start, band start
            float l[3];
            load_lin3<ST>(P, 0, s, x0, (y0 / kBand) * kBand, s_lut, cc, l);
            float o0 = opsin_row(0, l[0], l[1], l[2]);
            float o1 = opsin_row(1, l[0], l[1], l[2]);
            float o2 = opsin_row(2, l[0], l[1], l[2]);
            s_c[tid] = xyb_from_opsin(tid, o0, o1, o2);
        }
        // (s_c is read after the first row's barriers)

        const int x = x0 - 4 + col;
        const bool colin = (x >= 0) && (x < W);
        float wx[9], wy[9], wxx[9], wyy[9], wxy[9];
        double acc[6] = {0, 0, 0, 0, 0, 0};

        // Stage 1 for input row y: shifted XYB channel g of ref and dis plus
        // products; returns via the five values.
        auto stage1 = [&](int y, float &vx, float &vy, float &vxx, float &vyy, float &vxy) {
            const bool in = colin && y >= 0 && y < H;
            float pr = 0.f, pd = 0.f;
            if (in) {
                pr = load_pre<ST>(P, 0, s, x, y, g, s_lut, cc);
                pd = load_pre<ST>(P, 1, s, x, y, g, s_lut, cc);
            }
            s_lin[(0 * 3 + g) * kCols + col] = pr;
            s_lin[(1 * 3 + g) * kCols + col] = pd;
            __syncthreads();
            float orr = 0.f, odd = 0.f;
            if (in) {
                float a0 = s_lin[0 * kCols + col], a1 = s_lin[1 * kCols + col], a2 = s_lin[2 * kCols + col];
                float b0 = s_lin[3 * kCols + col], b1 = s_lin[4 * kCols + col], b2 = s_lin[5 * kCols + col];
                float r0 = fin_lin0(fmt, 0, a0, a1, a2, cc), r1 = fin_lin0(fmt, 1, a0, a1, a2, cc),
                      r2 = fin_lin0(fmt, 2, a0, a1, a2, cc);
                float d0 = fin_lin0(fmt, 0, b0, b1, b2, cc), d1 = fin_lin0(fmt, 1, b0, b1, b2, cc),
                      d2 = fin_lin0(fmt, 2, b0, b1, b2, cc);
                orr = opsin_row(g, r0, r1, r2);
                odd = opsin_row(g, d0, d1, d2);
            }
            s_op[(0 * 3 + g) * kCols + col] = orr;
            s_op[(1 * 3 + g) * kCols + col] = odd;
            __syncthreads();
            if (in) {
                float cg = s_c[g];
                float xr = xyb_from_opsin(g, s_op[0 * kCols + col], s_op[1 * kCols + col], s_op[2 * kCols + col]);
                float xd = xyb_from_opsin(g, s_op[3 * kCols + col], s_op[4 * kCols + col], s_op[5 * kCols + col]);
                vx = xr - cg;
                vy = xd - cg;
                vxx = vx * vx;
                vyy = vy * vy;
                vxy = vx * vy;
            } else {
                vx = vy = vxx = vyy = vxy = 0.f;
            }
        };

        // prime the windows with input rows y0-4 .. y0+3 (slots 0..7)
#pragma unroll
        for (int k = 0; k < 8; k++) stage1(y0 - 4 + k, wx[k], wy[k], wxx[k], wyy[k], wxy[k]);

        const int rows_out = y1 - y0;
        for (int r0 = 0; r0 < rows_out; r0 += kRowsPerBlk) {
            const int nr = min(kRowsPerBlk, rows_out - r0);
#pragma unroll
            for (int k = 0; k < kRowsPerBlk; k++) {
                if (k < nr) {
                    const int sl = (8 + k) % 9;  // slot of the new row
                    stage1(y0 + r0 + k + 4, wx[sl], wy[sl], wxx[sl], wyy[sl], wxy[sl]);
                    // window slots, oldest first: (sl+1)%9 ... sl
#define S2_W(a, j) a[(sl + 1 + (j)) % 9]
#define S2_FIR(a) fir9(S2_W(a, 0), S2_W(a, 1), S2_W(a, 2), S2_W(a, 3), S2_W(a, 4), S2_W(a, 5), S2_W(a, 6), S2_W(a, 7), S2_W(a, 8))
                    float *vo = s_vo + (k * 3 + g) * 5 * kCols + col;
                    vo[0 * kCols] = S2_FIR(wx);
                    vo[1 * kCols] = S2_FIR(wy);
                    vo[2 * kCols] = S2_FIR(wxx);
                    vo[3 * kCols] = S2_FIR(wyy);
                    vo[4 * kCols] = S2_FIR(wxy);
                    float *xo = s_xo + (k * 3 + g) * 2 * kCols + col;
                    xo[0] = S2_W(wx, 4);
                    xo[kCols] = S2_W(wy, 4);
#undef S2_FIR
#undef S2_W
                }
            }
            __syncthreads();
            // horizontal FIR + error maps: task = (row, channel g, segment)
            if (col < kRowsPerBlk * kSegs) {
                const int r = col / kSegs, sgi = col % kSegs;
                const int y = y0 + r0 + r;
                const int xs = sgi * kSegW;
                if (r < nr && x0 + xs < W) {
                    const float cv = s_c[g];
                    const float bv = border_gain(y, H);
                    const float *vo = s_vo + (r * 3 + g) * 5 * kCols;
                    const float *xo = s_xo + (r * 3 + g) * 2 * kCols;
#pragma unroll
                    for (int half = 0; half < 2; half++) {
                        const int c0 = xs + half * 5;  // first output (tile coords)
                        float o[5][5];
#pragma unroll
                        for (int p = 0; p < 5; p++) {
                            float v[13];
#pragma unroll
                            for (int j = 0; j < 13; j++) v[j] = vo[p * kCols + c0 + j];
#pragma unroll
                            for (int j = 0; j < 5; j++)
                                o[p][j] = fir9(v[j], v[j + 1], v[j + 2], v[j + 3], v[j + 4], v[j + 5], v[j + 6], v[j + 7], v[j + 8]);
                        }
                        float fs[3] = {0.f, 0.f, 0.f}, f4[3] = {0.f, 0.f, 0.f};
#pragma unroll
                        for (int j = 0; j < 5; j++) {
                            const int xx = x0 + c0 + j;
                            if (xx < W) {
                                const float m1 = o[0][j], m2 = o[1][j], s11 = o[2][j], s22 = o[3][j], s12 = o[4][j];
                                const float xp = xo[c0 + j + 4], yp = xo[kCols + c0 + j + 4];
                                const float bh = border_gain(xx, W);
                                const float corr = (float)(1.0 - (double)bh * (double)bv);
                                const float kk = cv * corr;
                                const float e = cv - kk;
                                const float v1 = fmaf(kk, fmaf(2.0f, m1, e), fmaf(-m1, m1, s11));
                                const float v2 = fmaf(kk, fmaf(2.0f, m2, e), fmaf(-m2, m2, s22));
                                const float cov = fmaf(kk, (m1 + m2) + e, fmaf(-m1, m2, s12));
                                const float md = m1 - m2;
                                const float num_m = fmaf(-md, md, 1.0f);
                                const float num_s = fmaf(2.0f, cov, kC2);
                                const float den = (v1 + v2) + kC2;
                                float d = fmaf(-num_m, num_s, den) / den;
                                d = fmaxf(d, 0.0f);
                                const float aa = fabsf((xp - m1) + kk);
                                const float bb = fabsf((yp - m2) + kk);
                                const float d1 = (bb - aa) / (1.0f + aa);
                                const float art = fmaxf(d1, 0.0f), det = fmaxf(-d1, 0.0f);
                                float q;
                                fs[0] += d;   q = d * d;     f4[0] += q * q;
                                fs[1] += art; q = art * art; f4[1] += q * q;
                                fs[2] += det; q = det * det; f4[2] += q * q;
                            }
                        }
#pragma unroll
                        for (int m = 0; m < 3; m++) {
                            acc[m] += (double)fs[m];
                            acc[3 + m] += (double)f4[m];
                        }
                    }
                }
            }
            __syncthreads();
        }

        // tile reduction: per channel g, warps g*4 .. g*4+3
#pragma unroll
        for (int m = 0; m < 6; m++) {
            double v = acc[m];
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
            acc[m] = v;
        }
        const int lane = col & 31, wg = col >> 5;  // warp within channel group
        if (lane == 0) {
#pragma unroll
            for (int m = 0; m < 6; m++) s_red[wg][g * 6 + m] = acc[m];
        }
        __syncthreads();
        if (tid < 18) {
            double v = ((s_red[0][tid] + s_red[1][tid]) + s_red[2][tid]) + s_red[3][tid];
            partials[(long long)item * 18 + tid] = v;
        }
    }
}

// ---------------------------------------------------------------------------
// finalize: tile sums -> 108 statistics -> score
// ---------------------------------------------------------------------------
__constant__ double c_weight[108];

__global__ void __launch_bounds__(128) finalize_kernel(const DevPair *__restrict__ pairs, int npairs,
                                                       const double *__restrict__ partials,
                                                       DevResult *__restrict__ out) {
    __shared__ double st[108];
    const int p = blockIdx.x;
    const DevPair &P = pairs[p];
    const int t = threadIdx.x;
    if (t < 108) {
        const int c = t / 36, s = (t % 36) / 6, k = t % 6;
        double sum = 0.0, v = 0.0;
        if (P.status == 0 && s < P.nscales) {
            const int base = P.tile_base[s], cnt = P.tile_cnt[s];
            for (int i = 0; i < cnt; i++) sum += partials[(long long)(base + i) * 18 + c * 6 + k];
            const double inv = 1.0 / ((double)P.w[s] * (double)P.h[s]);
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

template <typename ST> static const void *fused_fn() { return (const void *)fused_kernel<ST>; }

cudaError_t configure_kernels() {
    cudaError_t e;
    e = cudaFuncSetAttribute(fused_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fused_smem_bytes());
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(fused_kernel<__half>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fused_smem_bytes());
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(fused_kernel<__nv_bfloat16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fused_smem_bytes());
    return e;
}

int fused_blocks_per_sm(int storage) {
    int n = 0;
    const void *f = storage == ST_F16 ? fused_fn<__half>() : storage == ST_BF16 ? fused_fn<__nv_bfloat16>() : fused_fn<float>();
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, f, kFusedThreads, fused_smem_bytes()) != cudaSuccess) return 1;
    return n > 0 ? n : 1;
}

cudaError_t launch_pyramid(int storage, const DevPair *pairs, int npairs, const int *blk_first,
                           int total_blocks, const ColorConsts &cc, const float *lut, int grid,
                           cudaStream_t st) {
    if (total_blocks <= 0) return cudaSuccess;
    grid = grid > total_blocks ? total_blocks : grid;
    if (storage == ST_F16)
        pyramid_kernel<__half><<<grid, 256, 0, st>>>(pairs, npairs, blk_first, total_blocks, cc, lut);
    else if (storage == ST_BF16)
        pyramid_kernel<__nv_bfloat16><<<grid, 256, 0, st>>>(pairs, npairs, blk_first, total_blocks, cc, lut);
    else
        pyramid_kernel<float><<<grid, 256, 0, st>>>(pairs, npairs, blk_first, total_blocks, cc, lut);
    return cudaGetLastError();
}

cudaError_t launch_fused(int storage, const DevPair *pairs, const Seg *segs, int nseg, int total_tiles,
                         int *counter, double *partials, const ColorConsts &cc, const float *lut,
                         int grid, cudaStream_t st) {
    if (total_tiles <= 0) return cudaSuccess;
    grid = grid > total_tiles ? total_tiles : grid;
    dim3 block(kCols, 3);
    size_t sm = fused_smem_bytes();
    if (storage == ST_F16)
        fused_kernel<__half><<<grid, block, sm, st>>>(pairs, segs, nseg, total_tiles, counter, partials, cc, lut);
    else if (storage == ST_BF16)
        fused_kernel<__nv_bfloat16><<<grid, block, sm, st>>>(pairs, segs, nseg, total_tiles, counter, partials, cc, lut);
    else
        fused_kernel<float><<<grid, block, sm, st>>>(pairs, segs, nseg, total_tiles, counter, partials, cc, lut);
    return cudaGetLastError();
}

cudaError_t launch_finalize(const DevPair *pairs, int npairs, const double *partials, DevResult *out,
                            cudaStream_t st) {
    if (npairs <= 0) return cudaSuccess;
    finalize_kernel<<<npairs, 128, 0, st>>>(pairs, npairs, partials, out);
    return cudaGetLastError();
}

}  // namespace s2
