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

#include "ssim2_launch.h"

namespace s2 {

constexpr int kDsT = 32;             // output tile edge
constexpr int kDsThreads = 256;
constexpr int kDsRows = kDsThreads / kDsT;  // rows of outputs per pass (8)
constexpr int kDsR = kDsT + 8;       // raw a/b region (halo 4)
constexpr int kDsP = kDsT + 6;       // first a/b pre-blur (halo 3)
constexpr int kDsX = kDsT + 4;       // blur input x, y (halo 2)
constexpr int kDsB = kDsT + 2;       // first statistics blur (halo 1)
static_assert(2 * kDsX * kDsX <= 2 * kDsR * kDsR && 2 * kDsP * kDsP <= 5 * kDsB * kDsB, "buffer reuse");

// dssim-cuda-kernel/src/blur.rs:13-17
__device__ __forceinline__ float ds_k(int i) {
    return (i == 4) ? 0.146293f : ((i & 1) ? 0.118095f : 0.095332f);
}

// One 3x3 tap sum centred on (ci, cj) of an m-wide buffer.  KIND 0: v * k;
// 1: v * v * k; 2: v * u * k (blur.rs:46-54, :124-132, :160-170).
template <int KIND>
__device__ __forceinline__ float ds_blur_at(const float *in, const float *in2, int m, int ci, int cj) {
    float sum = 0.0f;
#pragma unroll
    for (int ky = 0; ky < 3; ky++)
#pragma unroll
        for (int kx = 0; kx < 3; kx++) {
            const int idx = (cj + ky - 1) * m + ci + kx - 1;
            const float v = in[idx];
            float t;
            if (KIND == 0) t = v * ds_k(ky * 3 + kx);
            else if (KIND == 1) t = v * v * ds_k(ky * 3 + kx);
            else t = v * in2[idx] * ds_k(ky * 3 + kx);
            sum = sum + t;
        }
    return sum;
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
__global__ void __launch_bounds__(kDsThreads, 4) dssim_tile_kernel(const DsPair *__restrict__ pairs,
                                                                   const DsSeg *__restrict__ segs, int nseg,
                                                                   int ntiles, double *__restrict__ partials) {
    __shared__ float bufA[2 * kDsR * kDsR];  // raw a/b, then x and y of the blur input
    __shared__ float bufB[5 * kDsB * kDsB];  // first pre-blur, then the five first blurs
    __shared__ double red[kDsThreads];
    const int t = threadIdx.x;
    const int tx = t % kDsT, ty = t / kDsT;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const DsSeg sg = segs[ds_find_seg(segs, nseg, tile)];
        const DsPair &P = pairs[sg.pair];
        const int s = sg.level;
        const int W = P.w[s], H = P.h[s];
        const long long pitch = P.pitch[s], plane = pitch * H;
        const int tl = tile - sg.first_tile;
        const int X0 = (tl % sg.tiles_x) * kDsT, Y0 = (tl / sg.tiles_x) * kDsT;
        // per output: sums over L, a, b of mu1^2, mu2^2, mu1 mu2, blur(x^2),
        // blur(y^2), blur(xy), added in channel order as ssim.rs:208-215 does
        float acc[kDsT / kDsRows][6];
#pragma unroll 1
        for (int c = 0; c < 3; c++) {
            const float *xr = P.lab[0][s] + c * plane;
            const float *yr = P.lab[1][s] + c * plane;
            __syncthreads();  // the previous channel's readers are done
            if (c == 0) {
                // L: the blur input is the plane itself (halo 2)
                for (int i = t; i < 2 * kDsX * kDsX; i += kDsThreads) {
                    const int img = i / (kDsX * kDsX), r = i % (kDsX * kDsX);
                    const int gx = ds_clamp(X0 - 2 + r % kDsX, W - 1), gy = ds_clamp(Y0 - 2 + r / kDsX, H - 1);
                    bufA[i] = (img ? yr : xr)[gy * pitch + gx];
                }
            } else {
                // a, b: pre-blurred twice first (lib.rs:296-316)
                for (int i = t; i < 2 * kDsR * kDsR; i += kDsThreads) {
                    const int img = i / (kDsR * kDsR), r = i % (kDsR * kDsR);
                    const int gx = ds_clamp(X0 - 4 + r % kDsR, W - 1), gy = ds_clamp(Y0 - 4 + r / kDsR, H - 1);
                    bufA[i] = (img ? yr : xr)[gy * pitch + gx];
                }
                __syncthreads();
                for (int i = t; i < 2 * kDsP * kDsP; i += kDsThreads) {
                    const int img = i / (kDsP * kDsP), r = i % (kDsP * kDsP);
                    const int ci = ds_clamp(X0 - 3 + r % kDsP, W - 1) - (X0 - 4);
                    const int cj = ds_clamp(Y0 - 3 + r / kDsP, H - 1) - (Y0 - 4);
                    bufB[i] = ds_blur_at<0>(bufA + img * kDsR * kDsR, nullptr, kDsR, ci, cj);
                }
                __syncthreads();
                for (int i = t; i < 2 * kDsX * kDsX; i += kDsThreads) {
                    const int img = i / (kDsX * kDsX), r = i % (kDsX * kDsX);
                    const int ci = ds_clamp(X0 - 2 + r % kDsX, W - 1) - (X0 - 3);
                    const int cj = ds_clamp(Y0 - 2 + r / kDsX, H - 1) - (Y0 - 3);
                    bufA[i] = ds_blur_at<0>(bufB + img * kDsP * kDsP, nullptr, kDsP, ci, cj);
                }
            }
            __syncthreads();
            // first blur of x, y, x^2, y^2, xy (halo 1)
            for (int i = t; i < kDsB * kDsB; i += kDsThreads) {
                const int ci = ds_clamp(X0 - 1 + i % kDsB, W - 1) - (X0 - 2);
                const int cj = ds_clamp(Y0 - 1 + i / kDsB, H - 1) - (Y0 - 2);
                const float *X = bufA, *Y = bufA + kDsX * kDsX;
                bufB[i] = ds_blur_at<0>(X, nullptr, kDsX, ci, cj);
                bufB[kDsB * kDsB + i] = ds_blur_at<0>(Y, nullptr, kDsX, ci, cj);
                bufB[2 * kDsB * kDsB + i] = ds_blur_at<1>(X, nullptr, kDsX, ci, cj);
                bufB[3 * kDsB * kDsB + i] = ds_blur_at<1>(Y, nullptr, kDsX, ci, cj);
                bufB[4 * kDsB * kDsB + i] = ds_blur_at<2>(X, Y, kDsX, ci, cj);
            }
            __syncthreads();
            // second blur at the tile's outputs
#pragma unroll
            for (int k = 0; k < kDsT / kDsRows; k++) {
                const int ci = tx + 1, cj = ty + k * kDsRows + 1;
                const float m1 = ds_blur_at<0>(bufB, nullptr, kDsB, ci, cj);
                const float m2 = ds_blur_at<0>(bufB + kDsB * kDsB, nullptr, kDsB, ci, cj);
                const float s1 = ds_blur_at<0>(bufB + 2 * kDsB * kDsB, nullptr, kDsB, ci, cj);
                const float s2 = ds_blur_at<0>(bufB + 3 * kDsB * kDsB, nullptr, kDsB, ci, cj);
                const float s12 = ds_blur_at<0>(bufB + 4 * kDsB * kDsB, nullptr, kDsB, ci, cj);
                if (c == 0) {
                    acc[k][0] = m1 * m1;
                    acc[k][1] = m2 * m2;
                    acc[k][2] = m1 * m2;
                    acc[k][3] = s1;
                    acc[k][4] = s2;
                    acc[k][5] = s12;
                } else {
                    acc[k][0] = acc[k][0] + m1 * m1;
                    acc[k][1] = acc[k][1] + m2 * m2;
                    acc[k][2] = acc[k][2] + m1 * m2;
                    acc[k][3] = acc[k][3] + s1;
                    acc[k][4] = acc[k][4] + s2;
                    acc[k][5] = acc[k][5] + s12;
                }
            }
        }
        // SSIM (ssim.rs:208-233), stored to the map and summed for the tile
        const float third = 1.0f / 3.0f, c1 = 0.0001f, c2 = 0.0009f;
        float *map = P.map[s];
        double tsum = 0.0;
#pragma unroll
        for (int k = 0; k < kDsT / kDsRows; k++) {
            const int ox = X0 + tx, oy = Y0 + ty + k * kDsRows;
            if (ox >= W || oy >= H) continue;
            const float mu1_sq = acc[k][0] * third, mu2_sq = acc[k][1] * third, mu1_mu2 = acc[k][2] * third;
            const float sigma1_sq = acc[k][3] * third - mu1_sq;
            const float sigma2_sq = acc[k][4] * third - mu2_sq;
            const float sigma12 = acc[k][5] * third - mu1_mu2;
            const float num = fmaf(2.0f, mu1_mu2, c1) * fmaf(2.0f, sigma12, c2);
            const float den = (mu1_sq + mu2_sq + c1) * (sigma1_sq + sigma2_sq + c2);
            const float v = num / den;
            map[oy * pitch + ox] = v;
            tsum += (double)v;
        }
        const double r = ds_block_reduce(tsum, red);
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

__global__ void __launch_bounds__(kDsThreads) dssim_mad_kernel(const DsPair *__restrict__ pairs,
                                                               const DsSeg *__restrict__ segs, int nseg, int ntiles,
                                                               const float *__restrict__ avg,
                                                               double *__restrict__ mad) {
    __shared__ double red[kDsThreads];
    const int t = threadIdx.x;
    const int tx = t % kDsT, ty = t / kDsT;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const DsSeg sg = segs[ds_find_seg(segs, nseg, tile)];
        const DsPair &P = pairs[sg.pair];
        const int s = sg.level;
        const int tl = tile - sg.first_tile;
        const int X0 = (tl % sg.tiles_x) * kDsT, Y0 = (tl / sg.tiles_x) * kDsT;
        const float a = avg[sg.pair * kDsLevels + s];
        const float *map = P.map[s];
        const long long pitch = P.pitch[s];
        double acc = 0.0;
#pragma unroll
        for (int k = 0; k < kDsT / kDsRows; k++) {
            const int ox = X0 + tx, oy = Y0 + ty + k * kDsRows;
            if (ox < P.w[s] && oy < P.h[s]) acc += (double)fabsf(a - map[oy * pitch + ox]);
        }
        const double r = ds_block_reduce(acc, red);
        if (t == 0) mad[tile] = r;
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

cudaError_t launch_dssim(const DsPair *pairs, int npairs, const DsSeg *segs, int nseg, int ntiles, bool clamp,
                         double *partials, float *avg, DevResult *out, bool write_all, int num_sms,
                         cudaStream_t st) {
    if (npairs <= 0) return cudaSuccess;
    if (clamp) dssim_clamp_kernel<<<npairs, kDsThreads, 0, st>>>(pairs);
    if (ntiles > 0) {
        const int grid = ntiles < num_sms * 4 ? ntiles : num_sms * 4;
        dssim_tile_kernel<<<grid, kDsThreads, 0, st>>>(pairs, segs, nseg, ntiles, partials);
        dssim_mean_kernel<<<npairs * kDsLevels, kDsThreads, 0, st>>>(pairs, partials, avg);
        dssim_mad_kernel<<<grid, kDsThreads, 0, st>>>(pairs, segs, nseg, ntiles, avg, partials + ntiles);
    }
    dssim_final_kernel<<<npairs, kDsThreads, 0, st>>>(pairs, partials + ntiles, out, write_all ? 1 : 0);
    return cudaGetLastError();
}

}  // namespace s2
