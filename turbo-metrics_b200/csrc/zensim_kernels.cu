// zensim_kernels.cu -- the zensim feature extraction of crates/zensim-cuda on
// sm_100a: positive XYB at the SIMD-padded width, a 4-scale box pyramid of
// the padded planes, and per (scale, channel) the radius-5 box blurs and the
// 17 pooled sums + 3 maxima from which the host forms the 228 features.
//
//   zs_xyb_kernel   one thread per pixel of the padded scale-0 plane: sRGB8
//                   through the reference table, opsin mix, the Halley cube
//                   root of cbrtf_fast, positive XYB (color.rs:70-149);
//                   padding columns take the XYB of their mirror column
//                   (lib.rs:236-252, pad.rs)
//   zs_down_kernel  2x2 box mean of the padded planes, source clamped at
//                   the far edge (downscale.rs:21-43)
//   zs_feat_kernel  one block per (scale, channel, 64-column strip); thread
//                   = one column, walking all rows: the horizontal box sums
//                   of its column (blur.rs:40-96) go to a per-thread ring of
//                   16 rows in shared memory, from which the vertical running
//                   sums (features.rs:83-193) are slid; per pixel the SSIM,
//                   edge, high-frequency and MSE terms (features.rs:102-176)
//                   are added to 17 f64 sums and 3 maxima.  The block's sums
//                   are reduced in a fixed order (lanes by a shuffle tree,
//                   warps in order) -- where the reference adds each column
//                   with a float atomic -- so results do not depend on
//                   scheduling.
//
// Compiled with -fmad=false: every fused multiply-add is explicit (fmaf where
// the reference uses mul_add), divisions are IEEE (__fdiv_rn).
#include <cuda_runtime.h>
#include <stdint.h>

#include "zensim_kernels.h"

namespace zs {

__constant__ float c_lut[256];

__device__ __forceinline__ int mirror(int i, int n) {
    if (n <= 1) return 0;
    const int period = 2 * (n - 1);
    const int m = ((i % period) + period) % period;
    return m < n ? m : period - m;
}

// cbrtf_fast (color.rs:70-91): bit seed, two Halley steps
__device__ __forceinline__ float cbrt_fast(float x) {
    if (x == 0.0f) return 0.0f;
    const unsigned ui = __float_as_uint(x);
    const unsigned hx = (ui & 0x7fffffffu) / 3u + 709958130u;
    float t = __uint_as_float((ui & 0x80000000u) | hx);
    float r = t * t * t;
    t = t * __fdiv_rn(fmaf(x, 2.0f, r), fmaf(r, 2.0f, x));
    r = t * t * t;
    t = t * __fdiv_rn(fmaf(x, 2.0f, r), fmaf(r, 2.0f, x));
    return t;
}

__device__ __forceinline__ void positive_xyb(const uint8_t *px, float o[3]) {
    const float M02 = 0.078f, M00 = 0.30f, M01 = 1.0f - M02 - M00;
    const float M12 = 0.078f, M10 = 0.23f, M11 = 1.0f - M12 - M10;
    const float M20 = 0.24342269f, M21 = 0.20476745f, M22 = 1.0f - M20 - M21;
    const float B0 = 0.0037930734f;
    const float r = c_lut[px[0]], g = c_lut[px[1]], b = c_lut[px[2]];
    const float m0 = fmaxf(fmaf(M00, r, fmaf(M01, g, fmaf(M02, b, B0))), 0.0f);
    const float m1 = fmaxf(fmaf(M10, r, fmaf(M11, g, fmaf(M12, b, B0))), 0.0f);
    const float m2 = fmaxf(fmaf(M20, r, fmaf(M21, g, fmaf(M22, b, B0))), 0.0f);
    const float bias = -cbrt_fast(B0);
    const float c0 = cbrt_fast(m0) + bias, c1 = cbrt_fast(m1) + bias, c2 = cbrt_fast(m2);
    const float xv = 0.5f * (c0 - c1), yv = 0.5f * (c0 + c1), bv = c2 - yv;
    o[0] = fmaf(xv, 14.0f, 0.42f);
    o[1] = yv + 0.01f;
    o[2] = bv + 0.55f;
}

__global__ void __launch_bounds__(256) zs_xyb_kernel(const uint8_t *__restrict__ img, size_t pitch, int w, int h,
                                                     ZsPlanes out) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= out.n || y >= h) return;
    const int sx = x < w ? x : mirror(x, w);
    float o[3];
    positive_xyb(img + (size_t)y * pitch + 3 * (size_t)sx, o);
#pragma unroll
    for (int c = 0; c < 3; c++) out.p[c][(size_t)y * out.pitch + x] = o[c];
}

__global__ void __launch_bounds__(256) zs_down_kernel(ZsPlanes src, int src_h, ZsPlanes dst, int dst_h) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= dst.n || y >= dst_h) return;
    const int x0 = 2 * x, y0 = 2 * y;
    const int x1 = x0 + 1 < src.n ? x0 + 1 : x0, y1 = y0 + 1 < src_h ? y0 + 1 : y0;
#pragma unroll
    for (int c = 0; c < 3; c++) {
        const float *s = src.p[c];
        float v = s[(size_t)y0 * src.pitch + x0] + s[(size_t)y0 * src.pitch + x1];
        v = v + s[(size_t)y1 * src.pitch + x0];
        v = v + s[(size_t)y1 * src.pitch + x1];
        dst.p[c][(size_t)y * dst.pitch + x] = v * 0.25f;
    }
}

constexpr int kRing = 16;  // rows of horizontal sums kept per column (>= 2 * 5 + 2 + the bottom mirror reach)

// One work item: (scale, channel, strip of kZsCols columns).
__global__ void __launch_bounds__(kZsCols) zs_feat_kernel(const ZsScale *__restrict__ scales,
                                                          const ZsItem *__restrict__ items,
                                                          double *__restrict__ out) {
    __shared__ float ring[kRing][4][kZsCols];
    __shared__ double s_warp[kZsCols / 32][kZsOut];
    const ZsItem it = items[blockIdx.x];
    const ZsScale &S = scales[it.scale];
    const int n = S.n, h = S.h, tid = threadIdx.x;
    const int x = it.x0 + tid;
    const bool on = x < n;
    const float *A = S.ref.p[it.ch], *D = S.dis.p[it.ch];
    const size_t pitch = S.ref.pitch;
    const int diam = 2 * kZsRadius + 1;
    const float inv = 1.0f / (float)diam;
    double acc[kZsOut];
#pragma unroll
    for (int i = 0; i < kZsOut; i++) acc[i] = 0.0;
    if (on) {
        // columns whose 11 taps stay inside the row need no mirror index
        const bool xin = x >= kZsRadius && x + kZsRadius < n;
        int done = -1;  // horizontal sums computed for rows 0 .. done
        auto ensure = [&](int row) {
            while (done < row) {
                ++done;
                float s1 = 0.0f, s2 = 0.0f, sq = 0.0f, s12 = 0.0f;
                const float *a = A + (size_t)done * pitch, *d = D + (size_t)done * pitch;
                for (int k = 0; k < diam; k++) {
                    const int ix = xin ? x + k - kZsRadius : mirror(x + k - kZsRadius, n);
                    const float s = a[ix], t = d[ix];
                    s1 += s;
                    s2 += t;
                    sq = sq + s * s + t * t;
                    s12 = s12 + s * t;
                }
                float *rr = &ring[done % kRing][0][tid];
                rr[0] = s1 * inv;
                rr[kZsCols] = s2 * inv;
                rr[2 * kZsCols] = sq * inv;
                rr[3 * kZsCols] = s12 * inv;
            }
        };
        auto get = [&](int row, int plane) { return ring[row % kRing][plane][tid]; };
        float sm1 = 0.0f, sm2 = 0.0f, ssq = 0.0f, ss12 = 0.0f;
        for (int k = 0; k < diam; k++) {
            const int r = mirror(k - kZsRadius, h);
            ensure(r);
            sm1 += get(r, 0);
            sm2 += get(r, 1);
            ssq += get(r, 2);
            ss12 += get(r, 3);
        }
        const float C2 = 0.0009f;
        float pk0 = 0.0f, pk1 = 0.0f, pk2 = 0.0f;
        for (int y = 0; y < h; y++) {
            const float mu1 = sm1 * inv, mu2 = sm2 * inv, sq = ssq * inv, s12 = ss12 * inv;
            const float sv = A[(size_t)y * pitch + x], dv = D[(size_t)y * pitch + x];
            const float md = mu1 - mu2;
            const float num_m = fmaf(md, -md, 1.0f);
            const float num_s = fmaf(2.0f, fmaf(-mu1, mu2, s12), C2);
            const float den_s = fmaf(-mu2, mu2, fmaf(-mu1, mu1, sq)) + C2;
            const float sd_raw = 1.0f - __fdiv_rn(num_m * num_s, den_s);
            const float sd = sd_raw > 0.0f ? sd_raw : 0.0f;
            const float sd2 = sd * sd, sd4 = sd2 * sd2;
            acc[0] += (double)sd;
            acc[1] += (double)sd4;
            acc[2] += (double)sd2;
            acc[14] += (double)(sd4 * sd4);
            pk0 = sd > pk0 ? sd : pk0;
            const float d1 = fabsf(sv - mu1), d2 = fabsf(dv - mu2);
            const float ed = __fdiv_rn(1.0f + d2, 1.0f + d1) - 1.0f;
            const float art = ed > 0.0f ? ed : 0.0f, det = ed < 0.0f ? -ed : 0.0f;
            const float a2 = art * art, l2 = det * det, a4 = a2 * a2, l4 = l2 * l2;
            acc[3] += (double)art;
            acc[4] += (double)a4;
            acc[5] += (double)a2;
            acc[6] += (double)det;
            acc[7] += (double)l4;
            acc[8] += (double)l2;
            acc[15] += (double)(a4 * a4);
            acc[16] += (double)(l4 * l4);
            pk1 = art > pk1 ? art : pk1;
            pk2 = det > pk2 ? det : pk2;
            const float vs = sv - mu1, vd = dv - mu2;
            acc[10] += (double)(vs * vs);
            acc[11] += (double)(vd * vd);
            acc[12] += (double)d1;
            acc[13] += (double)d2;
            const float pd = sv - dv;
            acc[9] += (double)(pd * pd);
            // slide the vertical window: (sum + entering row) - leaving row
            const int ai = y + kZsRadius + 1 < h ? y + kZsRadius + 1 : mirror(y + kZsRadius + 1, h);
            const int ri = y >= kZsRadius ? y - kZsRadius : mirror(y - kZsRadius, h);
            ensure(ai);
            sm1 = sm1 + get(ai, 0) - get(ri, 0);
            sm2 = sm2 + get(ai, 1) - get(ri, 1);
            ssq = ssq + get(ai, 2) - get(ri, 2);
            ss12 = ss12 + get(ai, 3) - get(ri, 3);
        }
        acc[17] = (double)pk0;
        acc[18] = (double)pk1;
        acc[19] = (double)pk2;
    }
    // fixed-order block reduction: sums, and maxima for the peaks
#pragma unroll
    for (int i = 0; i < kZsOut; i++) {
        double v = acc[i];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            const double o = __shfl_down_sync(0xffffffffu, v, off);
            v = i < kZsSums ? v + o : fmax(v, o);
        }
        if ((tid & 31) == 0) s_warp[tid >> 5][i] = v;
    }
    __syncthreads();
    if (tid < kZsOut) {
        double v = s_warp[0][tid];
        for (int w = 1; w < kZsCols / 32; w++) v = tid < kZsSums ? v + s_warp[w][tid] : fmax(v, s_warp[w][tid]);
        out[(size_t)blockIdx.x * kZsOut + tid] = v;
    }
}

cudaError_t zs_upload_lut(const float *lut256) { return cudaMemcpyToSymbol(c_lut, lut256, 256 * sizeof(float)); }

cudaError_t zs_launch_xyb(const uint8_t *img, size_t pitch, int w, int h, const ZsPlanes &out, cudaStream_t st) {
    dim3 grid((out.n + 255) / 256, h);
    zs_xyb_kernel<<<grid, 256, 0, st>>>(img, pitch, w, h, out);
    return cudaGetLastError();
}

cudaError_t zs_launch_down(const ZsPlanes &src, int src_h, const ZsPlanes &dst, int dst_h, cudaStream_t st) {
    dim3 grid((dst.n + 255) / 256, dst_h);
    zs_down_kernel<<<grid, 256, 0, st>>>(src, src_h, dst, dst_h);
    return cudaGetLastError();
}

cudaError_t zs_launch_feat(const ZsScale *scales, const ZsItem *items, int nitems, double *out, cudaStream_t st) {
    if (nitems <= 0) return cudaSuccess;
    zs_feat_kernel<<<nitems, kZsCols, 0, st>>>(scales, items, out);
    return cudaGetLastError();
}

}  // namespace zs
