// ssim2_iir.cu -- S2_BLUR_IIR_REF: the reference's own f32 arithmetic.
//
// The default blur of this engine is the exact closed form of the recursive
// Gaussian (a 9-tap FIR), which is far closer to the FP64 result than the
// reference's f32 recursion.  This mode instead reproduces the reference's
// recursion step for step, so that the 108 statistics match the arithmetic
// of crates/ssimulacra2-cuda:
//
//   iir_vertical_kernel    thread per (column, plane) of a (pair, scale): the
//                          walk of ssimulacra2-cuda-kernel/src/blur.rs:95-136
//                          (sum of the entering and leaving samples, three
//                          second-order recursions with the same FMA order,
//                          sum of the three outputs) down the column of one of
//                          the 15 blurred inputs (XYB of ref and dis, their
//                          squares and product, as NPP Mul forms them,
//                          ssimulacra2-cuda/src/lib.rs:868-886).  Output
//                          planes in HBM (the reference's img[3..7]).
//   iir_horizontal_kernel  thread per (row, channel): the same walk along the
//                          row of the five vertical outputs (the reference
//                          transposes and walks down again, lib.rs:911-947 --
//                          identical arithmetic), then the error maps of
//                          error_maps.rs:36-59 as written and the pooling of
//                          lib.rs:986-1016 (f64 sums of d and of the f32
//                          (d*d)*(d*d)); one partial-sum record per row.
//
// The XYB planes come from prep_kernel (same pyramid and XYB arithmetic as the
// reference, with the engine's own cube root); finalize_kernel reduces the row
// records in order.  The translation unit is compiled with -fmad=false: every
// FMA below is explicit, as in the reference (Rust never contracts).
#include "ssim2_device.cuh"
#include "ssim2_launch.h"

namespace s2 {

// f32 recursion constants (ssimulacra2-cuda-kernel/build.rs:28-145 evaluated
// in double and rounded, as printed in examples/cpu.rs:931-948).
#define S2_MUL_IN_1 0x1.c4fa84p-5f
#define S2_MUL_IN_3 -0x1.e1fd7ap-5f
#define S2_MUL_IN_5 0x1.a8894ap-7f
#define S2_MUL_PREV_1 0x1.e6f0e2p+0f
#define S2_MUL_PREV_3 0x1.2cf23p+0f
#define S2_MUL_PREV_5 0x1.1a6264p-53f
#define S2_MUL_PREV2 (-1.0f)

struct IirState {
    float p1, p3, p5, q1, q3, q5;  // prev, prev2
    __device__ __forceinline__ void zero() { p1 = p3 = p5 = q1 = q3 = q5 = 0.f; }
    // one step of blur.rs:95-136; returns out_1 + out_3 + out_5
    __device__ __forceinline__ float step(float sum) {
        float o1 = sum * S2_MUL_IN_1, o3 = sum * S2_MUL_IN_3, o5 = sum * S2_MUL_IN_5;
        o1 = fmaf(S2_MUL_PREV2, q1, o1);
        o3 = fmaf(S2_MUL_PREV2, q3, o3);
        o5 = fmaf(S2_MUL_PREV2, q5, o5);
        q1 = p1;
        q3 = p3;
        q5 = p5;
        o1 = fmaf(S2_MUL_PREV_1, p1, o1);
        o3 = fmaf(S2_MUL_PREV_3, p3, o3);
        o5 = fmaf(S2_MUL_PREV_5, p5, o5);
        p1 = o1;
        p3 = o3;
        p5 = o5;
        return (o1 + o3) + o5;
    }
};

constexpr int kN = 5;  // radius of the recursion

__device__ __forceinline__ int find_iseg(const IirSeg *segs, int nseg, int t) {
    int lo = 0, hi = nseg - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (segs[mid].first <= t) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// Input sample of blurred plane p (0..4 = x, y, x^2, y^2, xy) of channel c.
template <typename ST>
__device__ __forceinline__ float plane_in(const ST *xr, const ST *xd, long long i, int kind) {
    const float a = ld_store<ST>(xr + i), b = ld_store<ST>(xd + i);
    switch (kind) {
    case 0: return a;
    case 1: return b;
    case 2: return a * a;
    case 3: return b * b;
    default: return a * b;
    }
}

template <typename ST>
__global__ void __launch_bounds__(128) iir_vertical_kernel(const DevPair *__restrict__ pairs,
                                                           const IirSeg *__restrict__ segs, int nseg, int total) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= total) return;
    const IirSeg sg = segs[find_iseg(segs, nseg, t)];
    const DevPair &P = pairs[sg.pair];
    const int s = sg.scale, W = P.w[s], H = P.h[s], lp = P.lp[s];
    const int local = t - sg.first;
    // thread order: plane-major within a column group of 32 so that a warp's
    // lanes are 32 adjacent columns of one plane (coalesced)
    const int grp = local / (32 * 15), rem = local % (32 * 15);
    const int p = rem / 32, x = grp * 32 + rem % 32;
    if (x >= W) return;
    const int c = p / 5, kind = p % 5;
    const long long plane = (long long)lp * H;
    const ST *xr = (const ST *)P.lvl[0][s] + c * plane + x;
    const ST *xd = (const ST *)P.lvl[1][s] + c * plane + x;
    float *dst = sg.v + p * plane + x;
    IirState st;
    st.zero();
    float ring[2 * kN];
#pragma unroll
    for (int k = 0; k < 2 * kN; k++) ring[k] = 0.f;
    // step i: right = i, left = i - 2N, output row y = i - N + 1
    const int steps = H + kN - 1;
    for (int i0 = 0; i0 < steps; i0 += 2 * kN) {
#pragma unroll
        for (int k = 0; k < 2 * kN; k++) {
            const int i = i0 + k;
            if (i < steps) {
                const float right = i < H ? plane_in<ST>(xr, xd, (long long)i * lp, kind) : 0.f;
                const float left = ring[k];  // the sample that entered 2N steps ago (0 before the start)
                ring[k] = right;
                const float out = st.step(left + right);
                const int y = i - kN + 1;
                if (y >= 0) dst[(long long)y * lp] = out;
            }
        }
    }
}

template <typename ST>
__global__ void __launch_bounds__(128) iir_horizontal_kernel(const DevPair *__restrict__ pairs,
                                                             const IirSeg *__restrict__ segs, int nseg, int total,
                                                             double *__restrict__ partials) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= total) return;
    const IirSeg sg = segs[find_iseg(segs, nseg, t)];
    const DevPair &P = pairs[sg.pair];
    const int s = sg.scale, W = P.w[s], H = P.h[s], lp = P.lp[s];
    const int local = t - sg.first;
    const int y = local / 3, c = local % 3;
    const long long plane = (long long)lp * H;
    const float *v = sg.v + (long long)y * lp;
    const ST *xr = (const ST *)P.lvl[0][s] + c * plane + (long long)y * lp;
    const ST *xd = (const ST *)P.lvl[1][s] + c * plane + (long long)y * lp;
    IirState st[5];
#pragma unroll
    for (int k = 0; k < 5; k++) st[k].zero();
    double acc[6] = {0, 0, 0, 0, 0, 0};
    const float C2 = 0.0009f;
    for (int i = 0; i < W + kN - 1; i++) {
        const int right = i, left = i - 2 * kN;
        float o[5];
#pragma unroll
        for (int k = 0; k < 5; k++) {
            const float *vp = v + (c * 5 + k) * plane;
            const float rv = right < W ? vp[right] : 0.f;
            const float lv = left >= 0 ? vp[left] : 0.f;
            o[k] = st[k].step(lv + rv);
        }
        const int x = i - kN + 1;
        if (x < 0) continue;
        // error_maps.rs:36-59, as written
        const float mu1 = o[0], mu2 = o[1], sigma11 = o[2], sigma22 = o[3], sigma12 = o[4];
        const float source = ld_store<ST>(xr + x), distorted = ld_store<ST>(xd + x);
        const float mu11 = mu1 * mu1, mu22 = mu2 * mu2, mu12 = mu1 * mu2, mu_diff = mu1 - mu2;
        const float num_m = fmaf(mu_diff, -mu_diff, 1.0f);
        const float num_s = fmaf(2.0f, sigma12 - mu12, C2);
        const float denom_s = ((sigma11 - mu11) + (sigma22 - mu22)) + C2;
        const float d = fmaxf(1.0f - (num_m * num_s) / denom_s, 0.0f);
        const float denom = 1.0f / (1.0f + fabsf(source - mu1));
        const float numer = 1.0f + fabsf(distorted - mu2);
        const float d1 = fmaf(numer, denom, -1.0f);
        const float vals[3] = {d, fmaxf(d1, 0.0f), fmaxf(-d1, 0.0f)};
        // lib.rs:986-1016: f64 sum of d, f64 sum of the f32 (d*d)*(d*d)
#pragma unroll
        for (int m = 0; m < 3; m++) {
            const float sq = vals[m] * vals[m];
            acc[m] += (double)vals[m];
            acc[3 + m] += (double)(sq * sq);
        }
    }
    double *out = partials + (long long)(sg.rec_base + y) * 18 + c * 6;
#pragma unroll
    for (int m = 0; m < 6; m++) out[m] = acc[m];
}

cudaError_t launch_iir(int storage, const DevPair *pairs, const IirSeg *vsegs, int nvseg, int vtotal,
                       const IirSeg *hsegs, int nhseg, int htotal, double *partials, cudaStream_t st) {
    (void)storage;  // f32 planes only
    if (vtotal > 0) {
        const int g = (vtotal + 127) / 128;
        iir_vertical_kernel<float><<<g, 128, 0, st>>>(pairs, vsegs, nvseg, vtotal);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    if (htotal > 0) {
        const int g = (htotal + 127) / 128;
        iir_horizontal_kernel<float><<<g, 128, 0, st>>>(pairs, hsegs, nhseg, htotal, partials);
        return cudaGetLastError();
    }
    return cudaSuccess;
}

}  // namespace s2
