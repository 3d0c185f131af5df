/*
 * dssim_oracle.c -- CPU restatement of DSSIM as the turbo-metrics crate
 * dssim-cuda computes it: the sibling metric that shares SSIMULACRA2's
 * sRGB LUT and 2x2 linear-RGB pyramid.
 *
 * TEST INFRASTRUCTURE ONLY.  Parity tests and the benchmark's CPU-baseline
 * leg use it as the checker; the CUDA product path never does.
 *
 * Reference files restated here (paths inside the turbo-metrics project):
 *   pipeline, scale sizes, pooling  crates/dssim-cuda/src/lib.rs:184-205 (sizes,
 *                                   clamped to >= 8), :250-330 (per scale: RGB
 *                                   downscale, Lab, chroma pre-blur), :336-435
 *                                   (two-pass blurs, SSIM map, mean, MAD),
 *                                   :457-460 (1/ssim - 1)
 *   scale weights                   crates/dssim-cuda/src/lib.rs:77
 *   Lab conversion                  crates/dssim-cuda-kernel/src/lab.rs:15-86
 *   3x3 blur, squared, product      crates/dssim-cuda-kernel/src/blur.rs:13-173
 *   SSIM map from Lab statistics    crates/dssim-cuda-kernel/src/ssim.rs:18-19,
 *                                   :152-236; |avg - ssim| :240-262
 *   RGB 2x2 downscale               crates/dssim-cuda-kernel/src/downscale.rs:50-83
 *
 * Two arithmetic modes:
 *   OR_DSSIM_F32   the reference GPU's f32 arithmetic, operation for
 *                  operation: fused multiply-adds exactly where lab.rs and
 *                  ssim.rs use mul_add, separate multiply and add elsewhere
 *                  (the file is compiled with -ffp-contract=off), IEEE
 *                  division; sums of the SSIM map and of |avg - ssim| in
 *                  double (NPP Sum returns f64).  The cube root is
 *                  or_cbrtf, the engine's own (Kahan seed, Newton steps,
 *                  IEEE multiplies and FMAs only; within an ulp), where the
 *                  reference calls its GPU math library's cbrtf.
 *   OR_DSSIM_F64   every stage in double with the same constants: the
 *                  value the f32 pipeline approximates.
 */
#include "ssim2_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define DS_LEVELS 5

static const double DS_WEIGHTS[DS_LEVELS] = {0.028, 0.197, 0.322, 0.298, 0.155};
static const float DS_KERNEL[3][3] = {
    {0.095332f, 0.118095f, 0.095332f},
    {0.118095f, 0.146293f, 0.118095f},
    {0.095332f, 0.118095f, 0.095332f},
};

void or_dssim_level_dims(int w, int h, int dw[DS_LEVELS], int dh[DS_LEVELS]) {
    /* lib.rs:184-205: halve with rounding up, never below 8 */
    for (int s = 0; s < DS_LEVELS; s++) {
        dw[s] = w;
        dh[s] = h;
        w = (w + 1) / 2;
        h = (h + 1) / 2;
        if (w < 8) w = 8;
        if (h < 8) h = 8;
    }
}

static inline int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

/* ---- f32 mirror ---------------------------------------------------------- */

static inline float lab_f32(float t) {
    const float eps = 216.0f / 24389.0f;
    const float k = 24389.0f / (27.0f * 116.0f);
    return t > eps ? or_cbrtf(t) : fmaf(k, t, 16.0f / 116.0f);
}

void or_dssim_lab_f32(float r, float g, float b, float out[3]) {
    const float x = fmaf(0.4124f, r, fmaf(0.3576f, g, 0.1805f * b)) / 0.9505f;
    const float y = fmaf(0.2126f, r, fmaf(0.7152f, g, 0.0722f * b)) / 1.0f;
    const float z = fmaf(0.0193f, r, fmaf(0.1192f, g, 0.9505f * b)) / 1.089f;
    const float fx = lab_f32(x), fy = lab_f32(y), fz = lab_f32(z);
    out[0] = (fy - 16.0f / 116.0f) * 1.05f;
    out[1] = fmaf(fx - fy, 500.0f / 220.0f, 86.2f / 220.0f);
    out[2] = fmaf(fy - fz, 200.0f / 220.0f, 107.9f / 220.0f);
}

/* blur.rs:33-61 / :113-141 / :148-173: taps in row-major order, clamped
 * source, sum += v * k (or v * v * k, v1 * v2 * k) without contraction */
static void blur3_f32(const float *src, const float *src2, int kind, int w, int h, float *dst) {
    for (int y = 0; y < h; y++)
        for (int x = 0; x < w; x++) {
            float sum = 0.0f;
            for (int ky = 0; ky < 3; ky++)
                for (int kx = 0; kx < 3; kx++) {
                    const int sx = clampi(x + kx - 1, 0, w - 1), sy = clampi(y + ky - 1, 0, h - 1);
                    const float v = src[(size_t)sy * w + sx];
                    float t;
                    if (kind == 0) t = v * DS_KERNEL[ky][kx];
                    else if (kind == 1) t = v * v * DS_KERNEL[ky][kx];
                    else t = v * src2[(size_t)sy * w + sx] * DS_KERNEL[ky][kx];
                    sum += t;
                }
            dst[(size_t)y * w + x] = sum;
        }
}

static void downscale_rgb_f32(const float *src, int sw, int sh, float *dst, int dw, int dh) {
    for (int oy = 0; oy < dh; oy++)
        for (int ox = 0; ox < dw; ox++) {
            const int x0 = clampi(2 * ox, 0, sw - 1), x1 = clampi(2 * ox + 1, 0, sw - 1);
            const int y0 = clampi(2 * oy, 0, sh - 1), y1 = clampi(2 * oy + 1, 0, sh - 1);
            for (int c = 0; c < 3; c++) {
                const float v00 = src[((size_t)y0 * sw + x0) * 3 + c], v10 = src[((size_t)y0 * sw + x1) * 3 + c];
                const float v01 = src[((size_t)y1 * sw + x0) * 3 + c], v11 = src[((size_t)y1 * sw + x1) * 3 + c];
                dst[((size_t)oy * dw + ox) * 3 + c] = (v00 + v10 + v01 + v11) * 0.25f;
            }
        }
}

/* one scale: Lab planes of both images in, SSIM map out (ssim.rs:152-236) */
static void ssim_map_f32(float *lab[2][3], int w, int h, float *map) {
    const size_t n = (size_t)w * h;
    float *t = malloc(n * sizeof(float));
    float *st[3][5];
    for (int c = 0; c < 3; c++)
        for (int k = 0; k < 5; k++) st[c][k] = malloc(n * sizeof(float));
    for (int c = 0; c < 3; c++) {
        /* lib.rs:296-316: a and b of both images pre-blurred twice, in place */
        if (c > 0)
            for (int img = 0; img < 2; img++) {
                blur3_f32(lab[img][c], NULL, 0, w, h, t);
                blur3_f32(t, NULL, 0, w, h, lab[img][c]);
            }
        const float *x = lab[0][c], *y = lab[1][c];
        blur3_f32(x, NULL, 0, w, h, t);
        blur3_f32(t, NULL, 0, w, h, st[c][0]);
        blur3_f32(y, NULL, 0, w, h, t);
        blur3_f32(t, NULL, 0, w, h, st[c][1]);
        blur3_f32(x, NULL, 1, w, h, t);
        blur3_f32(t, NULL, 0, w, h, st[c][2]);
        blur3_f32(y, NULL, 1, w, h, t);
        blur3_f32(t, NULL, 0, w, h, st[c][3]);
        blur3_f32(x, y, 2, w, h, t);
        blur3_f32(t, NULL, 0, w, h, st[c][4]);
    }
    const float third = 1.0f / 3.0f, c1 = 0.0001f, c2 = 0.0009f;
    for (size_t i = 0; i < n; i++) {
        float m1[3], m2[3], s1[3], s2[3], cr[3];
        for (int c = 0; c < 3; c++) {
            m1[c] = st[c][0][i];
            m2[c] = st[c][1][i];
            s1[c] = st[c][2][i];
            s2[c] = st[c][3][i];
            cr[c] = st[c][4][i];
        }
        const float mu1_sq = (m1[0] * m1[0] + m1[1] * m1[1] + m1[2] * m1[2]) * third;
        const float mu2_sq = (m2[0] * m2[0] + m2[1] * m2[1] + m2[2] * m2[2]) * third;
        const float mu1_mu2 = (m1[0] * m2[0] + m1[1] * m2[1] + m1[2] * m2[2]) * third;
        const float i1 = (s1[0] + s1[1] + s1[2]) * third;
        const float i2 = (s2[0] + s2[1] + s2[2]) * third;
        const float i12 = (cr[0] + cr[1] + cr[2]) * third;
        const float sigma1_sq = i1 - mu1_sq, sigma2_sq = i2 - mu2_sq, sigma12 = i12 - mu1_mu2;
        const float num = fmaf(2.0f, mu1_mu2, c1) * fmaf(2.0f, sigma12, c2);
        const float den = (mu1_sq + mu2_sq + c1) * (sigma1_sq + sigma2_sq + c2);
        map[i] = num / den;
    }
    for (int c = 0; c < 3; c++)
        for (int k = 0; k < 5; k++) free(st[c][k]);
    free(t);
}

/* ---- f64 ----------------------------------------------------------------- */

static inline double lab_f64(double t) {
    const double eps = 216.0 / 24389.0, k = 24389.0 / (27.0 * 116.0);
    return t > eps ? cbrt(t) : k * t + 16.0 / 116.0;
}

static void lab_px_f64(double r, double g, double b, double out[3]) {
    const double x = (0.4124 * r + 0.3576 * g + 0.1805 * b) / 0.9505;
    const double y = 0.2126 * r + 0.7152 * g + 0.0722 * b;
    const double z = (0.0193 * r + 0.1192 * g + 0.9505 * b) / 1.089;
    const double fx = lab_f64(x), fy = lab_f64(y), fz = lab_f64(z);
    out[0] = (fy - 16.0 / 116.0) * 1.05;
    out[1] = (fx - fy) * (500.0 / 220.0) + 86.2 / 220.0;
    out[2] = (fy - fz) * (200.0 / 220.0) + 107.9 / 220.0;
}

static void blur3_f64(const double *src, const double *src2, int kind, int w, int h, double *dst) {
    for (int y = 0; y < h; y++)
        for (int x = 0; x < w; x++) {
            double sum = 0.0;
            for (int ky = 0; ky < 3; ky++)
                for (int kx = 0; kx < 3; kx++) {
                    const int sx = clampi(x + kx - 1, 0, w - 1), sy = clampi(y + ky - 1, 0, h - 1);
                    const double v = src[(size_t)sy * w + sx];
                    const double k = (double)DS_KERNEL[ky][kx];
                    sum += kind == 0 ? v * k : (kind == 1 ? v * v * k : v * src2[(size_t)sy * w + sx] * k);
                }
            dst[(size_t)y * w + x] = sum;
        }
}

static void downscale_rgb_f64(const double *src, int sw, int sh, double *dst, int dw, int dh) {
    for (int oy = 0; oy < dh; oy++)
        for (int ox = 0; ox < dw; ox++) {
            const int x0 = clampi(2 * ox, 0, sw - 1), x1 = clampi(2 * ox + 1, 0, sw - 1);
            const int y0 = clampi(2 * oy, 0, sh - 1), y1 = clampi(2 * oy + 1, 0, sh - 1);
            for (int c = 0; c < 3; c++)
                dst[((size_t)oy * dw + ox) * 3 + c] =
                    (src[((size_t)y0 * sw + x0) * 3 + c] + src[((size_t)y0 * sw + x1) * 3 + c] +
                     src[((size_t)y1 * sw + x0) * 3 + c] + src[((size_t)y1 * sw + x1) * 3 + c]) * 0.25;
        }
}

static void ssim_map_f64(double *lab[2][3], int w, int h, double *map) {
    const size_t n = (size_t)w * h;
    double *t = malloc(n * sizeof(double));
    double *st[3][5];
    for (int c = 0; c < 3; c++)
        for (int k = 0; k < 5; k++) st[c][k] = malloc(n * sizeof(double));
    for (int c = 0; c < 3; c++) {
        if (c > 0)
            for (int img = 0; img < 2; img++) {
                blur3_f64(lab[img][c], NULL, 0, w, h, t);
                blur3_f64(t, NULL, 0, w, h, lab[img][c]);
            }
        const double *x = lab[0][c], *y = lab[1][c];
        blur3_f64(x, NULL, 0, w, h, t);
        blur3_f64(t, NULL, 0, w, h, st[c][0]);
        blur3_f64(y, NULL, 0, w, h, t);
        blur3_f64(t, NULL, 0, w, h, st[c][1]);
        blur3_f64(x, NULL, 1, w, h, t);
        blur3_f64(t, NULL, 0, w, h, st[c][2]);
        blur3_f64(y, NULL, 1, w, h, t);
        blur3_f64(t, NULL, 0, w, h, st[c][3]);
        blur3_f64(x, y, 2, w, h, t);
        blur3_f64(t, NULL, 0, w, h, st[c][4]);
    }
    for (size_t i = 0; i < n; i++) {
        double mu1_sq = 0, mu2_sq = 0, mu1_mu2 = 0, i1 = 0, i2 = 0, i12 = 0;
        for (int c = 0; c < 3; c++) {
            mu1_sq += st[c][0][i] * st[c][0][i];
            mu2_sq += st[c][1][i] * st[c][1][i];
            mu1_mu2 += st[c][0][i] * st[c][1][i];
            i1 += st[c][2][i];
            i2 += st[c][3][i];
            i12 += st[c][4][i];
        }
        mu1_sq /= 3.0, mu2_sq /= 3.0, mu1_mu2 /= 3.0, i1 /= 3.0, i2 /= 3.0, i12 /= 3.0;
        const double c1 = (double)0.0001f, c2 = (double)0.0009f;
        map[i] = (2.0 * mu1_mu2 + c1) * (2.0 * (i12 - mu1_mu2) + c2) /
                 ((mu1_sq + mu2_sq + c1) * ((i1 - mu1_sq) + (i2 - mu2_sq) + c2));
    }
    for (int c = 0; c < 3; c++)
        for (int k = 0; k < 5; k++) free(st[c][k]);
    free(t);
}

/* ---- driver -------------------------------------------------------------- */

int or_dssim_linear(const float *ref, const float *dis, int w, int h, int mode, double level_score[DS_LEVELS],
                    double level_mean[DS_LEVELS], double *dssim) {
    if (w < 8 || h < 8) return 1;
    int dw[DS_LEVELS], dh[DS_LEVELS];
    or_dssim_level_dims(w, h, dw, dh);
    const size_t n0 = (size_t)w * h;
    double wsum = 0.0, wtot = 0.0;
    if (mode == OR_DSSIM_F32) {
        float *lin[2] = {malloc(n0 * 3 * sizeof(float)), malloc(n0 * 3 * sizeof(float))};
        memcpy(lin[0], ref, n0 * 3 * sizeof(float));
        memcpy(lin[1], dis, n0 * 3 * sizeof(float));
        for (int s = 0; s < DS_LEVELS; s++) {
            const int W = dw[s], H = dh[s];
            const size_t n = (size_t)W * H;
            if (s > 0)
                for (int img = 0; img < 2; img++) {
                    float *nl = malloc(n * 3 * sizeof(float));
                    downscale_rgb_f32(lin[img], dw[s - 1], dh[s - 1], nl, W, H);
                    free(lin[img]);
                    lin[img] = nl;
                }
            float *lab[2][3];
            for (int img = 0; img < 2; img++) {
                for (int c = 0; c < 3; c++) lab[img][c] = malloc(n * sizeof(float));
                for (size_t i = 0; i < n; i++) {
                    float o[3];
                    or_dssim_lab_f32(lin[img][i * 3], lin[img][i * 3 + 1], lin[img][i * 3 + 2], o);
                    for (int c = 0; c < 3; c++) lab[img][c][i] = o[c];
                }
            }
            float *map = malloc(n * sizeof(float));
            ssim_map_f32(lab, W, H, map);
            double sum = 0.0;
            for (size_t i = 0; i < n; i++) sum += map[i];
            const double mean = sum / (double)n;
            /* lib.rs:411-428: avg = max(mean, 0)^(0.5^s), |avg - ssim| in f32 */
            const float avg = (float)pow(mean > 0.0 ? mean : 0.0, ldexp(1.0, -s));
            double mad = 0.0;
            for (size_t i = 0; i < n; i++) mad += fabsf(avg - map[i]);
            level_mean[s] = mean;
            level_score[s] = 1.0 - mad / (double)n;
            wsum += level_score[s] * DS_WEIGHTS[s];
            wtot += DS_WEIGHTS[s];
            free(map);
            for (int img = 0; img < 2; img++)
                for (int c = 0; c < 3; c++) free(lab[img][c]);
        }
        free(lin[0]);
        free(lin[1]);
    } else {
        double *lin[2] = {malloc(n0 * 3 * sizeof(double)), malloc(n0 * 3 * sizeof(double))};
        for (size_t i = 0; i < n0 * 3; i++) lin[0][i] = ref[i], lin[1][i] = dis[i];
        for (int s = 0; s < DS_LEVELS; s++) {
            const int W = dw[s], H = dh[s];
            const size_t n = (size_t)W * H;
            if (s > 0)
                for (int img = 0; img < 2; img++) {
                    double *nl = malloc(n * 3 * sizeof(double));
                    downscale_rgb_f64(lin[img], dw[s - 1], dh[s - 1], nl, W, H);
                    free(lin[img]);
                    lin[img] = nl;
                }
            double *lab[2][3];
            for (int img = 0; img < 2; img++) {
                for (int c = 0; c < 3; c++) lab[img][c] = malloc(n * sizeof(double));
                for (size_t i = 0; i < n; i++) {
                    double o[3];
                    lab_px_f64(lin[img][i * 3], lin[img][i * 3 + 1], lin[img][i * 3 + 2], o);
                    for (int c = 0; c < 3; c++) lab[img][c][i] = o[c];
                }
            }
            double *map = malloc(n * sizeof(double));
            ssim_map_f64(lab, W, H, map);
            long double sum = 0.0L;
            for (size_t i = 0; i < n; i++) sum += map[i];
            const double mean = (double)(sum / (long double)n);
            const double avg = pow(mean > 0.0 ? mean : 0.0, ldexp(1.0, -s));
            long double mad = 0.0L;
            for (size_t i = 0; i < n; i++) mad += fabs(avg - map[i]);
            level_mean[s] = mean;
            level_score[s] = 1.0 - (double)(mad / (long double)n);
            wsum += level_score[s] * DS_WEIGHTS[s];
            wtot += DS_WEIGHTS[s];
            free(map);
            for (int img = 0; img < 2; img++)
                for (int c = 0; c < 3; c++) free(lab[img][c]);
        }
        free(lin[0]);
        free(lin[1]);
    }
    const double ssim = wsum / wtot;
    *dssim = 1.0 / (ssim > DBL_EPSILON ? ssim : DBL_EPSILON) - 1.0;
    return 0;
}
