/*
 * ssim2_oracle.c -- CPU restatement of the SSIMULACRA2 hot path of
 * imazen/turbo-metrics (see ssim2_oracle.h for the modes).
 *
 * TEST INFRASTRUCTURE ONLY.  Parity tests, the smoke check and the benchmark's
 * CPU-baseline leg use it as the checker; the CUDA product path never does.
 *
 * Reference files restated here (paths inside the turbo-metrics project):
 *   sRGB transfer / LUT      crates/ssimulacra2-cuda-kernel/src/srgb.rs:3-51
 *   XYB                      crates/ssimulacra2-cuda-kernel/src/xyb.rs:3-78
 *   2x2 downscale            crates/ssimulacra2-cuda-kernel/src/downscale.rs:4-35
 *   blur constants           crates/ssimulacra2-cuda-kernel/build.rs:28-145
 *   GPU IIR walk             crates/ssimulacra2-cuda-kernel/src/blur.rs:95-136
 *   CPU IIR walks            crates/ssimulacra2-cuda/examples/cpu.rs:967-1115
 *   error maps (GPU f32)     crates/ssimulacra2-cuda-kernel/src/error_maps.rs:20-59
 *   error maps (CPU f64)     crates/ssimulacra2-cuda/examples/cpu.rs:581-683
 *   pooling + score          crates/ssimulacra2-cuda/src/lib.rs:986-1192,
 *                            crates/ssimulacra2-cuda/examples/cpu.rs:728-871
 *   pyramid + stop rule      crates/ssimulacra2-cuda/examples/cpu.rs:342-410,
 *                            crates/ssim2-gpu/src/pipeline.rs:194-206
 *   NV12 -> linear           crates/cuda-colorspace-kernel/src/biplanar.rs:8-70,
 *                            crates/cuda-colorspace-kernel/src/lib.rs:188-238
 */
#include "ssim2_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define NSCALES 6

/* ------------------------------------------------------------------------ */
/* Recursive Gaussian (Charalampidis 2016, truncated cosines), sigma = 1.5.  */
/* Follows the derivation order of ssimulacra2-cuda-kernel/build.rs:28-145.  */
/* ------------------------------------------------------------------------ */

typedef struct {
    int radius;
    double n2[3], d1[3];
    float mul_in[3], mul_prev[3], mul_prev2[3];
    float vert_mul_in[3], vert_mul_prev[3];
    double fir[5]; /* exact-form taps, |k| = 0..4 */
} blur_consts;

static blur_consts g_bc;
static int g_bc_ready = 0;

static double det3(const double m[9]) {
    return m[0] * (m[4] * m[8] - m[5] * m[7]) - m[1] * (m[3] * m[8] - m[5] * m[6]) +
           m[2] * (m[3] * m[7] - m[4] * m[6]);
}

static void init_blur_consts(void) {
    if (g_bc_ready) return;
    const double sigma = 1.5;
    const double pi = 3.14159265358979323846;
    double radius = round(fma(3.2795, sigma, 0.2546)); /* eq. (57) */
    double w0 = pi / (2.0 * radius);
    double omega[3] = {w0, 3.0 * w0, 5.0 * w0};
    double p1 = 1.0 / tan(0.5 * omega[0]);
    double p3 = -1.0 / tan(0.5 * omega[1]);
    double p5 = 1.0 / tan(0.5 * omega[2]);
    double r1 = p1 * p1 / sin(omega[0]);
    double r3 = -p3 * p3 / sin(omega[1]);
    double r5 = p5 * p5 / sin(omega[2]);
    double rho[3];
    for (int i = 0; i < 3; i++)
        rho[i] = exp(-0.5 * sigma * sigma * omega[i] * omega[i]) / radius;
    double d13 = fma(p1, r3, -r1 * p3);
    double d35 = fma(p3, r5, -r3 * p5);
    double d51 = fma(p5, r1, -r5 * p1);
    double zeta15 = d35 / d13, zeta35 = d51 / d13;
    /* Solve M * beta = gamma by Cramer's rule (eq. 53-56). */
    double M[9] = {p1, p3, p5, r1, r3, r5, zeta15, zeta35, 1.0};
    double g[3] = {1.0, fma(radius, radius, -sigma * sigma),
                   fma(zeta15, rho[0], zeta35 * rho[1]) + rho[2]};
    double dm = det3(M), beta[3];
    for (int col = 0; col < 3; col++) {
        double Mc[9];
        memcpy(Mc, M, sizeof Mc);
        for (int r = 0; r < 3; r++) Mc[r * 3 + col] = g[r];
        beta[col] = det3(Mc) / dm;
    }
    g_bc.radius = (int)radius;
    for (int i = 0; i < 3; i++) {
        g_bc.n2[i] = -beta[i] * cos(omega[i] * (radius + 1.0)); /* eq. (33) */
        g_bc.d1[i] = -2.0 * cos(omega[i]);
        g_bc.mul_in[i] = (float)g_bc.n2[i];
        g_bc.mul_prev[i] = (float)(-g_bc.d1[i]);
        g_bc.mul_prev2[i] = -1.0f;
        g_bc.vert_mul_in[i] = (float)g_bc.n2[i];
        g_bc.vert_mul_prev[i] = (float)g_bc.d1[i];
    }
    /* Exact form: the impulse response of the double-precision recursion.
     * The truncated-cosine construction cancels every term beyond |k| = N-1,
     * so the response is a symmetric FIR of 2N-1 taps with zero padding. */
    {
        const int N = g_bc.radius, L = 64, c = 32;
        double in[64] = {0}, out[64] = {0};
        in[c] = 1.0;
        double prev[3] = {0}, prev2[3] = {0};
        for (int n = -N + 1; n < L; n++) {
            int left = n - N - 1, right = n + N - 1;
            double lv = (left >= 0) ? in[left] : 0.0;
            double rv = (right < L) ? in[right] : 0.0;
            double s = lv + rv, o = 0.0;
            for (int k = 0; k < 3; k++) {
                double ok = s * g_bc.n2[k] - g_bc.d1[k] * prev[k] - prev2[k];
                prev2[k] = prev[k];
                prev[k] = ok;
                o += ok;
            }
            if (n >= 0) out[n] = o;
        }
        for (int k = 0; k < 5; k++) g_bc.fir[k] = out[c + k];
    }
    g_bc_ready = 1;
}

int or_blur_constants(float mul_in[3], float mul_prev[3], float mul_prev2[3],
                      float vert_mul_in[3], float vert_mul_prev[3],
                      double fir_taps[5]) {
    init_blur_consts();
    for (int i = 0; i < 3; i++) {
        if (mul_in) mul_in[i] = g_bc.mul_in[i];
        if (mul_prev) mul_prev[i] = g_bc.mul_prev[i];
        if (mul_prev2) mul_prev2[i] = g_bc.mul_prev2[i];
        if (vert_mul_in) vert_mul_in[i] = g_bc.vert_mul_in[i];
        if (vert_mul_prev) vert_mul_prev[i] = g_bc.vert_mul_prev[i];
    }
    if (fir_taps)
        for (int k = 0; k < 5; k++) fir_taps[k] = g_bc.fir[k];
    return g_bc.radius;
}

/* ------------------------------------------------------------------------ */
/* Input conversions                                                         */
/* ------------------------------------------------------------------------ */

/* sRGB8 -> linear table of the reference (ssimulacra2-cuda-kernel/src/srgb.rs:23-51,
 * identical to examples/cpu.rs:20-277).  The entries follow the gamma-2.4 sRGB
 * curve with a linear toe (srgb.rs:3-15) but were printed with 6-9 decimal
 * digits, so they differ from the formula by up to 4.7e-6; the table itself
 * defines the conversion.  Values are the same numbers, written as hex floats. */
static const float SRGB8_LUT[256] = {
    0x0p+0f, 0x1.3e4568p-12f, 0x1.3e4568p-11f, 0x1.dd681ep-11f, 0x1.3e4568p-10f, 0x1.8dd6c2p-10f,
    0x1.dd681ep-10f, 0x1.167cbcp-9f, 0x1.3e4568p-9f, 0x1.660e16p-9f, 0x1.8dd6c2p-9f, 0x1.b6a31ap-9f,
    0x1.e1e31ap-9f, 0x1.07c38cp-8f, 0x1.1fcc2cp-8f, 0x1.390ffap-8f, 0x1.53936ep-8f, 0x1.6f5adep-8f,
    0x1.8c6a92p-8f, 0x1.aac6c2p-8f, 0x1.ca7382p-8f, 0x1.eb74ep-8f, 0x1.06e76ap-7f, 0x1.18c2a4p-7f,
    0x1.2b4e06p-7f, 0x1.3e8b7cp-7f, 0x1.527cd6p-7f, 0x1.6723eep-7f, 0x1.7c8292p-7f, 0x1.929a86p-7f,
    0x1.a96d8ep-7f, 0x1.c0fd62p-7f, 0x1.d94bbep-7f, 0x1.f25a44p-7f, 0x1.06155p-6f, 0x1.135f3ep-6f,
    0x1.210bb6p-6f, 0x1.2f1b8ap-6f, 0x1.3d8f84p-6f, 0x1.4c6866p-6f, 0x1.5ba6fap-6f, 0x1.6b4c02p-6f,
    0x1.7b584p-6f, 0x1.8bcc72p-6f, 0x1.9ca956p-6f, 0x1.adefaap-6f, 0x1.bfa02p-6f, 0x1.d1bb72p-6f,
    0x1.e44262p-6f, 0x1.f7358cp-6f, 0x1.054ad8p-5f, 0x1.0f31bep-5f, 0x1.194fcep-5f, 0x1.23a564p-5f,
    0x1.2e32cap-5f, 0x1.38f862p-5f, 0x1.43f67ep-5f, 0x1.4f2d6ap-5f, 0x1.5a9d7cp-5f, 0x1.664708p-5f,
    0x1.722a5cp-5f, 0x1.7e47ccp-5f, 0x1.8a9fa8p-5f, 0x1.97323ep-5f, 0x1.a3ffdep-5f, 0x1.b108d4p-5f,
    0x1.be4d6ep-5f, 0x1.cbcdfcp-5f, 0x1.d98ac8p-5f, 0x1.e7841ep-5f, 0x1.f5ba52p-5f, 0x1.0216cep-4f,
    0x1.096f2ap-4f, 0x1.10e66p-4f, 0x1.187c94p-4f, 0x1.2031ecp-4f, 0x1.28068ap-4f, 0x1.2ffa94p-4f,
    0x1.380e2cp-4f, 0x1.404176p-4f, 0x1.489496p-4f, 0x1.5107aep-4f, 0x1.599aep-4f, 0x1.624e5p-4f,
    0x1.6b2224p-4f, 0x1.741676p-4f, 0x1.7d2b6ap-4f, 0x1.866124p-4f, 0x1.8fb7c4p-4f, 0x1.992f6cp-4f,
    0x1.a2c83ep-4f, 0x1.ac8258p-4f, 0x1.b65ddep-4f, 0x1.c05aeep-4f, 0x1.ca79aap-4f, 0x1.d4ba32p-4f,
    0x1.df1caap-4f, 0x1.e9a126p-4f, 0x1.f447d4p-4f, 0x1.ff10c8p-4f, 0x1.04fe12p-3f, 0x1.0a8504p-3f,
    0x1.101d4ap-3f, 0x1.15c6f2p-3f, 0x1.1b820ep-3f, 0x1.214eaap-3f, 0x1.272cd8p-3f, 0x1.2d1ca6p-3f,
    0x1.331e22p-3f, 0x1.39315cp-3f, 0x1.3f5664p-3f, 0x1.458d46p-3f, 0x1.4bd616p-3f, 0x1.5230dap-3f,
    0x1.589da8p-3f, 0x1.5f1c8ap-3f, 0x1.65ad9p-3f, 0x1.6c50cap-3f, 0x1.730644p-3f, 0x1.79ce0cp-3f,
    0x1.80a832p-3f, 0x1.8794c4p-3f, 0x1.8e93dp-3f, 0x1.95a562p-3f, 0x1.9cc98cp-3f, 0x1.a40056p-3f,
    0x1.ab49d2p-3f, 0x1.b2a60ep-3f, 0x1.ba1516p-3f, 0x1.c196f8p-3f, 0x1.c92bcp-3f, 0x1.d0d37ep-3f,
    0x1.d88e4p-3f, 0x1.e05c18p-3f, 0x1.e83d08p-3f, 0x1.f0312p-3f, 0x1.f8387p-3f, 0x1.002984p-2f,
    0x1.044078p-2f, 0x1.08611ap-2f, 0x1.0c8b74p-2f, 0x1.10bf8ap-2f, 0x1.14fd64p-2f, 0x1.194506p-2f,
    0x1.1d967ap-2f, 0x1.21f1c2p-2f, 0x1.2656e8p-2f, 0x1.2ac5fp-2f, 0x1.2f3ee2p-2f, 0x1.33c1c4p-2f,
    0x1.384e9cp-2f, 0x1.3ce56ep-2f, 0x1.418644p-2f, 0x1.463124p-2f, 0x1.4ae61p-2f, 0x1.4fa512p-2f,
    0x1.546e3p-2f, 0x1.59416ep-2f, 0x1.5e1ed2p-2f, 0x1.630666p-2f, 0x1.67f83p-2f, 0x1.6cf43p-2f,
    0x1.71fa6ep-2f, 0x1.770af2p-2f, 0x1.7c25c2p-2f, 0x1.814ae2p-2f, 0x1.867a5ap-2f, 0x1.8bb42ep-2f,
    0x1.90f866p-2f, 0x1.964706p-2f, 0x1.9ba016p-2f, 0x1.a1039ap-2f, 0x1.a67198p-2f, 0x1.abea16p-2f,
    0x1.b16d1ap-2f, 0x1.b6faa8p-2f, 0x1.bc92cap-2f, 0x1.c23582p-2f, 0x1.c7e2d6p-2f, 0x1.cd9acep-2f,
    0x1.d35d6cp-2f, 0x1.d92abap-2f, 0x1.df02bap-2f, 0x1.e4e574p-2f, 0x1.ead2ecp-2f, 0x1.f0cb28p-2f,
    0x1.f6ce2ep-2f, 0x1.fcdc04p-2f, 0x1.017a5ap-1f, 0x1.048c1cp-1f, 0x1.07a34ep-1f, 0x1.0abff2p-1f,
    0x1.0de21p-1f, 0x1.1109a2p-1f, 0x1.1436aep-1f, 0x1.17693ap-1f, 0x1.1aa144p-1f, 0x1.1dded2p-1f,
    0x1.2121e4p-1f, 0x1.246a8p-1f, 0x1.27b8a6p-1f, 0x1.2b0c5ap-1f, 0x1.2e659ep-1f, 0x1.31c476p-1f,
    0x1.3528e2p-1f, 0x1.3892e6p-1f, 0x1.3c0286p-1f, 0x1.3f77c2p-1f, 0x1.42f2ap-1f, 0x1.46731ep-1f,
    0x1.49f944p-1f, 0x1.4d851p-1f, 0x1.511686p-1f, 0x1.54adaap-1f, 0x1.584a7ep-1f, 0x1.5bed02p-1f,
    0x1.5f953cp-1f, 0x1.634332p-1f, 0x1.66f6dcp-1f, 0x1.6ab044p-1f, 0x1.6e6f6ap-1f, 0x1.72345p-1f,
    0x1.75fefcp-1f, 0x1.79cf6ep-1f, 0x1.7da5a8p-1f, 0x1.8181acp-1f, 0x1.85638p-1f, 0x1.894b24p-1f,
    0x1.8d389ap-1f, 0x1.912be6p-1f, 0x1.952508p-1f, 0x1.992406p-1f, 0x1.9d28ep-1f, 0x1.a1339ap-1f,
    0x1.a54434p-1f, 0x1.a95ab2p-1f, 0x1.ad7718p-1f, 0x1.b19966p-1f, 0x1.b5c19ep-1f, 0x1.b9efc4p-1f,
    0x1.be23dcp-1f, 0x1.c25de4p-1f, 0x1.c69ddep-1f, 0x1.cae3d8p-1f, 0x1.cf2fc6p-1f, 0x1.d381b6p-1f,
    0x1.d7d99ap-1f, 0x1.dc3788p-1f, 0x1.e09b7p-1f, 0x1.e50568p-1f, 0x1.e9755cp-1f, 0x1.edeb66p-1f,
    0x1.f26772p-1f, 0x1.f6e996p-1f, 0x1.fb71cp-1f, 0x1p+0f,
};

void or_srgb8_lut(float lut[256]) { memcpy(lut, SRGB8_LUT, sizeof SRGB8_LUT); }

void or_srgb8_to_linear(const uint8_t *src, size_t n, float *dst) {
    for (size_t i = 0; i < n; i++) dst[i] = SRGB8_LUT[src[i]];
}

void or_srgb8_to_linear_f64(const uint8_t *src, size_t n, double *dst) {
    for (size_t i = 0; i < n; i++) dst[i] = (double)SRGB8_LUT[src[i]];
}

/* Kr/Kb from primaries and white point (cuda-colorspace-kernel/src/lib.rs:205-221). */
static void kr_kb_from_primaries(const double prim[8], double *kr, double *kb) {
    double xyz[4][3];
    for (int i = 0; i < 4; i++) {
        double x = prim[2 * i], y = prim[2 * i + 1];
        xyz[i][0] = x / y;
        xyz[i][1] = 1.0;
        xyz[i][2] = (1.0 - x - y) / y;
    }
    /* columns r,g,b; rows X,Y,Z */
    double X[3] = {xyz[0][0], xyz[1][0], xyz[2][0]};
    double Y[3] = {xyz[0][1], xyz[1][1], xyz[2][1]};
    double Z[3] = {xyz[0][2], xyz[1][2], xyz[2][2]};
    double cyz[3] = {Y[1] * Z[2] - Y[2] * Z[1], Y[2] * Z[0] - Y[0] * Z[2], Y[0] * Z[1] - Y[1] * Z[0]};
    double mul = 1.0 / (X[0] * cyz[0] + X[1] * cyz[1] + X[2] * cyz[2]);
    const double *r = xyz[0], *g = xyz[1], *b = xyz[2], *w = xyz[3];
    double gxb[3] = {g[1] * b[2] - g[2] * b[1], g[2] * b[0] - g[0] * b[2], g[0] * b[1] - g[1] * b[0]};
    double rxg[3] = {r[1] * g[2] - r[2] * g[1], r[2] * g[0] - r[0] * g[2], r[0] * g[1] - r[1] * g[0]};
    *kr = (w[0] * gxb[0] + w[1] * gxb[1] + w[2] * gxb[2]) * mul;
    *kb = (w[0] * rxg[0] + w[1] * rxg[1] + w[2] * rxg[2]) * mul;
}

static const double BT709_PRIM[8] = {0.640, 0.330, 0.300, 0.600, 0.150, 0.060, 0.3127, 0.3290};

/* BT.709 inverse OETF (cuda-colorspace-kernel/src/lib.rs:223-238). */
static double bt709_eotf_f64(double v) {
    const double beta = 0.018053968510807, alpha = 1.0 + 5.5 * beta;
    const double thr = 0.08124285829863521110029445797874;
    if (v >= thr) return pow((v + (alpha - 1.0)) / alpha, 1.0 / 0.45);
    return v / 4.5;
}
static inline float eng_pow_20_9(float p);
/* The engine's f32 BT.709 inverse OETF: divisions by alpha and 4.5 become
 * multiplications by their f32 reciprocals; both branches evaluated. */
static float bt709_eotf_f32(float v) {
    const float alpha_m1 = 0x1.96b84p-4f, inv_alpha = 0x1.d1c096p-1f;
    const float thr = 0.08124285829863521110029445797874f;
    const float hi = eng_pow_20_9((v + alpha_m1) * inv_alpha);
    const float lo = v * 0x1.c71c72p-3f;
    return v >= thr ? hi : lo;
}

static float clamp01f(float v) { return v < 0.0f ? 0.0f : (v > 1.0f ? 1.0f : v); }
static double clamp01(double v) { return v < 0.0 ? 0.0 : (v > 1.0 ? 1.0 : v); }

/* Primaries and white of the YUV matrices (cuda-colorspace-kernel/src/
 * constants.rs): BT.709, BT.601-525 (SMPTE C), BT.601-625 (EBU), D65. */
static const double BT601_525_PRIM[8] = {0.630, 0.340, 0.310, 0.595, 0.155, 0.070, 0.3127, 0.3290};
static const double BT601_625_PRIM[8] = {0.640, 0.330, 0.290, 0.600, 0.150, 0.060, 0.3127, 0.3290};

/* Coefficients of cuda-colorspace-kernel/src/lib.rs:188-203 for a matrix
 * (0 BT.709, 1 BT.601-525, 2 BT.601-625), range (0 limited, 1 full) and
 * sample depth (8 or 16 bits): luma and chroma ranges, the luma minimum and
 * the chroma neutral value of lib.rs:46-140 (limited: 16<<(N-8), 235<<(N-8),
 * 240<<(N-8); full: 0, 2^N - 1; neutral 2^(N-1)). */
static void yuv_coeffs(int matrix, int full, int bits, double c[5], int *ymin, int *neutral) {
    const double *prim = matrix == 1 ? BT601_525_PRIM : (matrix == 2 ? BT601_625_PRIM : BT709_PRIM);
    double kr, kb;
    kr_kb_from_primaries(prim, &kr, &kb);
    const double kg = 1.0 - kr - kb;
    const int sh = bits - 8;
    const double lrange = full ? (double)((1 << bits) - 1) : (double)((235 - 16) << sh);
    const double crange = full ? (double)((1 << bits) - 1) : (double)((240 - 16) << sh);
    c[0] = 1.0 / lrange;
    c[1] = 2.0 * (1.0 - kr) / crange;
    c[2] = 2.0 * (1.0 - kb) / crange;
    c[3] = -2.0 * (1.0 - kb) * kb / kg / crange;
    c[4] = -2.0 * (1.0 - kr) * kr / kg / crange;
    *ymin = full ? 0 : (16 << sh);
    *neutral = 1 << (bits - 1);
}

/* The reference's own f32 derivation of the same five coefficients
 * (cuda-colorspace-kernel/src/lib.rs:188-221 with const_algebra.rs): Kr / Kb
 * from the f32 primaries by constants_from_primaries, then
 * MatrixCoefficients::coefficients, every operation rounded to f32 in the
 * reference's order (this file is built with -ffp-contract=off). */
typedef struct { float x, y, z; } or_v3f;
static or_v3f or_xy_to_xyz(float x, float y) {
    or_v3f r = {x / y, 1.0f, ((1.0f - x) - y) / y};
    return r;
}
static float or_dot3f(or_v3f a, or_v3f b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
static or_v3f or_cross3f(or_v3f a, or_v3f b) {
    or_v3f r = {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
    return r;
}
void or_yuv_coeffs_ref_f32(int matrix, int full, int bits, float c[5], int *ymin, int *neutral) {
    static const float P709[8] = {0.640f, 0.330f, 0.300f, 0.600f, 0.150f, 0.060f, 0.3127f, 0.3290f};
    static const float P525[8] = {0.630f, 0.340f, 0.310f, 0.595f, 0.155f, 0.070f, 0.3127f, 0.3290f};
    static const float P625[8] = {0.640f, 0.330f, 0.290f, 0.600f, 0.150f, 0.060f, 0.3127f, 0.3290f};
    const float *p = matrix == 1 ? P525 : (matrix == 2 ? P625 : P709);
    or_v3f r = or_xy_to_xyz(p[0], p[1]), g = or_xy_to_xyz(p[2], p[3]), b = or_xy_to_xyz(p[4], p[5]),
           w = or_xy_to_xyz(p[6], p[7]);
    or_v3f xr = {r.x, g.x, b.x}, yr = {r.y, g.y, b.y}, zr = {r.z, g.z, b.z};
    float mul = 1.0f / or_dot3f(xr, or_cross3f(yr, zr));
    float kr = or_dot3f(w, or_cross3f(g, b)) * mul;
    float kb = or_dot3f(w, or_cross3f(r, g)) * mul;
    const int sh = bits - 8;
    float lrange = (float)(full ? (1u << bits) - 1u : (235u - 16u) << sh);
    float crange = (float)(full ? (1u << bits) - 1u : (240u - 16u) << sh);
    float kg = 1.0f - kr - kb;
    c[0] = 1.0f / lrange;
    c[1] = 2.0f * (1.0f - kr) * 1.0f / crange;
    c[2] = 2.0f * (1.0f - kb) * 1.0f / crange;
    c[3] = -2.0f * (1.0f - kb) * kb / kg * 1.0f / crange;
    c[4] = -2.0f * (1.0f - kr) * kr / kg * 1.0f / crange;
    if (ymin) *ymin = full ? 0 : (16 << sh);
    if (neutral) *neutral = 1 << (bits - 1);
}

/* The f32 constants of the BT.709 inverse OETF as the engine compiles them:
 * alpha - 1, 1 / alpha, the threshold, 1 / 4.5 (for the parity tests). */
void or_bt709_eotf_consts(float out[4]) {
    out[0] = 0x1.96b84p-4f;
    out[1] = 0x1.d1c096p-1f;
    out[2] = 0.08124285829863521110029445797874f;
    out[3] = 0x1.c71c72p-3f;
}

static inline int yuv_sample(const void *p, size_t byte_off, int bits) {
    return bits == 8 ? ((const uint8_t *)p)[byte_off] : *(const uint16_t *)((const uint8_t *)p + byte_off);
}

/* 4:2:0 biplanar YUV (NV12 8-bit, P016 16-bit samples) -> linear RGB in the
 * engine's f32 arithmetic (cuda-colorspace-kernel/src/biplanar.rs:8-70:
 * nearest chroma, luma floored at the range minimum, BT.709 inverse OETF,
 * clamp to [0, 1]).  pitch in bytes, shared by both planes. */
void or_yuv420_to_linear(const void *yp, const void *uvp, size_t pitch, int w, int h, int bits, int matrix,
                         int full, float *dst) {
    float cf[5];
    int ymin, neutral;
    or_yuv_coeffs_ref_f32(matrix, full, bits, cf, &ymin, &neutral);
    const int es = bits == 8 ? 1 : 2;
    float yc = cf[0], rc = cf[1], bc = cf[2], g1 = cf[3], g2 = cf[4];
    for (int y = 0; y < h; y++) {
        for (int x = 0; x < w; x++) {
            const size_t uvo = (size_t)(y / 2) * pitch + (size_t)es * 2 * (x / 2);
            float cb = (float)(yuv_sample(uvp, uvo, bits) - neutral);
            float cr = (float)(yuv_sample(uvp, uvo + es, bits) - neutral);
            float r_ = rc * cr, g_ = fmaf(g1, cb, g2 * cr), b_ = bc * cb;
            int Y = yuv_sample(yp, (size_t)y * pitch + (size_t)es * x, bits);
            float luma = (float)((Y < ymin ? ymin : Y) - ymin) * yc;
            float *o = dst + ((size_t)y * w + x) * 3;
            o[0] = clamp01f(bt709_eotf_f32(luma + r_));
            o[1] = clamp01f(bt709_eotf_f32(luma + g_));
            o[2] = clamp01f(bt709_eotf_f32(luma + b_));
        }
    }
}

void or_yuv420_to_linear_f64(const void *yp, const void *uvp, size_t pitch, int w, int h, int bits, int matrix,
                             int full, double *dst) {
    double c[5];
    int ymin, neutral;
    yuv_coeffs(matrix, full, bits, c, &ymin, &neutral);
    const int es = bits == 8 ? 1 : 2;
    for (int y = 0; y < h; y++) {
        for (int x = 0; x < w; x++) {
            const size_t uvo = (size_t)(y / 2) * pitch + (size_t)es * 2 * (x / 2);
            double cb = (double)(yuv_sample(uvp, uvo, bits) - neutral);
            double cr = (double)(yuv_sample(uvp, uvo + es, bits) - neutral);
            int Y = yuv_sample(yp, (size_t)y * pitch + (size_t)es * x, bits);
            double luma = (double)((Y < ymin ? ymin : Y) - ymin) * c[0];
            double *o = dst + ((size_t)y * w + x) * 3;
            o[0] = clamp01(bt709_eotf_f64(luma + c[1] * cr));
            o[1] = clamp01(bt709_eotf_f64(luma + c[3] * cb + c[4] * cr));
            o[2] = clamp01(bt709_eotf_f64(luma + c[2] * cb));
        }
    }
}

void or_nv12_to_linear(const uint8_t *yp, const uint8_t *uvp, size_t pitch, int w, int h, float *dst) {
    or_yuv420_to_linear(yp, uvp, pitch, w, h, 8, 0, 0, dst);
}

void or_nv12_to_linear_f64(const uint8_t *yp, const uint8_t *uvp, size_t pitch, int w, int h, double *dst) {
    or_yuv420_to_linear_f64(yp, uvp, pitch, w, h, 8, 0, 0, dst);
}

/* Linear BT.2020 RGB -> linear BT.709 RGB, derived from the published
 * primaries with the method of constants_from_primaries: RGB->XYZ matrices
 * normalised to the D65 white, M = M709^-1 * M2020. */
static void rgb_to_xyz(const double prim[8], double m[9]) {
    double P[9], S[3], W[3];
    for (int i = 0; i < 3; i++) {
        double x = prim[2 * i], y = prim[2 * i + 1];
        P[0 * 3 + i] = x / y;
        P[1 * 3 + i] = 1.0;
        P[2 * 3 + i] = (1.0 - x - y) / y;
    }
    W[0] = prim[6] / prim[7];
    W[1] = 1.0;
    W[2] = (1.0 - prim[6] - prim[7]) / prim[7];
    /* S = P^-1 W by Cramer */
    double dp = det3(P);
    for (int col = 0; col < 3; col++) {
        double Pc[9];
        memcpy(Pc, P, sizeof Pc);
        for (int r = 0; r < 3; r++) Pc[r * 3 + col] = W[r];
        S[col] = det3(Pc) / dp;
    }
    for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++) m[r * 3 + c] = P[r * 3 + c] * S[c];
}

static void inv3(const double m[9], double o[9]) {
    double d = det3(m);
    o[0] = (m[4] * m[8] - m[5] * m[7]) / d;
    o[1] = (m[2] * m[7] - m[1] * m[8]) / d;
    o[2] = (m[1] * m[5] - m[2] * m[4]) / d;
    o[3] = (m[5] * m[6] - m[3] * m[8]) / d;
    o[4] = (m[0] * m[8] - m[2] * m[6]) / d;
    o[5] = (m[2] * m[3] - m[0] * m[5]) / d;
    o[6] = (m[3] * m[7] - m[4] * m[6]) / d;
    o[7] = (m[1] * m[6] - m[0] * m[7]) / d;
    o[8] = (m[0] * m[4] - m[1] * m[3]) / d;
}

void or_bt2020_to_bt709_matrix(double m[9]) {
    static const double BT2020_PRIM[8] = {0.708, 0.292, 0.170, 0.797,
                                          0.131, 0.046, 0.3127, 0.3290};
    double a[9], b[9], bi[9];
    rgb_to_xyz(BT2020_PRIM, a);
    rgb_to_xyz(BT709_PRIM, b);
    inv3(b, bi);
    for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++)
            m[r * 3 + c] = bi[r * 3 + 0] * a[0 * 3 + c] + bi[r * 3 + 1] * a[1 * 3 + c] +
                           bi[r * 3 + 2] * a[2 * 3 + c];
}

void or_rgb16_bt2020_to_linear(const uint16_t *src, size_t n, int bits, float *dst) {
    double md[9];
    or_bt2020_to_bt709_matrix(md);
    float m[9];
    for (int i = 0; i < 9; i++) m[i] = (float)md[i];
    float inv_max = 1.0f / (float)((1 << bits) - 1);
    for (size_t p = 0; p < n; p++) {
        float l[3];
        for (int c = 0; c < 3; c++) l[c] = bt709_eotf_f32((float)src[3 * p + c] * inv_max);
        for (int r = 0; r < 3; r++) {
            float v = fmaf(m[3 * r + 0], l[0], fmaf(m[3 * r + 1], l[1], m[3 * r + 2] * l[2]));
            dst[3 * p + r] = v < 0.0f ? 0.0f : v;
        }
    }
}

void or_rgb16_bt2020_to_linear_f64(const uint16_t *src, size_t n, int bits, double *dst) {
    double m[9];
    or_bt2020_to_bt709_matrix(m);
    double inv_max = 1.0 / (double)((1 << bits) - 1);
    for (size_t p = 0; p < n; p++) {
        double l[3];
        for (int c = 0; c < 3; c++) l[c] = bt709_eotf_f64((double)src[3 * p + c] * inv_max);
        for (int r = 0; r < 3; r++) {
            double v = m[3 * r] * l[0] + m[3 * r + 1] * l[1] + m[3 * r + 2] * l[2];
            dst[3 * p + r] = v < 0.0 ? 0.0 : v;
        }
    }
}

/* ------------------------------------------------------------------------ */
/* Pyramid and XYB                                                           */
/* ------------------------------------------------------------------------ */

/* downscale.rs:4-35 -- 2x2 mean, source index clamped at the far edge,
 * accumulated ((a + b) + c) + d then times 0.25. */
void or_downscale_f32(const float *src, int w, int h, float *dst) {
    int ow = (w + 1) / 2, oh = (h + 1) / 2;
    for (int oy = 0; oy < oh; oy++)
        for (int ox = 0; ox < ow; ox++)
            for (int c = 0; c < 3; c++) {
                float s = 0.0f;
                for (int iy = 0; iy < 2; iy++)
                    for (int ix = 0; ix < 2; ix++) {
                        int x = 2 * ox + ix, y = 2 * oy + iy;
                        if (x > w - 1) x = w - 1;
                        if (y > h - 1) y = h - 1;
                        s += src[((size_t)y * w + x) * 3 + c];
                    }
                dst[((size_t)oy * ow + ox) * 3 + c] = s * 0.25f;
            }
}

static void downscale_f64(const double *src, int w, int h, double *dst) {
    int ow = (w + 1) / 2, oh = (h + 1) / 2;
    for (int oy = 0; oy < oh; oy++)
        for (int ox = 0; ox < ow; ox++)
            for (int c = 0; c < 3; c++) {
                double s = 0.0;
                for (int iy = 0; iy < 2; iy++)
                    for (int ix = 0; ix < 2; ix++) {
                        int x = 2 * ox + ix, y = 2 * oy + iy;
                        if (x > w - 1) x = w - 1;
                        if (y > h - 1) y = h - 1;
                        s += src[((size_t)y * w + x) * 3 + c];
                    }
                dst[((size_t)oy * ow + ox) * 3 + c] = s * 0.25;
            }
}

/* Opsin absorbance matrix and bias (xyb.rs:3-36). */
#define XM02 0.078f
#define XM00 0.30f
#define XM12 0.078f
#define XM10 0.23f
#define XM20 0.24342269f
#define XM21 0.20476745f
#define XB0 0.0037930734f
#define XB0_ROOT 0.1559542025327239180319220163705

/* Cube root as the CUDA engine computes it (ssim2_device.cuh s2_cbrtf):
 * Newton iteration on the reciprocal cube root r <- r + r (1 - x r^3) / 3
 * from W. Kahan's exponent-thirds bit seed, then y = x r^2 and one Newton
 * correction; selects instead of branches.  Multiplies and fmaf only, so it
 * rounds identically on every IEEE platform; <= 1 ulp from the true cube
 * root.  It stands in for libm's cbrtf (the reference calls libdevice cbrtf,
 * also <= 1 ulp). */
static inline float asf(uint32_t i) {
    float f;
    memcpy(&f, &i, 4);
    return f;
}
static inline uint32_t asu(float f) {
    uint32_t i;
    memcpy(&i, &f, 4);
    return i;
}
static inline float eng_cbrtf(float x) {
    const int pos = x > 0.0f, tiny = x < 0x1p-100f;
    float xs = tiny ? x * 0x1p102f : x;
    xs = pos ? xs : 1.0f;
    float r = asf(0x54a2fa8cu - asu(xs) / 3u);
    const float third = 0x1.555556p-2f;
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

/* a / b for b > 0 on the error maps' operand ranges, equal there to IEEE
 * division (checked in the tests): Newton reciprocal from the bit seed
 * 0x7EF311C3 - bits(b), three steps, then the residual correction of
 * q = a r that the engine's s2_div also ends with (the engine starts from
 * the hardware reciprocal approximation instead, which C cannot restate;
 * both give the IEEE quotient outside rare near-halfway cases). */
static inline float eng_div(float a, float b) {
    float r = asf(0x7EF311C3u - asu(b));
    r = fmaf(r, fmaf(-b, r, 1.0f), r);
    r = fmaf(r, fmaf(-b, r, 1.0f), r);
    r = fmaf(r, fmaf(-b, r, 1.0f), r);
    const float q = a * r;
    const float e = fmaf(-b, q, a);
    return fmaf(e, r, q);
}
float or_div(float a, float b) { return eng_div(a, b); }

/* p^(20/9) (= p^(1/0.45)) as the engine computes it (ssim2_device.cuh
 * s2_pow_20_9): p = m 2^e, m^(20/9) by a degree-7 polynomial in m - 1.5
 * (Horner, fmaf), times 2^(2e + k) 2^(r/9) with 2e = 9k + r.  <= 3.3 ulp. */
static inline float eng_pow2_r9(int r) {
    static const float T[9] = {0x1p+0f, 0x1.147eccp+0f, 0x1.2aa1a6p+0f, 0x1.428a3p+0f, 0x1.5c5cbcp+0f,
                               0x1.784086p+0f, 0x1.965feap+0f, 0x1.b6e8aep+0f, 0x1.da0c4p+0f};
    return T[r];
}
static inline float eng_pow_20_9(float p) {
    const int pos = p > 0.0f;
    const uint32_t b = asu(pos ? p : 1.0f);
    const int e = (int)((b >> 23) & 0xffu) - 127;
    const float t = asf((b & 0x7fffffu) | 0x3f800000u) - 1.5f;
    float y = 0x1.1eb37ap-12f;
    y = fmaf(y, t, -0x1.88e318p-11f);
    y = fmaf(y, t, 0x1.2713a6p-9f);
    y = fmaf(y, t, -0x1.37717ep-7f);
    y = fmaf(y, t, 0x1.2c9724p-4f);
    y = fmaf(y, t, 0x1.7c6f02p+0f);
    y = fmaf(y, t, 0x1.d2e55cp+1f);
    y = fmaf(y, t, 0x1.3b279ep+1f);
    const int n = 2 * e;
    const int k = (n + 261) / 9 - 29;
    const int r = n - 9 * k;
    y = y * eng_pow2_r9(r);
    y = y * asf((uint32_t)(2 * e + k + 127) << 23);
    return pos ? y : 0.0f;
}

float or_pow_20_9(float p) { return eng_pow_20_9(p); }

float or_cbrtf(float x) { return eng_cbrtf(x); }

/* The XYB cube root: the correctly rounded f32 cube root of x > 0 (0 for
 * x <= 0), from libm's double cbrt rounded once to f32.  The engine's XYB
 * cube root (ssim2_device.cuh s2_cbrtf_unit / s2_cbrtf_xyb) ends in a
 * Newton step with an exact residual, which gives this value in all but a
 * few cases per 10^5, and otherwise a neighbour within 1 ulp.  It stands in
 * for the reference's cbrtf (libdevice, xyb.rs:42-78; <= 1 ulp) in every
 * f32 mode. */
static inline float xyb_cbrtf(float x) { return x > 0.0f ? (float)cbrt((double)x) : 0.0f; }
float or_xyb_cbrtf(float x) { return xyb_cbrtf(x); }

/* The last step of the engine's XYB cube root (ssim2_device.cuh
 * s2_cbrt_step) from a seed r ~ x^(-1/3): y = x r^2, then one Newton step
 * with the residual y^3 - x formed from y^2 = hi + lo split exactly.  The
 * engine's seed comes from the SFU, which C cannot restate; the tests feed
 * this step perturbed exact seeds to show that its result is the correctly
 * rounded cube root whatever the seed's last bits. */
float or_cbrt_step(float x, float r) {
    float y = x * r;
    y = y * r;
    const float hi = y * y;
    const float lo = fmaf(y, y, -hi);
    float e = fmaf(hi, y, -x);
    e = fmaf(lo, y, e);
    const float c = (r * r) * 0x1.555556p-2f;
    return fmaf(-e, c, y);
}

static inline void xyb_f32(float r, float g, float b, float out[3]) {
    const float m01 = 1.0f - XM02 - XM00, m11 = 1.0f - XM12 - XM10, m22 = 1.0f - XM20 - XM21;
    const float root = 0.1559542025327239180319220163705f;
    float rg = fmaf(XM00, r, fmaf(m01, g, fmaf(XM02, b, XB0)));
    float gr = fmaf(XM10, r, fmaf(m11, g, fmaf(XM12, b, XB0)));
    float bb = fmaf(XM20, r, fmaf(XM21, g, fmaf(m22, b, XB0)));
    rg = xyb_cbrtf(rg) - root;
    gr = xyb_cbrtf(gr) - root;
    bb = xyb_cbrtf(bb) - root;
    float x = 0.5f * (rg - gr), y = 0.5f * (rg + gr);
    out[0] = fmaf(x, 14.0f, 0.42f);
    out[1] = y + 0.01f;
    out[2] = (bb - y) + 0.55f;
}

static inline void xyb_f64(double r, double g, double b, double out[3]) {
    const double m00 = 0.30, m02 = 0.078, m01 = 1.0 - 0.078 - 0.30;
    const double m10 = 0.23, m12 = 0.078, m11 = 1.0 - 0.078 - 0.23;
    const double m20 = 0.24342269, m21 = 0.20476745, m22 = 1.0 - 0.24342269 - 0.20476745;
    const double bias = 0.0037930734, root = cbrt(0.0037930734);
    double rg = m00 * r + m01 * g + m02 * b + bias;
    double gr = m10 * r + m11 * g + m12 * b + bias;
    double bb = m20 * r + m21 * g + m22 * b + bias;
    rg = cbrt(rg > 0.0 ? rg : 0.0) - root;
    gr = cbrt(gr > 0.0 ? gr : 0.0) - root;
    bb = cbrt(bb > 0.0 ? bb : 0.0) - root;
    double x = 0.5 * (rg - gr), y = 0.5 * (rg + gr);
    out[0] = x * 14.0 + 0.42;
    out[1] = y + 0.01;
    out[2] = bb - y + 0.55;
}

void or_linear_to_xyb_f32(const float *src, size_t n, float *dst) {
    for (size_t p = 0; p < n; p++) xyb_f32(src[3 * p], src[3 * p + 1], src[3 * p + 2], dst + 3 * p);
}

/* ------------------------------------------------------------------------ */
/* Blur                                                                      */
/* ------------------------------------------------------------------------ */

/* One IIR walk over `len` samples with stride `st` (blur.rs:95-136 form:
 * out = fma(MUL_PREV, prev, fma(MUL_PREV2, prev2, sum * MUL_IN))).
 * The recursion starts at n = -N+1 with zero state; inputs beyond either
 * end read as zero. */
static void iir_walk_gpu(const float *in, size_t st, int len, float *out, size_t ost) {
    const int N = g_bc.radius;
    float p1 = 0, p3 = 0, p5 = 0, q1 = 0, q3 = 0, q5 = 0; /* prev, prev2 */
    for (int n = -N + 1; n < len; n++) {
        int left = n - N - 1, right = n + N - 1;
        float lv = left >= 0 ? in[(size_t)left * st] : 0.0f;
        float rv = right < len ? in[(size_t)right * st] : 0.0f;
        float sum = lv + rv;
        float o1 = sum * g_bc.mul_in[0], o3 = sum * g_bc.mul_in[1], o5 = sum * g_bc.mul_in[2];
        o1 = fmaf(g_bc.mul_prev2[0], q1, o1);
        o3 = fmaf(g_bc.mul_prev2[1], q3, o3);
        o5 = fmaf(g_bc.mul_prev2[2], q5, o5);
        q1 = p1; q3 = p3; q5 = p5;
        o1 = fmaf(g_bc.mul_prev[0], p1, o1);
        o3 = fmaf(g_bc.mul_prev[1], p3, o3);
        o5 = fmaf(g_bc.mul_prev[2], p5, o5);
        p1 = o1; p3 = o3; p5 = o5;
        if (n >= 0) out[(size_t)n * ost] = (o1 + o3) + o5;
    }
}

/* cpu.rs:1054-1115 vertical form: out = fma(sum, VERT_MUL_IN, -fma(prev, VERT_MUL_PREV, prev2)). */
static void iir_walk_vert(const float *in, size_t st, int len, float *out, size_t ost) {
    const int N = g_bc.radius;
    float p[3] = {0, 0, 0}, q[3] = {0, 0, 0};
    for (int n = -N + 1; n < len; n++) {
        int top = n - N - 1, bot = n + N - 1;
        float tv = top >= 0 ? in[(size_t)top * st] : 0.0f;
        float bv = bot < len ? in[(size_t)bot * st] : 0.0f;
        float sum = tv + bv;
        float o[3];
        for (int k = 0; k < 3; k++) {
            float t = fmaf(p[k], g_bc.vert_mul_prev[k], q[k]);
            o[k] = fmaf(sum, g_bc.vert_mul_in[k], -t);
        }
        for (int k = 0; k < 3; k++) { q[k] = p[k]; p[k] = o[k]; }
        if (n >= 0) out[(size_t)n * ost] = (o[0] + o[1]) + o[2];
    }
}

/* The f32 FIR in the order the CUDA kernels use:
 * acc = t4*(x[-4]+x[4]); acc = fma(t3, x[-3]+x[3], acc); ... ;
 * acc = fma(t0, x[0], acc).  Samples outside [0, len) read as zero. */
static void fir_walk_f32(const float *in, size_t st, int len, float *out, size_t ost) {
    float t[5];
    for (int k = 0; k < 5; k++) t[k] = (float)g_bc.fir[k];
    for (int n = 0; n < len; n++) {
        float xm[5], xp[5];
        for (int k = 0; k < 5; k++) {
            int a = n - k, b = n + k;
            xm[k] = a >= 0 ? in[(size_t)a * st] : 0.0f;
            xp[k] = b < len ? in[(size_t)b * st] : 0.0f;
        }
        float acc = t[4] * (xm[4] + xp[4]);
        acc = fmaf(t[3], xm[3] + xp[3], acc);
        acc = fmaf(t[2], xm[2] + xp[2], acc);
        acc = fmaf(t[1], xm[1] + xp[1], acc);
        acc = fmaf(t[0], xm[0], acc);
        out[(size_t)n * ost] = acc;
    }
}

void or_blur_plane_f32(const float *src, int w, int h, int mode, float *dst) {
    init_blur_consts();
    float *tmp = (float *)malloc((size_t)w * h * sizeof(float));
    if (mode == OR_MODE_CPU32) {
        for (int y = 0; y < h; y++) iir_walk_gpu(src + (size_t)y * w, 1, w, tmp + (size_t)y * w, 1);
        for (int x = 0; x < w; x++) iir_walk_vert(tmp + x, (size_t)w, h, dst + x, (size_t)w);
    } else if (mode == OR_MODE_FIR32) {
        for (int x = 0; x < w; x++) fir_walk_f32(src + x, (size_t)w, h, tmp + x, (size_t)w);
        for (int y = 0; y < h; y++) fir_walk_f32(tmp + (size_t)y * w, 1, w, dst + (size_t)y * w, 1);
    } else { /* OR_MODE_CUDA32: vertical walk, then a walk along rows */
        for (int x = 0; x < w; x++) iir_walk_gpu(src + x, (size_t)w, h, tmp + x, (size_t)w);
        for (int y = 0; y < h; y++) iir_walk_gpu(tmp + (size_t)y * w, 1, w, dst + (size_t)y * w, 1);
    }
    free(tmp);
}

static void fir_walk_f64(const double *in, size_t st, int len, double *out, size_t ost) {
    for (int n = 0; n < len; n++) {
        double acc = 0.0;
        for (int k = 4; k >= 1; k--) {
            int a = n - k, b = n + k;
            double s = (a >= 0 ? in[(size_t)a * st] : 0.0) + (b < len ? in[(size_t)b * st] : 0.0);
            acc += g_bc.fir[k] * s;
        }
        acc += g_bc.fir[0] * in[(size_t)n * st];
        out[(size_t)n * ost] = acc;
    }
}

void or_blur_plane_f64(const double *src, int w, int h, double *dst) {
    init_blur_consts();
    double *tmp = (double *)malloc((size_t)w * h * sizeof(double));
    for (int x = 0; x < w; x++) fir_walk_f64(src + x, (size_t)w, h, tmp + x, (size_t)w);
    for (int y = 0; y < h; y++) fir_walk_f64(tmp + (size_t)y * w, 1, w, dst + (size_t)y * w, 1);
    free(tmp);
}

/* ------------------------------------------------------------------------ */
/* Scoring                                                                   */
/* ------------------------------------------------------------------------ */

/* WEIGHT[108] of the published SSIMULACRA2 (ssimulacra2-cuda/src/lib.rs:1023-1153,
 * cpu.rs:729-838), indexed c*36 + scale*6 + norm*3 + map. */
static const double WEIGHT[108] = {
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

void or_weights(double w[108]) { memcpy(w, WEIGHT, sizeof WEIGHT); }

double or_score_from_stats(const double stats[108]) {
    double s = 0.0;
    for (int i = 0; i < 108; i++) s = fma(WEIGHT[i], fabs(stats[i]), s);
    s *= 0.9562382616834844;
    s = fma(6.248496625763138e-5 * s * s, s, fma(2.326765642916932, s, -0.020884521182843837 * s * s));
    if (s > 0.0) return fma(pow(s, 0.6276336467831387), -10.0, 100.0);
    return 100.0;
}

/* Note: the two non-ALL6 rules differ only in which size is tested.  Under
 * OR_SCALES_CPU, scale s (s >= 1) is scored when scale s-1 is at least 8x8
 * (so a 16x16 input scores 16, 8 and 4); under OR_SCALES_MIN8 only scales of
 * at least 8x8 are scored (16 and 8). */
static int scales_for(int w, int h, int rule) {
    if (rule == OR_SCALES_ALL6) return NSCALES;
    if (w < 8 || h < 8) return 0;
    if (rule == OR_SCALES_MIN8) {
        int n = 0;
        while (n < NSCALES && w >= 8 && h >= 8) {
            n++;
            w = (w + 1) / 2;
            h = (h + 1) / 2;
        }
        return n;
    }
    int n = 1, pw = w, ph = h;
    for (int s = 1; s < NSCALES; s++) {
        if (pw < 8 || ph < 8) break;
        n++;
        pw = (pw + 1) / 2;
        ph = (ph + 1) / 2;
    }
    return n;
}

int or_num_scales(int w, int h, int rule) { return scales_for(w, h, rule); }

/* Per-scale f32 scoring.  xr/xd: planar XYB (3 planes of n). */
static void score_scale_f32(const float *xr, const float *xd, int w, int h, int mode,
                            double st[18], double sums[18]) {
    size_t n = (size_t)w * h;
    float *mul = (float *)malloc(n * sizeof(float));
    float *bl = (float *)malloc(5 * n * sizeof(float));
    for (int c = 0; c < 3; c++) {
        const float *a = xr + c * n, *b = xd + c * n;
        float *mu1 = bl, *mu2 = bl + n, *s11 = bl + 2 * n, *s22 = bl + 3 * n, *s12 = bl + 4 * n;
        for (size_t i = 0; i < n; i++) mul[i] = a[i] * a[i];
        or_blur_plane_f32(mul, w, h, mode, s11);
        for (size_t i = 0; i < n; i++) mul[i] = b[i] * b[i];
        or_blur_plane_f32(mul, w, h, mode, s22);
        for (size_t i = 0; i < n; i++) mul[i] = a[i] * b[i];
        or_blur_plane_f32(mul, w, h, mode, s12);
        or_blur_plane_f32(a, w, h, mode, mu1);
        or_blur_plane_f32(b, w, h, mode, mu2);
        double acc[6] = {0}; /* ssim, art, det sums; then their 4th-power sums */
        const float C2 = 0.0009f;
        for (size_t i = 0; i < n; i++) {
            float m1 = mu1[i], m2 = mu2[i];
            float mu11 = m1 * m1, mu22 = m2 * m2, mu12 = m1 * m2, md = m1 - m2;
            float num_m = fmaf(md, -md, 1.0f);
            float num_s = fmaf(2.0f, s12[i] - mu12, C2);
            float den_s = ((s11[i] - mu11) + (s22[i] - mu22)) + C2;
            if (mode == OR_MODE_CPU32) {
                double d = 1.0 - (double)((num_m * num_s) / den_s);
                if (d < 0.0) d = 0.0;
                acc[0] += d;
                acc[3] += (d * d) * (d * d);
                double d1 = (1.0 + (double)fabsf(b[i] - m2)) / (1.0 + (double)fabsf(a[i] - m1)) - 1.0;
                double ar = d1 > 0.0 ? d1 : 0.0, de = -d1 > 0.0 ? -d1 : 0.0;
                acc[1] += ar;
                acc[4] += (ar * ar) * (ar * ar);
                acc[2] += de;
                acc[5] += (de * de) * (de * de);
            } else {
                float d = 1.0f - (num_m * num_s) / den_s;
                d = d > 0.0f ? d : 0.0f;
                float den = 1.0f / (1.0f + fabsf(a[i] - m1));
                float num = 1.0f + fabsf(b[i] - m2);
                float d1 = fmaf(num, den, -1.0f);
                float ar = d1 > 0.0f ? d1 : 0.0f, de = -d1 > 0.0f ? -d1 : 0.0f;
                float v[3] = {d, ar, de};
                for (int k = 0; k < 3; k++) {
                    float sq = v[k] * v[k];
                    acc[k] += (double)v[k];
                    acc[3 + k] += (double)(sq * sq);
                }
            }
        }
        double inv = 1.0 / (double)n;
        for (int k = 0; k < 3; k++) {
            st[c * 6 + k] = acc[k] * inv;
            st[c * 6 + 3 + k] = sqrt(sqrt(acc[3 + k] * inv));
            sums[c * 6 + k] = acc[k];
            sums[c * 6 + 3 + k] = acc[3 + k];
        }
    }
    free(mul);
    free(bl);
}

/* ---- FIR32: the arithmetic of this repository's fused CUDA pass --------- */
/* f32 taps of the exact form, as compiled into the kernels. */
static const float FT0 = 0x1.0ef8d6p-2f, FT1 = 0x1.b413e8p-3f, FT2 = 0x1.bfd672p-4f,
                   FT3 = 0x1.2700c8p-5f, FT4 = 0x1.347d7p-7f;

static inline float fir9f(float a0, float a1, float a2, float a3, float a4, float a5, float a6,
                          float a7, float a8) {
    float acc = FT4 * (a0 + a8);
    acc = fmaf(FT3, a1 + a7, acc);
    acc = fmaf(FT2, a2 + a6, acc);
    acc = fmaf(FT1, a3 + a5, acc);
    return fmaf(FT0, a4, acc);
}

/* Response of the FIR to a constant 1 under zero padding at x in [0, n),
 * from double prefix sums of the exact taps; 1.0f in the interior. */
static float border_gain_f(int x, int n) {
    int lo = x < 4 ? x : 4, hi = (n - 1 - x) < 4 ? (n - 1 - x) : 4;
    if (lo == 4 && hi == 4) return 1.0f;
    static const double S[5] = {0x1.0ef8d5c79cdafp-2, 0x1.e902c9b3e2946p-2, 0x1.2c7c332eb15f4p-1,
                                0x1.3eec3fae31770p-1, 0x1.43be3571e736ap-1};
    double s = S[lo] + S[hi];
    return (float)(s - S[0]);
}

#define FIR_TW 120  /* output columns per tile of the fused pass */
#define FIR_BAND 64 /* rows per shift band */
#define FIR_SEG 8   /* pixels per f32 partial sum (one horizontal task) */

static inline float fmaxf0(float v) { return v > 0.0f ? v : 0.0f; }

/* One scale in FIR32 arithmetic (the fused CUDA pass of this repository,
 * csrc/ssim2_kernels.cu fused_kernel).  xr/xd: planar XYB (3 planes of W*H).
 * Tiles of 120 columns x 64-row bands share one shift per channel (the
 * reference XYB at the tile's first column and the band's first row):
 * x' = ref - shift, y' = dis - shift (0 outside the image).  Four planes are
 * blurred, in the kernels' 9-tap order, vertical then horizontal: x', the
 * difference e = ref - dis, e^2 and x'y'.  With mu1 = blur(x'),
 * md = blur(e) = mu1 - mu2, mu2 = mu1 - md, the SSIM terms are
 *   num_s = 2 (blur(x'y') - mu1 mu2) + C2      (+ the border correction)
 *   Vd    = blur(e^2) - md^2                   (var1 + var2 - 2 cov)
 *   den   = Vd + num_s
 *   d     = (Vd + md^2 num_s) / den           (= 1 - num_m num_s / den)
 * so the small difference between the two images is blurred as such, not
 * recovered from the difference of two large moments.  Maps are pooled in
 * f32 over 8-pixel segments of a row, then in f64.  sums[c*6 + n*3 + m].
 * With `maps` (9 planes of W*H, [channel][ssim, artifact, detail]) every
 * pixel's error values are stored too. */
static void score_scale_fir32(const float *xr, const float *xd, int W, int H, double sums[18], float *maps) {
    const int TC = FIR_TW + 8, TR = FIR_BAND + 8;
    const int NP = 4; /* x', e, e^2, x'y' */
    float *P = (float *)malloc((size_t)NP * TC * TR * sizeof(float));
    float *V = (float *)malloc((size_t)NP * TC * FIR_BAND * sizeof(float));
    float *X = (float *)malloc((size_t)2 * TC * FIR_BAND * sizeof(float));
    double acc[18] = {0};
    size_t n = (size_t)W * H;
    const float C2 = 0.0009f;
    for (int c = 0; c < 3; c++) {
        const float *a = xr + c * n, *b = xd + c * n;
        for (int y0 = 0; y0 < H; y0 += FIR_BAND) {
            int y1 = y0 + FIR_BAND < H ? y0 + FIR_BAND : H;
            for (int x0 = 0; x0 < W; x0 += FIR_TW) {
                const float cv = a[(size_t)y0 * W + x0];
                for (int r = 0; r < (y1 - y0) + 8; r++) {
                    int y = y0 - 4 + r;
                    for (int k = 0; k < TC; k++) {
                        int x = x0 - 4 + k;
                        float vx = 0, ve = 0, vee = 0, vxy = 0;
                        if (x >= 0 && x < W && y >= 0 && y < H) {
                            const float ra = a[(size_t)y * W + x], rb = b[(size_t)y * W + x];
                            vx = ra - cv;
                            ve = ra - rb;
                            vee = ve * ve;
                            vxy = vx * (rb - cv);
                        }
                        size_t o = (size_t)r * TC + k;
                        P[0 * TC * TR + o] = vx;
                        P[1 * TC * TR + o] = ve;
                        P[2 * TC * TR + o] = vee;
                        P[3 * TC * TR + o] = vxy;
                    }
                }
                for (int r = 0; r < y1 - y0; r++)
                    for (int k = 0; k < TC; k++) {
                        for (int p = 0; p < NP; p++) {
                            const float *q = P + (size_t)p * TC * TR + k;
                            V[(size_t)p * TC * FIR_BAND + (size_t)r * TC + k] =
                                fir9f(q[(size_t)(r + 0) * TC], q[(size_t)(r + 1) * TC], q[(size_t)(r + 2) * TC],
                                      q[(size_t)(r + 3) * TC], q[(size_t)(r + 4) * TC], q[(size_t)(r + 5) * TC],
                                      q[(size_t)(r + 6) * TC], q[(size_t)(r + 7) * TC], q[(size_t)(r + 8) * TC]);
                        }
                        /* raw x' and e of the output row */
                        X[(size_t)0 * TC * FIR_BAND + (size_t)r * TC + k] = P[0 * TC * TR + (size_t)(r + 4) * TC + k];
                        X[(size_t)1 * TC * FIR_BAND + (size_t)r * TC + k] = P[1 * TC * TR + (size_t)(r + 4) * TC + k];
                    }
                for (int r = 0; r < y1 - y0; r++) {
                    int y = y0 + r;
                    float bv = border_gain_f(y, H);
                    for (int c0 = 0; c0 < FIR_TW; c0 += FIR_SEG) {
                        if (x0 + c0 >= W) break;
                        float fs[3] = {0, 0, 0}, f4[3] = {0, 0, 0};
                        for (int j = 0; j < FIR_SEG; j++) {
                            int xx = x0 + c0 + j;
                            if (xx >= W) break;
                            float o[4];
                            for (int p = 0; p < NP; p++) {
                                const float *q = V + (size_t)p * TC * FIR_BAND + (size_t)r * TC + c0 + j;
                                o[p] = fir9f(q[0], q[1], q[2], q[3], q[4], q[5], q[6], q[7], q[8]);
                            }
                            float m1 = o[0], md = o[1], ed2 = o[2], s12 = o[3];
                            float m2 = m1 - md;
                            float xp = X[(size_t)r * TC + c0 + j + 4];
                            float ep = X[(size_t)TC * FIR_BAND + (size_t)r * TC + c0 + j + 4];
                            float bh = border_gain_f(xx, W);
                            float corr = (bh == 1.0f && bv == 1.0f) ? 0.0f : (float)(1.0 - (double)bh * (double)bv);
                            float kk = cv * corr;
                            float h = (m1 + m2) + (cv - kk);
                            float cov = fmaf(kk, h, fmaf(-m1, m2, s12));
                            float num_s = fmaf(2.0f, cov, C2);
                            float vd = fmaf(-md, md, ed2);
                            float den = vd + num_s;
                            float nn = fmaf(md * md, num_s, vd);
                            float d = fmaxf0(eng_div(nn, den));
                            float t1 = xp - m1, u = ep - md;
                            float t2 = t1 - u; /* y' - mu2 */
                            float aa = fabsf(t1 + kk);
                            float bb = fabsf(t2 + kk);
                            float d1 = eng_div(bb - aa, 1.0f + aa);
                            float v[3] = {d, fmaxf0(d1), fmaxf0(-d1)};
                            if (maps)
                                for (int m = 0; m < 3; m++) maps[((size_t)(3 * c + m) * H + y) * W + xx] = v[m];
                            for (int m = 0; m < 3; m++) {
                                fs[m] += v[m];
                                float q = v[m] * v[m];
                                f4[m] = fmaf(q, q, f4[m]);
                            }
                        }
                        for (int m = 0; m < 3; m++) {
                            acc[c * 6 + m] += (double)fs[m];
                            acc[c * 6 + 3 + m] += (double)f4[m];
                        }
                    }
                }
            }
        }
    }
    memcpy(sums, acc, sizeof acc);
    free(P);
    free(V);
    free(X);
}

static void to_planar_xyb_f32(const float *lin, size_t n, float *pl) {
    for (size_t p = 0; p < n; p++) {
        float o[3];
        xyb_f32(lin[3 * p], lin[3 * p + 1], lin[3 * p + 2], o);
        pl[p] = o[0];
        pl[n + p] = o[1];
        pl[2 * n + p] = o[2];
    }
}

static int ssim2_linear_impl(const float *ref, const float *dis, int w, int h, int mode, int rule,
                             double stats[108], double sums_out[108], double *score, int *n_scales,
                             int maps_scale, float *maps) {
    init_blur_consts();
    if (w < 1 || h < 1) return -1;
    if (rule != OR_SCALES_ALL6 && (w < 8 || h < 8)) return -1;
    int ns = scales_for(w, h, rule);
    double st[108] = {0}, su[108] = {0};
    size_t n0 = (size_t)w * h;
    float *r = (float *)malloc(n0 * 3 * sizeof(float)), *d = (float *)malloc(n0 * 3 * sizeof(float));
    float *r2 = (float *)malloc(n0 * 3 * sizeof(float)), *d2 = (float *)malloc(n0 * 3 * sizeof(float));
    float *pr = (float *)malloc(n0 * 3 * sizeof(float)), *pd = (float *)malloc(n0 * 3 * sizeof(float));
    memcpy(r, ref, n0 * 3 * sizeof(float));
    memcpy(d, dis, n0 * 3 * sizeof(float));
    int cw = w, ch = h;
    for (int s = 0; s < ns; s++) {
        if (s > 0) {
            or_downscale_f32(r, cw, ch, r2);
            or_downscale_f32(d, cw, ch, d2);
            cw = (cw + 1) / 2;
            ch = (ch + 1) / 2;
            float *t = r; r = r2; r2 = t;
            t = d; d = d2; d2 = t;
        }
        size_t n = (size_t)cw * ch;
        to_planar_xyb_f32(r, n, pr);
        to_planar_xyb_f32(d, n, pd);
        double sst[18], ssu[18];
        if (mode == OR_MODE_FIR32) {
            score_scale_fir32(pr, pd, cw, ch, ssu, (maps && s == maps_scale) ? maps : NULL);
            double inv = 1.0 / (double)n;
            for (int c = 0; c < 3; c++)
                for (int k = 0; k < 3; k++) {
                    sst[c * 6 + k] = ssu[c * 6 + k] * inv;
                    sst[c * 6 + 3 + k] = sqrt(sqrt(ssu[c * 6 + 3 + k] * inv));
                }
        } else {
            score_scale_f32(pr, pd, cw, ch, mode, sst, ssu);
        }
        for (int c = 0; c < 3; c++)
            for (int k = 0; k < 6; k++) {
                st[c * 36 + s * 6 + k] = sst[c * 6 + k];
                su[c * 36 + s * 6 + k] = ssu[c * 6 + k];
            }
    }
    free(r); free(d); free(r2); free(d2); free(pr); free(pd);
    if (stats) memcpy(stats, st, sizeof st);
    if (sums_out) memcpy(sums_out, su, sizeof su);
    if (n_scales) *n_scales = ns;
    if (score) {
        if (mode == OR_MODE_CUDA32) {
            /* lib.rs:1155-1189: weight each stat, sum in the scores[] memory
             * order (scale-major: scale*18 + kind*3 + c), then remap. */
            double acc = 0.0;
            for (int sc = 0; sc < NSCALES; sc++)
                for (int kind = 0; kind < 6; kind++)
                    for (int c = 0; c < 3; c++) {
                        int i = c * 36 + sc * 6 + kind;
                        acc += fabs(st[i]) * WEIGHT[i];
                    }
            acc *= 0.9562382616834844;
            acc = fma(6.248496625763138e-5 * acc * acc, acc,
                      fma(2.326765642916932, acc, -0.020884521182843837 * acc * acc));
            *score = acc > 0.0 ? fma(pow(acc, 0.6276336467831387), -10.0, 100.0) : 100.0;
        } else {
            *score = or_score_from_stats(st);
        }
    }
    return 0;
}

int or_ssim2_linear(const float *ref, const float *dis, int w, int h, int mode, int rule,
                    double stats[108], double sums_out[108], double *score, int *n_scales) {
    return ssim2_linear_impl(ref, dis, w, h, mode, rule, stats, sums_out, score, n_scales, -1, NULL);
}

/* FIR32 error maps of one scale: 9 planes of w_s * h_s floats,
 * [channel X, Y, B][ssim error, artifact, detail loss], row-major. */
int or_ssim2_maps_fir32(const float *ref, const float *dis, int w, int h, int rule, int scale, float *maps) {
    int ns = scales_for(w, h, rule);
    if (scale < 0 || scale >= ns) return -1;
    return ssim2_linear_impl(ref, dis, w, h, OR_MODE_FIR32, rule, NULL, NULL, NULL, NULL, scale, maps);
}

/* FP64 oracle. */
int or_ssim2_linear_f64(const double *ref, const double *dis, int w, int h, int rule,
                        double stats[108], double sums_out[108], double *score, int *n_scales) {
    init_blur_consts();
    if (w < 1 || h < 1) return -1;
    if (rule != OR_SCALES_ALL6 && (w < 8 || h < 8)) return -1;
    int ns = scales_for(w, h, rule);
    double st[108] = {0}, su[108] = {0};
    size_t n0 = (size_t)w * h;
    double *r = (double *)malloc(n0 * 3 * sizeof(double)), *d = (double *)malloc(n0 * 3 * sizeof(double));
    double *r2 = (double *)malloc(n0 * 3 * sizeof(double)), *d2 = (double *)malloc(n0 * 3 * sizeof(double));
    double *pr = (double *)malloc(n0 * 3 * sizeof(double)), *pd = (double *)malloc(n0 * 3 * sizeof(double));
    double *mul = (double *)malloc(n0 * sizeof(double)), *bl = (double *)malloc(5 * n0 * sizeof(double));
    memcpy(r, ref, n0 * 3 * sizeof(double));
    memcpy(d, dis, n0 * 3 * sizeof(double));
    int cw = w, ch = h;
    for (int s = 0; s < ns; s++) {
        if (s > 0) {
            downscale_f64(r, cw, ch, r2);
            downscale_f64(d, cw, ch, d2);
            cw = (cw + 1) / 2;
            ch = (ch + 1) / 2;
            double *t = r; r = r2; r2 = t;
            t = d; d = d2; d2 = t;
        }
        size_t n = (size_t)cw * ch;
        for (size_t p = 0; p < n; p++) {
            double o[3];
            xyb_f64(r[3 * p], r[3 * p + 1], r[3 * p + 2], o);
            pr[p] = o[0]; pr[n + p] = o[1]; pr[2 * n + p] = o[2];
            xyb_f64(d[3 * p], d[3 * p + 1], d[3 * p + 2], o);
            pd[p] = o[0]; pd[n + p] = o[1]; pd[2 * n + p] = o[2];
        }
        for (int c = 0; c < 3; c++) {
            const double *a = pr + c * n, *b = pd + c * n;
            double *mu1 = bl, *mu2 = bl + n, *s11 = bl + 2 * n, *s22 = bl + 3 * n, *s12 = bl + 4 * n;
            for (size_t i = 0; i < n; i++) mul[i] = a[i] * a[i];
            or_blur_plane_f64(mul, cw, ch, s11);
            for (size_t i = 0; i < n; i++) mul[i] = b[i] * b[i];
            or_blur_plane_f64(mul, cw, ch, s22);
            for (size_t i = 0; i < n; i++) mul[i] = a[i] * b[i];
            or_blur_plane_f64(mul, cw, ch, s12);
            or_blur_plane_f64(a, cw, ch, mu1);
            or_blur_plane_f64(b, cw, ch, mu2);
            long double acc[6] = {0};
            for (size_t i = 0; i < n; i++) {
                double m1 = mu1[i], m2 = mu2[i], md = m1 - m2;
                double num_m = 1.0 - md * md;
                double num_s = 2.0 * (s12[i] - m1 * m2) + 0.0009;
                double den_s = (s11[i] - m1 * m1) + (s22[i] - m2 * m2) + 0.0009;
                double dd = 1.0 - num_m * num_s / den_s;
                if (dd < 0.0) dd = 0.0;
                double d1 = (1.0 + fabs(b[i] - m2)) / (1.0 + fabs(a[i] - m1)) - 1.0;
                double ar = d1 > 0.0 ? d1 : 0.0, de = d1 < 0.0 ? -d1 : 0.0;
                double v[3] = {dd, ar, de};
                for (int k = 0; k < 3; k++) {
                    acc[k] += v[k];
                    acc[3 + k] += (long double)(v[k] * v[k]) * (long double)(v[k] * v[k]);
                }
            }
            double inv = 1.0 / (double)n;
            for (int k = 0; k < 3; k++) {
                int i = c * 36 + s * 6;
                st[i + k] = (double)acc[k] * inv;
                st[i + 3 + k] = sqrt(sqrt((double)acc[3 + k] * inv));
                su[i + k] = (double)acc[k];
                su[i + 3 + k] = (double)acc[3 + k];
            }
        }
    }
    free(r); free(d); free(r2); free(d2); free(pr); free(pd); free(mul); free(bl);
    if (stats) memcpy(stats, st, sizeof st);
    if (sums_out) memcpy(sums_out, su, sizeof su);
    if (n_scales) *n_scales = ns;
    if (score) *score = or_score_from_stats(st);
    return 0;
}
