/*
 * ssim2_oracle.h -- CPU restatement of the SSIMULACRA2 hot path of
 * imazen/turbo-metrics.  TEST INFRASTRUCTURE ONLY: the parity tests, the
 * smoke check and the CPU-baseline leg of the benchmark call it as the
 * checker.  The product path (the CUDA library) never links or calls it.
 *
 * Three arithmetic modes restate three implementations of the same metric:
 *
 *   OR_MODE_FP64     FP64 oracle.  Every stage in double; the recursive
 *                    Gaussian is applied in its exact closed form (the 9-tap
 *                    symmetric FIR the recursion equals in exact arithmetic);
 *                    pooled sums in long double.
 *   OR_MODE_CUDA32   f32 mirror of crates/ssimulacra2-cuda (the drop-in
 *                    target): IIR walked down columns first, then along
 *                    rows (ssimulacra2-cuda/src/lib.rs:897-947 runs the
 *                    vertical kernel, transposes, runs it again), FMA
 *                    placement of ssimulacra2-cuda-kernel/src/blur.rs:95-136
 *                    and error_maps.rs:36-59, f64 sums of f32 d and of the
 *                    f32 (d*d)*(d*d) (NPP Sqr + SqrIP, lib.rs:986-1016).
 *   OR_MODE_CPU32    f32 mirror of the CPU crate the repo validates against
 *                    (ssimulacra2-cuda/examples/cpu.rs, extracted from
 *                    rust-av/ssimulacra2 0.5.1): horizontal IIR first
 *                    (cpu.rs:967-1022), vertical in the VERT_* form
 *                    (cpu.rs:1054-1115), d and d1 pooled in f64
 *                    (cpu.rs:581-683).  This is the timed CPU baseline.
 *   OR_MODE_FIR32    f32 restatement of the fused CUDA pass of this
 *                    repository: the separable 9-tap FIR in its operation
 *                    order (vertical taps, then horizontal taps) on values
 *                    shifted by one anchor per 120-column x 64-row block;
 *                    four blurred planes -- the shifted reference x', the
 *                    difference e = ref - dis, e^2 and x'y' -- and the SSIM
 *                    error formed from the blurred difference (no
 *                    cancellation between large moments); f32 sums over
 *                    8-pixel row segments.  Used to check the device kernels.
 *
 * Pyramid stop rules (which scales are scored):
 *   OR_SCALES_CPU    cpu.rs:359-361 -- before producing scale s>0, stop if
 *                    the previous scale is narrower or shorter than 8.
 *   OR_SCALES_MIN8   ssim2-gpu/src/pipeline.rs:194-206 -- a scale is scored
 *                    only if it is itself at least 8x8.
 *   OR_SCALES_ALL6   ssimulacra2-cuda/src/lib.rs:138-143 -- always 6 scales.
 *
 * The 108 statistics use the weight-table order of the reference
 * (cpu.rs:838-852): index = c*36 + scale*6 + norm*3 + map, with
 * norm 0 = mean (L1), 1 = fourth root of the mean fourth power (L4), and
 * map 0 = SSIM error, 1 = artifact (ringing), 2 = detail loss (blur).
 * Unscored scales hold 0.
 */
#ifndef SSIM2_ORACLE_H
#define SSIM2_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { OR_MODE_FP64 = 0, OR_MODE_CUDA32 = 1, OR_MODE_CPU32 = 2, OR_MODE_FIR32 = 3 };
enum { OR_SCALES_CPU = 0, OR_SCALES_MIN8 = 1, OR_SCALES_ALL6 = 2 };

/* Recursive-Gaussian constants (f32, as the reference kernels use them) and
 * the FIR taps of the exact form (double).  Returns the radius N. */
int or_blur_constants(float mul_in[3], float mul_prev[3], float mul_prev2[3],
                      float vert_mul_in[3], float vert_mul_prev[3],
                      double fir_taps[5]);

/* Input conversions.  Output is packed interleaved RGB (3 floats/pixel). */
void or_srgb8_lut(float lut[256]);
void or_srgb8_to_linear(const uint8_t *src, size_t n_samples, float *dst);
void or_srgb8_to_linear_f64(const uint8_t *src, size_t n_samples, double *dst);
/* NV12, 8 bit, BT.709 matrix, limited range, nearest 2x2 chroma. */
/* 4:2:0 biplanar YUV: bits 8 (NV12) or 16 (P016), matrix 0 BT.709 / 1 BT.601-525 /
 * 2 BT.601-625, full 0 limited / 1 full range; pitch in bytes. */
void or_yuv420_to_linear(const void *y, const void *uv, size_t pitch, int w, int h, int bits, int matrix,
                         int full, float *dst);
void or_yuv420_to_linear_f64(const void *y, const void *uv, size_t pitch, int w, int h, int bits, int matrix,
                             int full, double *dst);
void or_nv12_to_linear(const uint8_t *y, const uint8_t *uv, size_t pitch,
                       int w, int h, float *dst);
void or_nv12_to_linear_f64(const uint8_t *y, const uint8_t *uv, size_t pitch,
                           int w, int h, double *dst);
/* Packed RGB, uint16 holding `bits`-bit code values, BT.2020 primaries and
 * BT.709/BT.2020 transfer, converted to linear BT.709 RGB, clamped >= 0. */
/* The reference's f32 derivation of the 4:2:0 coefficients (y, r, b, g1, g2;
 * cuda-colorspace-kernel/src/lib.rs:188-221), luma minimum and chroma
 * neutral value; matrix 0 BT.709, 1 BT.601-525, 2 BT.601-625. */
void or_yuv_coeffs_ref_f32(int matrix, int full, int bits, float c[5], int *ymin, int *neutral);
/* alpha - 1, 1 / alpha, threshold, 1 / 4.5 of the f32 BT.709 inverse OETF. */
void or_bt709_eotf_consts(float out[4]);
void or_rgb16_bt2020_to_linear(const uint16_t *src, size_t n_pixels, int bits,
                               float *dst);
void or_rgb16_bt2020_to_linear_f64(const uint16_t *src, size_t n_pixels,
                                   int bits, double *dst);
void or_bt2020_to_bt709_matrix(double m[9]);

/* Single stages (f32 modes use the mode's arithmetic). */
void or_downscale_f32(const float *src, int w, int h, float *dst);
void or_linear_to_xyb_f32(const float *src, size_t n_pixels, float *dst);
/* Blur one plane (w x h, row-major) in the given mode. */
void or_blur_plane_f32(const float *src, int w, int h, int mode, float *dst);
void or_blur_plane_f64(const double *src, int w, int h, double *dst);

/* Number of scales scored for a w x h image under a stop rule. */
int or_num_scales(int w, int h, int rule);

/* Full metric from packed linear RGB.  Returns 0 on success, -1 on invalid
 * size (w or h < 8 under the CPU/MIN8 rules, or < 1).  `sums` (optional,
 * 108 doubles, same index order) receives the raw pooled sums
 * (sum of d for L1 slots, sum of d^4 for L4 slots). */
int or_ssim2_linear(const float *ref, const float *dis, int w, int h, int mode,
                    int rule, double stats[108], double sums[108],
                    double *score, int *n_scales);
int or_ssim2_linear_f64(const double *ref, const double *dis, int w, int h,
                        int rule, double stats[108], double sums[108],
                        double *score, int *n_scales);

/* The engine's cube root (ssim2_device.cuh s2_cbrtf), used by every f32 mode. */
/* FIR32 error maps of one scale (the engine's s2_error_maps): 9 planes of
 * w_s * h_s floats, [channel][ssim error, artifact, detail loss]. */
int or_ssim2_maps_fir32(const float *ref, const float *dis, int w, int h, int rule, int scale, float *maps);
float or_cbrtf(float x);
/* The engine's division for b > 0 (Newton reciprocal + correction). */
float or_div(float a, float b);
/* The engine's p^(20/9) (BT.709 inverse OETF power). */
float or_pow_20_9(float p);

/* Final score from the 108 statistics (cpu.rs:728-871 / lib.rs:1155-1189). */
double or_score_from_stats(const double stats[108]);
void or_weights(double w[108]);

/* ---- DSSIM (dssim_oracle.c) ----------------------------------------------
 * The sibling metric of crates/dssim-cuda: five scales of a clamped 2x2
 * linear-RGB pyramid (sizes halved rounding up, never below 8), dssim-core's
 * scaled Lab, two-pass 3x3 blurs, a channel-averaged SSIM map, per-scale
 * 1 - mean |mean^(0.5^s) - ssim|, weighted, then 1/ssim - 1. */
enum { OR_DSSIM_F64 = 0, OR_DSSIM_F32 = 1 };
void or_dssim_level_dims(int w, int h, int dw[5], int dh[5]);
void or_dssim_lab_f32(float r, float g, float b, float out[3]);
/* Packed linear RGB in; per-level scores (1 - MAD) and SSIM means out.
 * Returns 1 for images below 8x8. */
int or_dssim_linear(const float *ref, const float *dis, int w, int h, int mode, double level_score[5],
                    double level_mean[5], double *dssim);

#ifdef __cplusplus
}
#endif
#endif
