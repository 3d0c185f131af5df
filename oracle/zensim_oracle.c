/* zensim_oracle.c -- CPU restatement of the zensim feature extraction of
 * crates/zensim-cuda (test infrastructure only: the tests compare the
 * engine's zensim path with it; nothing in the product calls it).
 *
 * Follows crates/zensim-cuda-kernel/src/{color,downscale,pad,blur,features}.rs
 * and the host side of crates/zensim-cuda/src/lib.rs:
 *   - sRGB8 -> linear by the reference table (color.rs:31-66), opsin mix with
 *     fused multiply-adds clipped at 0 (color.rs:126-134), the Halley cube
 *     root of cbrtf_fast from the bit seed of cbrtf_initial
 *     (color.rs:70-91), positive XYB (color.rs:136-149);
 *   - scale 0 widened to simd_padded_width with mirror-reflected columns
 *     (lib.rs:58-66, :236-252; pad.rs), scales 1..3 by 2x2 box means over
 *     the padded planes with the source clamped at the far edge
 *     (downscale.rs:21-43), scales kept while the logical width and the
 *     height are >= 8 (lib.rs:222-233);
 *   - per scale and channel: horizontal box sums of radius 5 (diameter 11)
 *     with mirrored borders of x, y, x^2 + y^2 and x y (blur.rs:40-96), a
 *     vertical running box sum over mirrored rows (features.rs:83-193), the
 *     SSIM, edge, high-frequency and MSE terms per pixel and their 17 f64
 *     sums and 3 maxima (features.rs:102-176);
 *   - the 228 features from the sums (lib.rs:686-819).
 * Every f32 operation is written out (compiled with -ffp-contract=off);
 * fmaf where the reference uses mul_add.  Column sums are added in column
 * order.  No published zensim features or scores exist in the reference
 * tree (the CPU crate and its weights are absent), so this restatement is
 * pinned only to the engine: "parity unpinned". */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

void or_srgb8_lut(float *out);

#define ZS_SCALES 4
#define ZS_RADIUS 5
#define ZS_NACC 17
#define ZS_FEATURES 228

static float g_lut[256];
static int g_lut_ready = 0;

static inline float asf(uint32_t u) { float f; memcpy(&f, &u, 4); return f; }
static inline uint32_t asu(float f) { uint32_t u; memcpy(&u, &f, 4); return u; }

int zs_padded_width(int w) {
    int aligned = (w + 15) & ~15;
    return (aligned >= 512 && (aligned / 16) % 2 == 0) ? aligned + 16 : aligned;
}

static inline int zs_mirror(int i, int n) {
    if (n <= 1) return 0;
    int period = 2 * (n - 1);
    int m = ((i % period) + period) % period;
    return m < n ? m : period - m;
}

/* color.rs:70-91 */
static float zs_cbrt(float x) {
    if (x == 0.0f) return 0.0f;
    uint32_t ui = asu(x);
    uint32_t hx = (ui & 0x7fffffffu) / 3u + 709958130u;
    float t = asf((ui & 0x80000000u) | hx);
    float r = t * t * t;
    t = t * (fmaf(x, 2.0f, r) / fmaf(r, 2.0f, x));
    r = t * t * t;
    t = t * (fmaf(x, 2.0f, r) / fmaf(r, 2.0f, x));
    return t;
}

static void zs_xyb(const uint8_t *px, float out[3]) {
    const float M02 = 0.078f, M00 = 0.30f, M01 = 1.0f - M02 - M00;
    const float M12 = 0.078f, M10 = 0.23f, M11 = 1.0f - M12 - M10;
    const float M20 = 0.24342269f, M21 = 0.20476745f, M22 = 1.0f - M20 - M21;
    const float B0 = 0.0037930734f;
    float r = g_lut[px[0]], g = g_lut[px[1]], b = g_lut[px[2]];
    float m0 = fmaxf(fmaf(M00, r, fmaf(M01, g, fmaf(M02, b, B0))), 0.0f);
    float m1 = fmaxf(fmaf(M10, r, fmaf(M11, g, fmaf(M12, b, B0))), 0.0f);
    float m2 = fmaxf(fmaf(M20, r, fmaf(M21, g, fmaf(M22, b, B0))), 0.0f);
    float bias = -zs_cbrt(B0);
    float c0 = zs_cbrt(m0) + bias, c1 = zs_cbrt(m1) + bias, c2 = zs_cbrt(m2);
    float xv = 0.5f * (c0 - c1), yv = 0.5f * (c0 + c1), bv = c2 - yv;
    out[0] = fmaf(xv, 14.0f, 0.42f);
    out[1] = yv + 0.01f;
    out[2] = bv + 0.55f;
}

/* Accumulator sums of one channel of one scale: planes a (reference) and d
 * (distorted), n x h at pitch n. */
static void zs_channel(const float *a, const float *d, int n, int h, double acc[ZS_NACC], float peak[3]) {
    const int diam = 2 * ZS_RADIUS + 1;
    const float inv = 1.0f / (float)diam;
    const float C2 = 0.0009f;
    size_t np = (size_t)n * h;
    float *hm1 = (float *)malloc(np * 4), *hm2 = (float *)malloc(np * 4);
    float *hsq = (float *)malloc(np * 4), *h12 = (float *)malloc(np * 4);
    for (int y = 0; y < h; y++)
        for (int x = 0; x < n; x++) {
            float s1 = 0, s2 = 0, sq = 0, s12 = 0;
            for (int k = 0; k < diam; k++) {
                int ix = zs_mirror(x + k - ZS_RADIUS, n);
                float s = a[(size_t)y * n + ix], t = d[(size_t)y * n + ix];
                s1 += s;
                s2 += t;
                sq = sq + s * s + t * t;
                s12 = s12 + s * t;
            }
            size_t o = (size_t)y * n + x;
            hm1[o] = s1 * inv;
            hm2[o] = s2 * inv;
            hsq[o] = sq * inv;
            h12[o] = s12 * inv;
        }
    memset(acc, 0, sizeof(double) * ZS_NACC);
    peak[0] = peak[1] = peak[2] = 0.0f;
    for (int x = 0; x < n; x++) {
        float sm1 = 0, sm2 = 0, ssq = 0, ss12 = 0;
        for (int k = 0; k < diam; k++) {
            size_t o = (size_t)zs_mirror(k - ZS_RADIUS, h) * n + x;
            sm1 += hm1[o];
            sm2 += hm2[o];
            ssq += hsq[o];
            ss12 += h12[o];
        }
        double c[ZS_NACC] = {0};
        float pk[3] = {0, 0, 0};
        for (int y = 0; y < h; y++) {
            float mu1 = sm1 * inv, mu2 = sm2 * inv, sq = ssq * inv, s12 = ss12 * inv;
            float sv = a[(size_t)y * n + x], dv = d[(size_t)y * n + x];
            float md = mu1 - mu2;
            float num_m = fmaf(md, -md, 1.0f);
            float num_s = fmaf(2.0f, fmaf(-mu1, mu2, s12), C2);
            float den_s = fmaf(-mu2, mu2, fmaf(-mu1, mu1, sq)) + C2;
            float sd_raw = 1.0f - (num_m * num_s) / den_s;
            float sd = sd_raw > 0.0f ? sd_raw : 0.0f;
            float sd2 = sd * sd, sd4 = sd2 * sd2;
            c[0] += sd;
            c[1] += sd4;
            c[2] += sd2;
            c[14] += sd4 * sd4;
            if (sd > pk[0]) pk[0] = sd;
            float d1 = fabsf(sv - mu1), d2 = fabsf(dv - mu2);
            float ed = (1.0f + d2) / (1.0f + d1) - 1.0f;
            float art = ed > 0.0f ? ed : 0.0f, det = ed < 0.0f ? -ed : 0.0f;
            float a2 = art * art, l2 = det * det, a4 = a2 * a2, l4 = l2 * l2;
            c[3] += art;
            c[4] += a4;
            c[5] += a2;
            c[6] += det;
            c[7] += l4;
            c[8] += l2;
            c[15] += a4 * a4;
            c[16] += l4 * l4;
            if (art > pk[1]) pk[1] = art;
            if (det > pk[2]) pk[2] = det;
            float vs = sv - mu1, vd = dv - mu2;
            c[10] += vs * vs;
            c[11] += vd * vd;
            c[12] += d1;
            c[13] += d2;
            float pd = sv - dv;
            c[9] += pd * pd;
            size_t ai = (size_t)zs_mirror(y + ZS_RADIUS + 1, h) * n + x;
            size_t ri = (size_t)zs_mirror(y - ZS_RADIUS, h) * n + x;
            sm1 = sm1 + hm1[ai] - hm1[ri];
            sm2 = sm2 + hm2[ai] - hm2[ri];
            ssq = ssq + hsq[ai] - hsq[ri];
            ss12 = ss12 + h12[ai] - h12[ri];
        }
        for (int i = 0; i < ZS_NACC; i++) acc[i] += c[i];
        for (int i = 0; i < 3; i++)
            if (pk[i] > peak[i]) peak[i] = pk[i];
    }
    free(hm1); free(hm2); free(hsq); free(h12);
}

/* lib.rs:686-819 */
void zs_assemble(const double *acc, const uint32_t *peaks, const int *npix, int ns, double *feat) {
    memset(feat, 0, sizeof(double) * ZS_FEATURES);
    int basic_total = ns * 13 * 3;
    for (int s = 0; s < ns; s++) {
        double inv_n = 1.0 / (double)npix[s];
        for (int c = 0; c < 3; c++) {
            const double *r = acc + (s * 3 + c) * ZS_NACC;
            const uint32_t *pk = peaks + (s * 3 + c) * 3;
            double l2 = fabs(r[10]) > 0.0 ? r[11] / r[10] : 0.0;
            double l1 = fabs(r[12]) > 0.0 ? r[13] / r[12] : 0.0;
            double *o = feat + s * 3 * 13 + c * 13;
            o[0] = fabs(r[0] * inv_n);
            o[1] = pow(fmax(r[1] * inv_n, 0.0), 0.25);
            o[2] = sqrt(fmax(r[2] * inv_n, 0.0));
            o[3] = fabs(r[3] * inv_n);
            o[4] = pow(fmax(r[4] * inv_n, 0.0), 0.25);
            o[5] = sqrt(fmax(r[5] * inv_n, 0.0));
            o[6] = fabs(r[6] * inv_n);
            o[7] = pow(fmax(r[7] * inv_n, 0.0), 0.25);
            o[8] = sqrt(fmax(r[8] * inv_n, 0.0));
            o[9] = r[9] * inv_n;
            o[10] = fmax(1.0 - l2, 0.0);
            o[11] = fmax(1.0 - l1, 0.0);
            o[12] = fmax(l2 - 1.0, 0.0);
            double *p = feat + basic_total + s * 3 * 6 + c * 6;
            p[0] = asf(pk[0]);
            p[1] = asf(pk[1]);
            p[2] = asf(pk[2]);
            p[3] = pow(fmax(r[14] * inv_n, 0.0), 0.125);
            p[4] = pow(fmax(r[15] * inv_n, 0.0), 0.125);
            p[5] = pow(fmax(r[16] * inv_n, 0.0), 0.125);
        }
    }
}

/* ref, dis: packed sRGB8, rows of `pitch` bytes.  acc: [scale][channel][17];
 * peaks: [scale][channel][3] (f32 bits); feat: 228.  Returns the number of
 * scales, or -1 below 8x8. */
int zs_features_srgb8(const uint8_t *ref, const uint8_t *dis, int w, int h, size_t pitch, double *acc,
                      uint32_t *peaks, double *feat) {
    if (w < 8 || h < 8) return -1;
    if (!g_lut_ready) {
        or_srgb8_lut(g_lut);
        g_lut_ready = 1;
    }
    int pw = zs_padded_width(w);
    float *pl[2][3];
    for (int i = 0; i < 2; i++)
        for (int c = 0; c < 3; c++) pl[i][c] = (float *)malloc((size_t)pw * h * 4);
    for (int i = 0; i < 2; i++) {
        const uint8_t *img = i ? dis : ref;
        for (int y = 0; y < h; y++)
            for (int x = 0; x < pw; x++) {
                int sx = x < w ? x : zs_mirror(x, w);
                float o[3];
                zs_xyb(img + (size_t)y * pitch + 3 * (size_t)sx, o);
                for (int c = 0; c < 3; c++) pl[i][c][(size_t)y * pw + x] = o[c];
            }
    }
    memset(acc, 0, sizeof(double) * ZS_SCALES * 3 * ZS_NACC);
    memset(peaks, 0, sizeof(uint32_t) * ZS_SCALES * 3 * 3);
    /* (lw, n, hh): logical width, padded width and height of scale s;
     * (pn, ph): those of scale s - 1, which scale s is downscaled from */
    int lw = w, n = pw, hh = h, pn = 0, ph = 0, ns = 0, npix[ZS_SCALES] = {0, 0, 0, 0};
    for (int s = 0; s < ZS_SCALES; s++) {
        if (lw < 8 || hh < 8) break;
        if (s > 0) {
            for (int i = 0; i < 2; i++)
                for (int c = 0; c < 3; c++) {
                    float *dst = (float *)malloc((size_t)n * hh * 4);
                    const float *src = pl[i][c];
                    for (int y = 0; y < hh; y++)
                        for (int x = 0; x < n; x++) {
                            int x0 = 2 * x, y0 = 2 * y;
                            int x1 = x0 + 1 < pn ? x0 + 1 : x0, y1 = y0 + 1 < ph ? y0 + 1 : y0;
                            float v = src[(size_t)y0 * pn + x0] + src[(size_t)y0 * pn + x1];
                            v = v + src[(size_t)y1 * pn + x0];
                            v = v + src[(size_t)y1 * pn + x1];
                            dst[(size_t)y * n + x] = v * 0.25f;
                        }
                    free(pl[i][c]);
                    pl[i][c] = dst;
                }
        }
        for (int c = 0; c < 3; c++) {
            float pk[3];
            zs_channel(pl[0][c], pl[1][c], n, hh, acc + (s * 3 + c) * ZS_NACC, pk);
            for (int k = 0; k < 3; k++) peaks[(s * 3 + c) * 3 + k] = asu(pk[k]);
        }
        npix[s] = n * hh;
        ns++;
        pn = n;
        ph = hh;
        lw = (lw + 1) / 2;
        n = n / 2;
        hh = (hh + 1) / 2;
    }
    for (int i = 0; i < 2; i++)
        for (int c = 0; c < 3; c++) free(pl[i][c]);
    zs_assemble(acc, peaks, npix, ns, feat);
    return ns;
}
