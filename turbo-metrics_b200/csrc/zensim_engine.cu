// zensim_engine.cu -- C ABI of the zensim feature path (s2_zensim_*):
// Zensim::new / set_reference / compute_with_reference / compute_features /
// has_reference / clear_reference / debug_compute_raw of crates/zensim-cuda
// (src/lib.rs:168-819).  The reference's XYB pyramid stays resident after
// set_reference; every compute converts the distorted image, builds its
// pyramid, runs one feature launch over all (scale, channel, strip) items and
// forms the 228 features on the host from the fixed-order sums.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/ssim2b200.h"
#include "zensim_kernels.h"

using namespace zs;

s2_status s2_cuda_fail(cudaError_t e, const char *what);
void s2_set_last_error(const char *msg);
extern const float s2_srgb8_lut[256];

#define ZS_CUDA(call)                                          \
    do {                                                       \
        cudaError_t e_ = (call);                               \
        if (e_ != cudaSuccess) return s2_cuda_fail(e_, #call); \
    } while (0)

namespace {

size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

// crates/zensim-cuda/src/lib.rs:58-66
int simd_padded_width(int w) {
    const int aligned = (w + 15) & ~15;
    return (aligned >= 512 && (aligned / 16) % 2 == 0) ? aligned + 16 : aligned;
}

}  // namespace

struct s2_zensim {
    int device = 0;
    uint32_t w = 0, h = 0;
    int ns = 0;
    int n[kZsScales] = {0, 0, 0, 0}, hh[kZsScales] = {0, 0, 0, 0};
    ZsScale sc[kZsScales];
    void *planes = nullptr;      // both pyramids
    uint8_t *stage = nullptr;    // device copy of host inputs (w * 3 * h bytes)
    ZsScale *sc_d = nullptr;     // scale descriptors
    ZsItem *items_d = nullptr;   // work items
    double *out_d = nullptr;     // kZsOut doubles per item
    std::vector<ZsItem> items;
    std::vector<double> out_h;
    bool has_ref = false;
    double raw_acc[kZsScales][3][kZsSums];
    uint32_t raw_peak[kZsScales][3][3];
};

static bool g_zs_lut_ready[64];

s2_status s2_zensim_create(int32_t device, uint32_t width, uint32_t height, s2_zensim **out) {
    if (!out) return S2_ERR_INVALID_ARG;
    *out = nullptr;
    // zensim-cuda/src/lib.rs:200-205
    if (width < 8 || height < 8 || width > (1u << 16) || height > (1u << 16)) return S2_ERR_INVALID_SIZE;
    ZS_CUDA(cudaSetDevice(device));
    if (device >= 0 && device < 64 && !g_zs_lut_ready[device]) {
        ZS_CUDA(zs_upload_lut(s2_srgb8_lut));
        g_zs_lut_ready[device] = true;
    }
    s2_zensim *z = new s2_zensim();
    std::memset(z->raw_acc, 0, sizeof z->raw_acc);
    std::memset(z->raw_peak, 0, sizeof z->raw_peak);
    z->device = device;
    z->w = width;
    z->h = height;
    // scales while the logical width and the height are >= 8 (lib.rs:222-233)
    int lw = (int)width, n = simd_padded_width((int)width), h = (int)height;
    size_t bytes = 0, off[kZsScales][2];
    for (int s = 0; s < kZsScales; s++) {
        if (lw < 8 || h < 8) break;
        z->n[s] = n;
        z->hh[s] = h;
        const size_t pitch = align_up((size_t)n, 64);
        for (int img = 0; img < 2; img++) {
            off[s][img] = bytes;
            bytes += 3 * align_up(pitch * h * sizeof(float), 256);
        }
        z->ns++;
        lw = (lw + 1) / 2;
        n = n / 2;
        h = (h + 1) / 2;
    }
    for (int s = 0; s < z->ns; s++)
        for (int c = 0; c < 3; c++)
            for (int x0 = 0; x0 < z->n[s]; x0 += kZsCols) z->items.push_back(ZsItem{s, c, x0});
    z->out_h.resize(z->items.size() * kZsOut);
    cudaError_t e = cudaMalloc(&z->planes, bytes);
    if (e == cudaSuccess) e = cudaMalloc((void **)&z->stage, (size_t)width * 3 * height);
    if (e == cudaSuccess) e = cudaMalloc((void **)&z->sc_d, sizeof(ZsScale) * kZsScales);
    if (e == cudaSuccess) e = cudaMalloc((void **)&z->items_d, sizeof(ZsItem) * z->items.size());
    if (e == cudaSuccess) e = cudaMalloc((void **)&z->out_d, sizeof(double) * z->out_h.size());
    if (e != cudaSuccess) {
        s2_zensim_destroy(z);
        return e == cudaErrorMemoryAllocation ? S2_ERR_OOM : s2_cuda_fail(e, "zensim buffers");
    }
    for (int s = 0; s < z->ns; s++) {
        const size_t pitch = align_up((size_t)z->n[s], 64);
        const size_t plane = align_up(pitch * z->hh[s] * sizeof(float), 256);
        ZsPlanes *pl[2] = {&z->sc[s].ref, &z->sc[s].dis};
        for (int img = 0; img < 2; img++) {
            for (int c = 0; c < 3; c++) pl[img]->p[c] = (float *)((char *)z->planes + off[s][img] + c * plane);
            pl[img]->n = z->n[s];
            pl[img]->pitch = pitch;
        }
        z->sc[s].n = z->n[s];
        z->sc[s].h = z->hh[s];
    }
    e = cudaMemcpy(z->sc_d, z->sc, sizeof(ZsScale) * kZsScales, cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy(z->items_d, z->items.data(), sizeof(ZsItem) * z->items.size(), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        s2_zensim_destroy(z);
        return s2_cuda_fail(e, "zensim descriptors");
    }
    *out = z;
    return S2_OK;
}

void s2_zensim_destroy(s2_zensim *z) {
    if (!z) return;
    cudaSetDevice(z->device);
    cudaDeviceSynchronize();
    cudaFree(z->planes);
    cudaFree(z->stage);
    cudaFree(z->sc_d);
    cudaFree(z->items_d);
    cudaFree(z->out_d);
    delete z;
}

// Convert one image (img 0 reference, 1 distorted) and build its pyramid.
static s2_status zs_pyramid(s2_zensim *z, int img, const uint8_t *src, size_t pitch, int32_t on_host,
                            cudaStream_t st) {
    if (!src) return S2_ERR_INVALID_ARG;
    const size_t row = (size_t)z->w * 3;
    if (pitch < row) return S2_ERR_DIM_MISMATCH;
    if (on_host) {
        ZS_CUDA(cudaMemcpy2DAsync(z->stage, row, src, pitch, row, z->h, cudaMemcpyHostToDevice, st));
        src = z->stage;
        pitch = row;
    }
    ZsPlanes ZsScale::*which = img ? &ZsScale::dis : &ZsScale::ref;
    ZS_CUDA(zs_launch_xyb(src, pitch, (int)z->w, (int)z->h, z->sc[0].*which, st));
    for (int s = 1; s < z->ns; s++)
        ZS_CUDA(zs_launch_down(z->sc[s - 1].*which, z->hh[s - 1], z->sc[s].*which, z->hh[s], st));
    return S2_OK;
}

s2_status s2_zensim_set_reference_srgb8(s2_zensim *z, const uint8_t *ref, size_t pitch, int32_t on_host,
                                        void *stream) {
    if (!z) return S2_ERR_INVALID_ARG;
    ZS_CUDA(cudaSetDevice(z->device));
    z->has_ref = false;
    cudaStream_t st = (cudaStream_t)stream;
    s2_status r = zs_pyramid(z, 0, ref, pitch, on_host, st);
    if (r != S2_OK) return r;
    ZS_CUDA(cudaStreamSynchronize(st));
    z->has_ref = true;
    return S2_OK;
}

// lib.rs:686-819: the 228 features from the sums of each (scale, channel)
static void zs_assemble(s2_zensim *z, double *feat) {
    std::memset(feat, 0, sizeof(double) * kZsFeatures);
    const int basic_total = z->ns * 13 * 3;
    for (int s = 0; s < z->ns; s++) {
        const double inv_n = 1.0 / ((double)z->n[s] * (double)z->hh[s]);
        for (int c = 0; c < 3; c++) {
            const double *r = z->raw_acc[s][c];
            const uint32_t *pk = z->raw_peak[s][c];
            const double l2 = std::fabs(r[10]) > 0.0 ? r[11] / r[10] : 0.0;
            const double l1 = std::fabs(r[12]) > 0.0 ? r[13] / r[12] : 0.0;
            double *o = feat + s * 3 * 13 + c * 13;
            o[0] = std::fabs(r[0] * inv_n);
            o[1] = std::pow(std::fmax(r[1] * inv_n, 0.0), 0.25);
            o[2] = std::sqrt(std::fmax(r[2] * inv_n, 0.0));
            o[3] = std::fabs(r[3] * inv_n);
            o[4] = std::pow(std::fmax(r[4] * inv_n, 0.0), 0.25);
            o[5] = std::sqrt(std::fmax(r[5] * inv_n, 0.0));
            o[6] = std::fabs(r[6] * inv_n);
            o[7] = std::pow(std::fmax(r[7] * inv_n, 0.0), 0.25);
            o[8] = std::sqrt(std::fmax(r[8] * inv_n, 0.0));
            o[9] = r[9] * inv_n;
            o[10] = std::fmax(1.0 - l2, 0.0);
            o[11] = std::fmax(1.0 - l1, 0.0);
            o[12] = std::fmax(l2 - 1.0, 0.0);
            double *p = feat + basic_total + s * 3 * 6 + c * 6;
            float f;
            for (int k = 0; k < 3; k++) {
                std::memcpy(&f, &pk[k], 4);
                p[k] = (double)f;
            }
            p[3] = std::pow(std::fmax(r[14] * inv_n, 0.0), 0.125);
            p[4] = std::pow(std::fmax(r[15] * inv_n, 0.0), 0.125);
            p[5] = std::pow(std::fmax(r[16] * inv_n, 0.0), 0.125);
        }
    }
}

s2_status s2_zensim_compute_with_reference_srgb8(s2_zensim *z, const uint8_t *dis, size_t pitch, int32_t on_host,
                                                 void *stream, double *features, int32_t *n_scales) {
    if (!z || !features) return S2_ERR_INVALID_ARG;
    if (!z->has_ref) return S2_ERR_NO_REFERENCE;
    ZS_CUDA(cudaSetDevice(z->device));
    cudaStream_t st = (cudaStream_t)stream;
    s2_status r = zs_pyramid(z, 1, dis, pitch, on_host, st);
    if (r != S2_OK) return r;
    ZS_CUDA(zs_launch_feat(z->sc_d, z->items_d, (int)z->items.size(), z->out_d, st));
    ZS_CUDA(cudaMemcpyAsync(z->out_h.data(), z->out_d, sizeof(double) * z->out_h.size(), cudaMemcpyDeviceToHost,
                            st));
    ZS_CUDA(cudaStreamSynchronize(st));
    // items are ordered (scale, channel, strip): strips added left to right
    std::memset(z->raw_acc, 0, sizeof z->raw_acc);
    float peak[kZsScales][3][3] = {};
    for (size_t i = 0; i < z->items.size(); i++) {
        const ZsItem &it = z->items[i];
        const double *o = &z->out_h[i * kZsOut];
        for (int k = 0; k < kZsSums; k++) z->raw_acc[it.scale][it.ch][k] += o[k];
        for (int k = 0; k < 3; k++) peak[it.scale][it.ch][k] = std::fmax(peak[it.scale][it.ch][k], (float)o[kZsSums + k]);
    }
    for (int s = 0; s < kZsScales; s++)
        for (int c = 0; c < 3; c++)
            for (int k = 0; k < 3; k++) std::memcpy(&z->raw_peak[s][c][k], &peak[s][c][k], 4);
    zs_assemble(z, features);
    if (n_scales) *n_scales = z->ns;
    return S2_OK;
}

s2_status s2_zensim_compute_features_srgb8(s2_zensim *z, const uint8_t *ref, size_t ref_pitch, const uint8_t *dis,
                                           size_t dis_pitch, int32_t on_host, void *stream, double *features,
                                           int32_t *n_scales) {
    s2_status r = s2_zensim_set_reference_srgb8(z, ref, ref_pitch, on_host, stream);
    if (r != S2_OK) return r;
    return s2_zensim_compute_with_reference_srgb8(z, dis, dis_pitch, on_host, stream, features, n_scales);
}

int32_t s2_zensim_has_reference(const s2_zensim *z) { return z && z->has_ref ? 1 : 0; }

s2_status s2_zensim_clear_reference(s2_zensim *z) {
    if (!z) return S2_ERR_INVALID_ARG;
    z->has_ref = false;
    return S2_OK;
}

s2_status s2_zensim_raw(const s2_zensim *z, double *acc, uint32_t *peaks) {
    if (!z || !acc || !peaks) return S2_ERR_INVALID_ARG;
    std::memcpy(acc, z->raw_acc, sizeof z->raw_acc);
    std::memcpy(peaks, z->raw_peak, sizeof z->raw_peak);
    return S2_OK;
}

s2_status s2_zensim_mem_usage(const s2_zensim *z, size_t *bytes) {
    if (!z || !bytes) return S2_ERR_INVALID_ARG;
    size_t b = (size_t)z->w * 3 * z->h + sizeof(ZsScale) * kZsScales + sizeof(ZsItem) * z->items.size() +
               sizeof(double) * z->out_h.size();
    for (int s = 0; s < z->ns; s++)
        b += 6 * align_up(align_up((size_t)z->n[s], 64) * z->hh[s] * sizeof(float), 256);
    *bytes = b;
    return S2_OK;
}
