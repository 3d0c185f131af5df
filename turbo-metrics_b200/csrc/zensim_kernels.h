// zensim_kernels.h -- device descriptors and launch entry points of the
// zensim feature path (zensim_kernels.cu).
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

namespace zs {

constexpr int kZsScales = 4;
constexpr int kZsRadius = 5;   // box radius of the V0.2 profile (crates/zensim-cuda/src/lib.rs:36-50)
constexpr int kZsCols = 64;    // columns (threads) per feature work item
constexpr int kZsSums = 17;    // pooled sums per (scale, channel)
constexpr int kZsOut = 20;     // + the 3 maxima
constexpr int kZsFeatures = 228;

// Three planar f32 planes (X, Y, B) of width n (the padded width), rows of
// `pitch` floats.
struct ZsPlanes {
    float *p[3];
    int n;
    size_t pitch;
};

struct ZsScale {
    ZsPlanes ref, dis;
    int n, h;
};

struct ZsItem {
    int scale, ch, x0;
};

cudaError_t zs_upload_lut(const float *lut256);
cudaError_t zs_launch_xyb(const uint8_t *img, size_t pitch, int w, int h, const ZsPlanes &out, cudaStream_t st);
cudaError_t zs_launch_down(const ZsPlanes &src, int src_h, const ZsPlanes &dst, int dst_h, cudaStream_t st);
// out: kZsOut doubles per item (17 sums, then the 3 maxima)
cudaError_t zs_launch_feat(const ZsScale *scales, const ZsItem *items, int nitems, double *out, cudaStream_t st);

}  // namespace zs
