// ssim2_noalloc.cu -- scoring one sRGB8 pair without allocating device memory.
//
// Some callers cannot call cudaMalloc: code that runs inside a host framework
// which owns all device memory through its own pool and forbids other
// allocations, plug-ins that must not change a process's memory footprint
// after start-up, or code paths that must not block on the allocator (a
// cudaMalloc can synchronise the device).  For them this entry point keeps
// every intermediate of the pipeline -- the XYB planes of all scales, the tile
// sums, the work counter, the pair descriptor and the sRGB table -- in one
// file-scope device array of fixed size, held by every GPU that loads the
// library's device code until the process exits.  The driver reserves it when
// it loads the module that holds it: at library load with eager module
// loading, or -- under CUDA's lazy module loading, the default since CUDA
// 12.2 -- at the first call on each device, which may then synchronise.
// Callers that must never block make that first call at start-up.
//
// Limits and rules:
//   * the array holds 16 MiB; a pair whose layout needs more is rejected with
//     S2_ERR_INVALID_SIZE (every pair whose width and height are both at most
//     512 fits; larger ones are checked exactly, call by call);
//   * every call shares the array, so calls whose GPU work overlaps (other
//     streams, other host threads) race and corrupt each other; serialise them;
//   * the first call on a device looks the array's device address up and
//     copies the sRGB table into it (a synchronous copy); make that first
//     call before any stream capture on that device;
//   * the per-call pair descriptor reaches the array through a kernel that
//     takes it as a by-value argument, so no call reads host memory after
//     it returns;
//   * nothing here calls cudaMalloc, cudaFree or an allocating library
//     routine; the caller passes the inputs and a device buffer for the result.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <mutex>

#include "../../include/ssim2b200.h"
#include "ssim2_launch.h"

using namespace s2;

static_assert(sizeof(s2_result) == sizeof(DevResult), "the result is written in the C-ABI layout");

namespace {

constexpr size_t kScratchBytes = size_t(16) << 20;
static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

const float kLut[256] = {
#include "srgb8_lut.inc"
};

constexpr int kMaxDevices = 64;
std::mutex g_mu;
unsigned char *g_base[kMaxDevices];  // device address of g_scratch, per device

size_t up(size_t v, size_t a) { return (v + a - 1) / a * a; }

// Offsets inside the array.
constexpr size_t kOffLut = 0;
constexpr size_t kOffCounter = 1024;
constexpr size_t kOffDesc = 2048;  // DevPair, block table, segments

s2_status fail(const char *msg) {
    fprintf(stderr, "ssim2b200 (no-alloc): %s\n", msg);
    return S2_ERR_CUDA;
}

// Per-device set-up on the first call with that device current.
s2_status device_base(unsigned char **out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return fail("cudaGetDevice");
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_base[dev]) {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_scratch) != cudaSuccess) return fail("cudaGetSymbolAddress");
        if (configure_kernels() != cudaSuccess || upload_weights() != cudaSuccess) return fail("kernel set-up");
        if (cudaMemcpy((unsigned char *)p + kOffLut, kLut, sizeof kLut, cudaMemcpyHostToDevice) != cudaSuccess)
            return fail("copying the sRGB table");
        g_base[dev] = (unsigned char *)p;
    }
    *out = g_base[dev];
    return S2_OK;
}

// The descriptors of one call, passed by value to desc_kernel (kernel
// arguments are copied when the launch is enqueued).
struct NoallocDesc {
    DevPair pair;
    Seg segs[kScales];
    int nseg;
    int blk_first;
    unsigned off_pair, off_blk, off_seg;
};
static_assert(sizeof(NoallocDesc) < 4000, "kernel argument size");
static_assert(sizeof(DevPair) % 4 == 0 && sizeof(Seg) % 4 == 0, "copied as 32-bit words");

// Writes the descriptors into the array and zeroes the work counter.
__global__ void desc_kernel(NoallocDesc d, unsigned char *base) {
    const int t = threadIdx.x;
    const unsigned *pw = (const unsigned *)&d.pair;
    for (int i = t; i < (int)(sizeof(DevPair) / 4); i += blockDim.x) ((unsigned *)(base + d.off_pair))[i] = pw[i];
    const unsigned *sw = (const unsigned *)d.segs;
    for (int i = t; i < (int)(d.nseg * sizeof(Seg) / 4); i += blockDim.x) ((unsigned *)(base + d.off_seg))[i] = sw[i];
    if (t == 0) {
        *(int *)(base + d.off_blk) = d.blk_first;
        *(int *)(base + kOffCounter) = 0;      // the tile pass's work counter
        *(int *)(base + kOffCounter + 4) = 0;  // and its time-out word
    }
}

}  // namespace

extern "C" s2_status s2_compute_srgb8_noalloc(const uint8_t *ref, size_t ref_pitch, const uint8_t *dis,
                                              size_t dis_pitch, uint32_t width, uint32_t height,
                                              s2_result *out_device, void *stream) {
    if (!ref || !dis || !out_device) return S2_ERR_INVALID_ARG;
    if (ref_pitch < (size_t)width * 3 || dis_pitch < (size_t)width * 3) return S2_ERR_DIM_MISMATCH;
    const int ns = s2_num_scales(width, height, S2_SCALES_CPU);
    if (ns == 0 || width > 65536 || height > 65536) return S2_ERR_INVALID_SIZE;

    // Layout of this pair: same geometry as the allocating entry points.
    DevPair P;
    memset(&P, 0, sizeof P);
    P.in[0] = ref;
    P.in[1] = dis;
    P.pitch[0] = (long long)ref_pitch;
    P.pitch[1] = (long long)dis_pitch;
    P.fmt = FMT_SRGB8;
    P.nscales = ns;
    P.status = S2_OK;
    P.prep_mask = 3;  // convert both images
    P.lvl_ext = 0;
    P.w[0] = (int)width;
    P.h[0] = (int)height;
    for (int s = 1; s < kScales; s++) {
        P.w[s] = (P.w[s - 1] + 1) / 2;
        P.h[s] = (P.h[s - 1] + 1) / 2;
    }
    P.blk_x = (P.w[0] + kPyrBlk - 1) / kPyrBlk;
    P.blk_y = (P.h[0] + kPyrBlk - 1) / kPyrBlk;
    P.blk_base = 0;
    const int strip = kStripMid;
    Seg segs[kScales];
    int nseg = 0, tiles = 0;
    for (int s = 0; s < ns; s++) {
        Seg &sg = segs[nseg++];
        sg.first_tile = tiles;
        sg.pair = 0;
        sg.scale = s;
        sg.tiles_x = (P.w[s] + kTileW - 1) / kTileW;
        sg.strip_rows = strip;
        P.tile_base[s] = tiles;
        P.tile_cnt[s] = sg.tiles_x * ((P.h[s] + strip - 1) / strip);
        tiles += P.tile_cnt[s];
    }
    const int blk_first = 0;
    size_t off = kOffDesc;
    const size_t off_pair = off;
    off = up(off + sizeof(DevPair), 256);
    const size_t off_blk = off;
    off = up(off + sizeof(int), 256);
    const size_t off_seg = off;
    off = up(off + sizeof segs, 256);
    const size_t off_part = off;
    off = up(off + (size_t)tiles * 18 * sizeof(double), 256);
    size_t lvl_off[kScales][2];
    for (int s = 0; s < ns; s++) {
        P.lp[s] = (int)up((size_t)P.w[s], 64);
        const size_t bytes = up((size_t)3 * P.lp[s] * P.h[s] * sizeof(float), 256);
        for (int img = 0; img < 2; img++) {
            lvl_off[s][img] = off;
            off += bytes;
        }
    }
    if (off > kScratchBytes) {
        fprintf(stderr, "ssim2b200 (no-alloc): a %ux%u pair needs %zu bytes of scratch, over the %zu-byte array\n",
                width, height, off, kScratchBytes);
        return S2_ERR_INVALID_SIZE;
    }

    unsigned char *base = nullptr;
    s2_status st = device_base(&base);
    if (st != S2_OK) return st;
    for (int s = 0; s < ns; s++)
        for (int img = 0; img < 2; img++) P.lvl[img][s] = base + lvl_off[s][img];

    // Descriptors into the array, as kernel arguments (copied at enqueue:
    // nothing reads this stack frame after the call returns).
    cudaStream_t cs = (cudaStream_t)stream;
    NoallocDesc nd;
    memset(&nd, 0, sizeof nd);
    nd.pair = P;
    memcpy(nd.segs, segs, sizeof(Seg) * nseg);
    nd.nseg = nseg;
    nd.blk_first = blk_first;
    nd.off_pair = (unsigned)off_pair;
    nd.off_blk = (unsigned)off_blk;
    nd.off_seg = (unsigned)off_seg;
    desc_kernel<<<1, 64, 0, cs>>>(nd, base);
    if (cudaGetLastError() != cudaSuccess) return fail("staging the pair descriptor");

    const DevPair *dp = (const DevPair *)(base + off_pair);
    const ColorConsts cc{};  // sRGB8 input uses the table, not these constants
    const float *lut = (const float *)(base + kOffLut);
    int sms = 148, bps = fused_blocks_per_sm(ST_F32), dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (launch_pyramid(ST_F32, dp, 1, (const int *)(base + off_blk), 0, P.blk_x * P.blk_y, cc, lut, sms * 8, cs) !=
            cudaSuccess ||
        launch_fused(ST_F32, dp, (const Seg *)(base + off_seg), nseg, 0, tiles, (int *)(base + kOffCounter),
                     tile_check((int *)(base + kOffCounter + 4)), (double *)(base + off_part), sms * bps,
                     cs) != cudaSuccess ||
        launch_finalize(dp, 1, (const double *)(base + off_part), (const int *)(base + kOffCounter + 4),
                        (DevResult *)out_device, cs) != cudaSuccess)
        return fail("kernel launch");
    return S2_OK;
}
