// ssim2_engine.cu -- host side of the B200 SSIMULACRA2 engine: planning of
// pairs into pyramid blocks and fused tiles, device memory, launches, and
// the C ABI of include/ssim2b200.h.
//
// Reference host pipeline being replaced: crates/ssimulacra2-cuda/src/lib.rs
// (Ssimulacra2::new :80-197, record :237-326, process_scale :862-984,
// reduce :986-1016, post_process_scores :1018-1192).  There, one pair costs
// ~305 graph nodes (20 packed planes per scale, 7 transposes per scale, 72 NPP
// reductions each with its own allocation and D2H copy).  Here one pair, or a
// whole batch of pairs of any sizes, costs three kernel launches and two small
// copies.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/ssim2b200.h"
#include "ssim2_engine_internal.h"

using namespace s2;

// ---------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------
static thread_local std::string g_last_error;

s2_status s2_cuda_fail(cudaError_t e, const char *what) {
    char buf[256];
    snprintf(buf, sizeof buf, "%s: %s (%d)", what, cudaGetErrorString(e), (int)e);
    g_last_error = buf;
    return e == cudaErrorMemoryAllocation ? S2_ERR_OOM : S2_ERR_CUDA;
}
void s2_set_last_error(const char *msg) { g_last_error = msg; }

// ---------------------------------------------------------------------------
// constants shared by all engines
// ---------------------------------------------------------------------------
// sRGB8 -> linear table of the reference (ssimulacra2-cuda-kernel/src/srgb.rs:23-51).
// The entries follow the gamma-2.4 sRGB curve with a linear toe but were
// printed with 6-9 decimal digits; the table, not the formula, defines the
// reference's conversion, so the same numbers are used (hex-float spelling).
const float s2_srgb8_lut[256] = {
#include "srgb8_lut.inc"
};

static double det3(const double m[9]) {
    return m[0] * (m[4] * m[8] - m[5] * m[7]) - m[1] * (m[3] * m[8] - m[5] * m[6]) +
           m[2] * (m[3] * m[7] - m[4] * m[6]);
}

// RGB -> XYZ matrix of a primary set normalised to its white point.
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

static const double BT709[8] = {0.640, 0.330, 0.300, 0.600, 0.150, 0.060, 0.3127, 0.3290};

// 4:2:0 YUV coefficients of a matrix, range and sample depth, with the
// range's luma minimum and chroma neutral value (cuda-colorspace-kernel/src/
// lib.rs:46-140).  Derived in f32 with the reference's operations and their
// order, so the five values are the reference's to the bit: Kr / Kb by
// constants_from_primaries (lib.rs:205-221; the const Vec2 / Vec3 algebra of
// const_algebra.rs, every product and sum rounded to f32, no fused
// multiply-adds: this unit is built with -ffp-contract=off), then
// MatrixCoefficients::coefficients (lib.rs:188-203), e.g. r_coeff =
// ((2 * (1 - kr)) * 1) / chroma_range.  Primaries: constants.rs.
namespace {
struct V2f {
    float x, y;
};
struct V3f {
    float x, y, z;
};
V3f xy_to_xyz(V2f p) { return V3f{p.x / p.y, 1.0f, ((1.0f - p.x) - p.y) / p.y}; }
float dot3(V3f a, V3f b) {
    float s = a.x * b.x;
    s = s + a.y * b.y;
    return s + a.z * b.z;
}
V3f cross3(V3f a, V3f b) {
    return V3f{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
const float kPrim709[8] = {0.640f, 0.330f, 0.300f, 0.600f, 0.150f, 0.060f, 0.3127f, 0.3290f};
const float kPrim601_525[8] = {0.630f, 0.340f, 0.310f, 0.595f, 0.155f, 0.070f, 0.3127f, 0.3290f};
const float kPrim601_625[8] = {0.640f, 0.330f, 0.290f, 0.600f, 0.150f, 0.060f, 0.3127f, 0.3290f};
}  // namespace

void s2_yuv_coeffs(int matrix, int range, int bits, float out[5], int *ymin, int *neutral) {
    const float *pr = matrix == S2_MATRIX_BT601_525 ? kPrim601_525 : (matrix == S2_MATRIX_BT601_625 ? kPrim601_625 : kPrim709);
    const V3f r = xy_to_xyz({pr[0], pr[1]}), g = xy_to_xyz({pr[2], pr[3]}), b = xy_to_xyz({pr[4], pr[5]}),
              w = xy_to_xyz({pr[6], pr[7]});
    const V3f x_rgb{r.x, g.x, b.x}, y_rgb{r.y, g.y, b.y}, z_rgb{r.z, g.z, b.z};
    const float mul = 1.0f / dot3(x_rgb, cross3(y_rgb, z_rgb));
    const float kr = dot3(w, cross3(g, b)) * mul;
    const float kb = dot3(w, cross3(r, g)) * mul;
    const bool full = range == S2_RANGE_FULL;
    const int sh = bits - 8;
    const float lrange = (float)(full ? (1u << bits) - 1u : (235u - 16u) << sh);
    const float crange = (float)(full ? (1u << bits) - 1u : (240u - 16u) << sh);
    const float kg = (1.0f - kr) - kb;
    out[0] = 1.0f / lrange;
    out[1] = ((2.0f * (1.0f - kr)) * 1.0f) / crange;
    out[2] = ((2.0f * (1.0f - kb)) * 1.0f) / crange;
    out[3] = (((((-2.0f) * (1.0f - kb)) * kb) / kg) * 1.0f) / crange;
    out[4] = (((((-2.0f) * (1.0f - kr)) * kr) / kg) * 1.0f) / crange;
    *ymin = full ? 0 : (16 << sh);
    *neutral = 1 << (bits - 1);
}

extern "C" s2_status s2_yuv_coefficients(int32_t matrix, int32_t range, int32_t bits, float coeffs[5],
                                         int32_t *luma_min, int32_t *chroma_neutral) {
    if (!coeffs || matrix < S2_MATRIX_BT709 || matrix > S2_MATRIX_BT601_625 ||
        (range != S2_RANGE_LIMITED && range != S2_RANGE_FULL) || (bits != 8 && bits != 16))
        return S2_ERR_INVALID_ARG;
    int ymin = 0, neutral = 0;
    s2_yuv_coeffs(matrix, range, bits, coeffs, &ymin, &neutral);
    if (luma_min) *luma_min = ymin;
    if (chroma_neutral) *chroma_neutral = neutral;
    return S2_OK;
}

ColorConsts s2_make_color_consts() {
    static const double BT2020[8] = {0.708, 0.292, 0.170, 0.797, 0.131, 0.046, 0.3127, 0.3290};
    ColorConsts cc;
    double a[9], b[9], bi[9];
    rgb_to_xyz(BT2020, a);
    rgb_to_xyz(BT709, b);
    inv3(b, bi);
    for (int r = 0; r < 3; r++)
        for (int k = 0; k < 3; k++)
            cc.m2020[r * 3 + k] = (float)(bi[r * 3 + 0] * a[0 * 3 + k] + bi[r * 3 + 1] * a[1 * 3 + k] +
                                          bi[r * 3 + 2] * a[2 * 3 + k]);
    return cc;
}

// Re-derive the FIR taps (Charalampidis 2016 truncated-cosine recursion,
// sigma 1.5; ssimulacra2-cuda-kernel/build.rs:28-145) in double and check the
// f32 values compiled into the kernels.
static bool check_taps() {
    const double sigma = 1.5, pi = 3.14159265358979323846;
    double radius = std::round(std::fma(3.2795, sigma, 0.2546));
    double w0 = pi / (2.0 * radius);
    double om[3] = {w0, 3.0 * w0, 5.0 * w0};
    double p1 = 1.0 / std::tan(0.5 * om[0]), p3 = -1.0 / std::tan(0.5 * om[1]), p5 = 1.0 / std::tan(0.5 * om[2]);
    double r1 = p1 * p1 / std::sin(om[0]), r3 = -p3 * p3 / std::sin(om[1]), r5 = p5 * p5 / std::sin(om[2]);
    double rho[3];
    for (int i = 0; i < 3; i++) rho[i] = std::exp(-0.5 * sigma * sigma * om[i] * om[i]) / radius;
    double d13 = std::fma(p1, r3, -r1 * p3), d35 = std::fma(p3, r5, -r3 * p5), d51 = std::fma(p5, r1, -r5 * p1);
    double z15 = d35 / d13, z35 = d51 / d13;
    double M[9] = {p1, p3, p5, r1, r3, r5, z15, z35, 1.0};
    double gm[3] = {1.0, std::fma(radius, radius, -sigma * sigma), std::fma(z15, rho[0], z35 * rho[1]) + rho[2]};
    double dm = det3(M), beta[3];
    for (int col = 0; col < 3; col++) {
        double Mc[9];
        memcpy(Mc, M, sizeof Mc);
        for (int r = 0; r < 3; r++) Mc[r * 3 + col] = gm[r];
        beta[col] = det3(Mc) / dm;
    }
    double n2[3], d1[3];
    for (int i = 0; i < 3; i++) {
        n2[i] = -beta[i] * std::cos(om[i] * (radius + 1.0));
        d1[i] = -2.0 * std::cos(om[i]);
    }
    // impulse response of the double recursion = the FIR taps
    const int N = (int)radius, L = 64, c = 32;
    double in[64] = {0}, out[64] = {0}, prev[3] = {0}, prev2[3] = {0};
    in[c] = 1.0;
    for (int n = -N + 1; n < L; n++) {
        int left = n - N - 1, right = n + N - 1;
        double s = (left >= 0 ? in[left] : 0.0) + (right < L ? in[right] : 0.0), o = 0.0;
        for (int k = 0; k < 3; k++) {
            double ok = s * n2[k] - d1[k] * prev[k] - prev2[k];
            prev2[k] = prev[k];
            prev[k] = ok;
            o += ok;
        }
        if (n >= 0) out[n] = o;
    }
    const float t32[5] = {S2_T0, S2_T1, S2_T2, S2_T3, S2_T4};
    for (int k = 0; k < 5; k++)
        if ((float)out[c + k] != t32[k]) return false;
    return true;
}

static std::once_flag g_init_once;
static s2_status g_init_status = S2_OK;

s2_status s2_global_init() {
    std::call_once(g_init_once, [] {
        if (!check_taps()) {
            g_last_error = "FIR taps compiled into the kernels do not match the derivation";
            g_init_status = S2_ERR_CUDA;
            return;
        }
        cudaError_t e = configure_kernels();
        if (e == cudaSuccess) e = upload_weights();
        if (e != cudaSuccess) g_init_status = s2_cuda_fail(e, "kernel set-up");
    });
    return g_init_status;
}


// ---------------------------------------------------------------------------
// tile-height autotuner cache
// ---------------------------------------------------------------------------
static std::mutex g_tune_mu;
static std::unordered_map<uint64_t, int> g_tune;

uint64_t s2_tune_signature(uint64_t items63, int storage, int num_sms, int bps) {
    // half-octave bucket of the work-item count
    int b = 0;
    if (items63 > 0) {
        const double l = std::log2((double)items63);
        b = (int)std::floor(2.0 * l);
    }
    return ((uint64_t)(b & 0xff) << 32) | ((uint64_t)(storage & 0xf) << 24) | ((uint64_t)(num_sms & 0xfff) << 8) |
           (uint64_t)(bps & 0xff);
}

int s2_tuned_strip(uint64_t sig) {
    std::lock_guard<std::mutex> g(g_tune_mu);
    auto it = g_tune.find(sig);
    return it == g_tune.end() ? 0 : it->second;
}

void s2_set_tuned_strip(uint64_t sig, int strip) {
    std::lock_guard<std::mutex> g(g_tune_mu);
    g_tune[sig] = strip;
}

// ---------------------------------------------------------------------------
// single-pair context
// ---------------------------------------------------------------------------
struct s2_ctx {
    Engine eng;
    uint32_t w = 0, h = 0;
    DevBuf stage[4];     // host-input staging: ref, dis (+ uv planes)
    bool has_ref = false;
    bool last_was_ref_build = false;
    DevBuf ref_levels;   // the cached reference's XYB planes, every scored scale
    PairExtra ref_extra; // points the pairs of compute_with_reference at them
    Plan plan;
};

// A batch has two submission slots (engines with their own workspaces), so a
// caller may enqueue submission k+1 before reading submission k's results:
// k+1's uploads and preps then overlap k's tile pass.  Device-input
// submissions use slot 0; host-input submissions take a slot whose results
// are not pending (slot 1 is allocated on first such use).  Results are read
// oldest first.
struct s2_batch {
    Engine eng[2];
    bool ready[2] = {false, false};
    Plan plan[2];
    std::deque<int> unread;  // slots whose results were not read, oldest first
    int last_slot = 0;
    bool profiling = false, graphs = true;
    int metrics = S2_METRIC_SSIMULACRA2;
    s2_config cfg;
    uint32_t max_pairs = 0;
    uint64_t max_pixels = 0;
    // cached reference (s2_batch_set_reference): its XYB pyramid
    DevBuf ref_buf;
    bool has_ref = false;
    uint32_t ref_w = 0, ref_h = 0;
    PairExtra ref_extra;  // what each candidate of submit_with_reference gets

    s2_status open_slot(int k) {
        if (ready[k]) return S2_OK;
        s2_status st = eng[k].init(&cfg);
        if (st == S2_OK) st = eng[k].reserve(max_pairs, max_pixels, false);
        if (st == S2_OK) st = eng[k].set_profiling(profiling);
        if (st != S2_OK) {
            eng[k].release();
            return st;
        }
        eng[k].graphs = graphs;
        eng[k].metrics = metrics;
        ready[k] = true;
        return S2_OK;
    }
    // the slot for the next submission; a slot whose results are pending is
    // reused only when both are (its results are then dropped)
    int take_slot(bool host) {
        auto pending = [&](int k) { return std::find(unread.begin(), unread.end(), k) != unread.end(); };
        int k = 0;
        if (host && pending(0)) k = pending(1) ? unread.front() : 1;
        unread.erase(std::remove(unread.begin(), unread.end(), k), unread.end());
        return k;
    }
};

// The tile pass's wait bound and the failure test's withheld work item.
static std::atomic<long long> g_tile_wait_cycles{1ll << 31};
static std::atomic<int> g_tile_drop_item{-1};

namespace s2 {
TileCheck tile_check(int *err) { return TileCheck{err, g_tile_wait_cycles.load(), g_tile_drop_item.load()}; }
}  // namespace s2

extern "C" {

const char *s2_version(void) { return "ssim2b200 1.0.0 (sm_100a)"; }

const char *s2_status_string(s2_status st) {
    switch (st) {
    case S2_OK: return "ok";
    case S2_ERR_OOM: return "out of device memory or over the HBM budget";
    case S2_ERR_INVALID_SIZE: return "invalid image size";
    case S2_ERR_DIM_MISMATCH: return "dimension mismatch";
    case S2_ERR_NO_REFERENCE: return "no cached reference";
    case S2_ERR_CUDA: return "CUDA error";
    case S2_ERR_TIMEOUT: return "timeout";
    case S2_ERR_BUSY: return "busy";
    case S2_ERR_INVALID_ARG: return "invalid argument";
    case S2_ERR_NOT_READY: return "not ready";
    case S2_ERR_CANCELLED: return "cancelled";
    }
    return "unknown status";
}

const char *s2_last_error(void) { return g_last_error.c_str(); }

s2_status s2_debug_tile_timeout(int32_t drop_item, int64_t wait_cycles) {
    if (wait_cycles < 0) return S2_ERR_INVALID_ARG;
    g_tile_drop_item.store(drop_item < 0 ? -1 : drop_item);
    g_tile_wait_cycles.store(wait_cycles == 0 ? (1ll << 31) : wait_cycles);
    return S2_OK;
}

void s2_config_default(s2_config *cfg) {
    if (!cfg) return;
    memset(cfg, 0, sizeof *cfg);
    cfg->struct_size = sizeof *cfg;
    cfg->device = 0;
    cfg->blur = S2_BLUR_FIR;
    cfg->storage = S2_STORAGE_F32;
    cfg->scale_rule = S2_SCALES_CPU;
    cfg->strip_rows = 0;
    cfg->hbm_budget = 0;
}

int s2_num_scales(uint32_t w, uint32_t h, int32_t rule) { return s2_num_scales_rule(w, h, rule); }

static s2_status check_cfg(const s2_config *cfg) {
    if (!cfg || cfg->struct_size != sizeof(s2_config)) return S2_ERR_INVALID_ARG;
    if (cfg->blur != S2_BLUR_FIR && cfg->blur != S2_BLUR_IIR_REF) return S2_ERR_INVALID_ARG;
    // 16-bit storage is not offered: the passes are compute-bound, so halving
    // the plane bytes bought no time, and it cost up to 0.2 (f16) and 4
    // (bf16) in score
    if (cfg->storage != S2_STORAGE_F32) return S2_ERR_INVALID_ARG;
    if (cfg->scale_rule < 0 || cfg->scale_rule > 2) return S2_ERR_INVALID_ARG;
    if (cfg->strip_rows != 0 && cfg->strip_rows != kStripMin && cfg->strip_rows != kStripMid &&
        cfg->strip_rows != kStripMax)
        return S2_ERR_INVALID_ARG;
    return S2_OK;
}

static s2_status ctx_create(const s2_config *cfg_in, uint32_t width, uint32_t height, int metrics, s2_ctx **out);

s2_status s2_create(const s2_config *cfg_in, uint32_t width, uint32_t height, s2_ctx **out) {
    return ctx_create(cfg_in, width, height, S2_METRIC_SSIMULACRA2, out);
}

static s2_status ctx_create(const s2_config *cfg_in, uint32_t width, uint32_t height, int metrics, s2_ctx **out) {
    if (!out) return S2_ERR_INVALID_ARG;
    *out = nullptr;
    s2_config cfg;
    if (cfg_in) cfg = *cfg_in;
    else s2_config_default(&cfg);
    s2_status st = check_cfg(&cfg);
    if (st != S2_OK) return st;
    if (((metrics & S2_METRIC_SSIMULACRA2) && s2_num_scales_rule(width, height, cfg.scale_rule) == 0) ||
        ((metrics & S2_METRIC_DSSIM) && (width < 8 || height < 8)) || width > 65536 || height > 65536)
        return S2_ERR_INVALID_SIZE;
    // pre-flight: levels (2 images, ~1/3 of scale 0) + partials + staging
    {
        size_t free_b = 0, total_b = 0;
        if (cudaSetDevice(cfg.device) != cudaSuccess) return s2_cuda_fail(cudaGetLastError(), "cudaSetDevice");
        if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess) {
            uint64_t est = (uint64_t)width * height * 40 + (64u << 20);
            if (est > free_b || (cfg.hbm_budget && est > cfg.hbm_budget)) return S2_ERR_OOM;
        }
    }
    s2_ctx *c = new (std::nothrow) s2_ctx();
    if (!c) return S2_ERR_OOM;
    c->w = width;
    c->h = height;
    st = c->eng.init(&cfg);
    c->eng.graphs = true;
    c->eng.metrics = metrics;
    if (st == S2_OK) {
        // allocate the steady-state buffers now (like the reference's new)
        s2_pair_desc d;
        memset(&d, 0, sizeof d);
        d.width = width;
        d.height = height;
        d.format = S2_FMT_LINEAR_F32;
        d.ref = d.dis = (const void *)16;  // placeholder, only sizes are used
        st = c->eng.plan(&d, 1, c->plan);
        if (st == S2_OK) st = c->eng.ensure(c->eng.levels_d, std::max<size_t>(c->plan.level_bytes, 256));
        if (st == S2_OK)
            st = c->eng.ensure(c->eng.partials_d, std::max<size_t>((size_t)c->plan.total_tiles * 18 * 8, 256));
        if (st == S2_OK) st = c->eng.ensure(c->eng.results_d, sizeof(DevResult));
        if (st == S2_OK && (metrics & S2_METRIC_DSSIM)) st = c->eng.ensure(c->eng.ds_d, Engine::ds_bytes(c->plan));
    }
    if (st != S2_OK) {
        c->eng.release();
        delete c;
        return st;
    }
    *out = c;
    return S2_OK;
}

void s2_destroy(s2_ctx *ctx) {
    if (!ctx) return;
    for (DevBuf &b : ctx->stage)
        if (b.p) cudaFree(b.p);
    if (ctx->ref_levels.p) cudaFree(ctx->ref_levels.p);
    ctx->eng.release();
    delete ctx;
}

s2_status s2_mem_usage(const s2_ctx *ctx, size_t *bytes) {
    if (!ctx || !bytes) return S2_ERR_INVALID_ARG;
    size_t n = ctx->eng.allocated + ctx->ref_levels.n;
    for (const DevBuf &b : ctx->stage) n += b.n;
    *bytes = n;
    return S2_OK;
}

s2_status s2_dimensions(const s2_ctx *ctx, uint32_t *w, uint32_t *h) {
    if (!ctx) return S2_ERR_INVALID_ARG;
    if (w) *w = ctx->w;
    if (h) *h = ctx->h;
    return S2_OK;
}

static s2_status ctx_run(s2_ctx *ctx, const s2_pair_desc &d, void *stream, const PairExtra *ex = nullptr) {
    // the cached-reference path keeps SSIMULACRA2's XYB planes only
    if (ex && !ex->dssim && !(ctx->eng.metrics & S2_METRIC_SSIMULACRA2)) return S2_ERR_INVALID_ARG;
    s2_status st = ctx->eng.plan(&d, 1, ctx->plan, ex);
    if (st == S2_OK && ctx->plan.pairs[0].status == S2_OK && (!ex || ex->score))
        st = ctx->eng.tune(&d, 1, ctx->plan, ex, (cudaStream_t)stream);
    if (st != S2_OK) return st;
    if (ctx->plan.pairs[0].status != S2_OK) return (s2_status)ctx->plan.pairs[0].status;
    ctx->last_was_ref_build = ex && !ex->score;
    return ctx->eng.enqueue(ctx->plan, (cudaStream_t)stream);
}

// Copy a host image into a device staging buffer (pitched rows).
static s2_status stage_host(s2_ctx *ctx, int slot, const void *src, size_t pitch, size_t row_bytes,
                            size_t rows, void *stream, const void **dev, size_t *dev_pitch) {
    DevBuf &b = ctx->stage[slot];
    size_t need = row_bytes * rows;
    if (b.n < need) {
        if (b.p) {
            cudaStreamSynchronize((cudaStream_t)stream);
            cudaFree(b.p);
        }
        b.p = nullptr;
        b.n = 0;
        S2_CUDA(cudaMalloc(&b.p, need));
        b.n = need;
    }
    S2_CUDA(cudaMemcpy2DAsync(b.p, row_bytes, src, pitch, row_bytes, rows, cudaMemcpyHostToDevice,
                              (cudaStream_t)stream));
    *dev = b.p;
    *dev_pitch = row_bytes;
    return S2_OK;
}

static s2_pair_desc make_desc(uint32_t w, uint32_t h, int fmt, const void *ref, size_t rp, const void *dis,
                              size_t dp) {
    s2_pair_desc d;
    memset(&d, 0, sizeof d);
    d.width = w;
    d.height = h;
    d.format = fmt;
    d.ref = ref;
    d.dis = dis;
    d.ref_pitch = rp;
    d.dis_pitch = dp;
    return d;
}

s2_status s2_compute_linear_f32(s2_ctx *ctx, const float *ref, size_t ref_pitch, const float *dis,
                                size_t dis_pitch, void *stream) {
    if (!ctx || !ref || !dis) return S2_ERR_INVALID_ARG;
    if (ref_pitch < (size_t)ctx->w * 12 || dis_pitch < (size_t)ctx->w * 12) return S2_ERR_DIM_MISMATCH;
    return ctx_run(ctx, make_desc(ctx->w, ctx->h, S2_FMT_LINEAR_F32, ref, ref_pitch, dis, dis_pitch), stream);
}

s2_status s2_compute_srgb8(s2_ctx *ctx, const uint8_t *ref, size_t ref_pitch, const uint8_t *dis,
                           size_t dis_pitch, int32_t on_host, void *stream) {
    if (!ctx || !ref || !dis) return S2_ERR_INVALID_ARG;
    const size_t row = (size_t)ctx->w * 3;
    if (ref_pitch < row || dis_pitch < row) return S2_ERR_DIM_MISMATCH;
    const void *r = ref, *d = dis;
    size_t rp = ref_pitch, dp = dis_pitch;
    if (on_host) {
        s2_status st = stage_host(ctx, 0, ref, ref_pitch, row, ctx->h, stream, &r, &rp);
        if (st == S2_OK) st = stage_host(ctx, 1, dis, dis_pitch, row, ctx->h, stream, &d, &dp);
        if (st != S2_OK) return st;
    }
    return ctx_run(ctx, make_desc(ctx->w, ctx->h, S2_FMT_SRGB8, r, rp, d, dp), stream);
}

// 4:2:0 biplanar pair (NV12 / P016) through the single-pair context.
static s2_status ctx_yuv420(s2_ctx *ctx, int fmt, const void *ref_y, const void *ref_uv, size_t ref_pitch,
                            const void *dis_y, const void *dis_uv, size_t dis_pitch, int32_t matrix, int32_t range,
                            int32_t on_host, void *stream) {
    if (!ctx || !ref_y || !ref_uv || !dis_y || !dis_uv) return S2_ERR_INVALID_ARG;
    if (matrix < S2_MATRIX_BT709 || matrix > S2_MATRIX_BT601_625 || (range != S2_RANGE_LIMITED && range != S2_RANGE_FULL))
        return S2_ERR_INVALID_ARG;
    if ((ctx->w & 1) || (ctx->h & 1)) return S2_ERR_INVALID_SIZE;
    const size_t row = (size_t)ctx->w * (fmt == S2_FMT_P016 ? 2 : 1);
    if (ref_pitch < row || dis_pitch < row) return S2_ERR_DIM_MISMATCH;
    const void *ry = ref_y, *ru = ref_uv, *dy = dis_y, *du = dis_uv;
    size_t rp = ref_pitch, dp = dis_pitch, tmp;
    if (on_host) {
        s2_status st = stage_host(ctx, 0, ref_y, ref_pitch, row, ctx->h, stream, &ry, &rp);
        if (st == S2_OK) st = stage_host(ctx, 1, dis_y, dis_pitch, row, ctx->h, stream, &dy, &dp);
        if (st == S2_OK) st = stage_host(ctx, 2, ref_uv, ref_pitch, row, ctx->h / 2, stream, &ru, &tmp);
        if (st == S2_OK) st = stage_host(ctx, 3, dis_uv, dis_pitch, row, ctx->h / 2, stream, &du, &tmp);
        if (st != S2_OK) return st;
    }
    s2_pair_desc d = make_desc(ctx->w, ctx->h, fmt, ry, rp, dy, dp);
    d.ref_uv = ru;
    d.dis_uv = du;
    d.matrix = matrix;
    d.range = range;
    return ctx_run(ctx, d, stream);
}

s2_status s2_compute_nv12(s2_ctx *ctx, const uint8_t *ref_y, const uint8_t *ref_uv, size_t ref_pitch,
                          const uint8_t *dis_y, const uint8_t *dis_uv, size_t dis_pitch, int32_t matrix,
                          int32_t range, int32_t on_host, void *stream) {
    return ctx_yuv420(ctx, S2_FMT_NV12, ref_y, ref_uv, ref_pitch, dis_y, dis_uv, dis_pitch, matrix, range, on_host,
                      stream);
}

s2_status s2_compute_p016(s2_ctx *ctx, const uint16_t *ref_y, const uint16_t *ref_uv, size_t ref_pitch,
                          const uint16_t *dis_y, const uint16_t *dis_uv, size_t dis_pitch, int32_t matrix,
                          int32_t range, int32_t on_host, void *stream) {
    return ctx_yuv420(ctx, S2_FMT_P016, ref_y, ref_uv, ref_pitch, dis_y, dis_uv, dis_pitch, matrix, range, on_host,
                      stream);
}

s2_status s2_compute_rgb16(s2_ctx *ctx, const uint16_t *ref, size_t ref_pitch, const uint16_t *dis,
                           size_t dis_pitch, int32_t bits, int32_t on_host, void *stream) {
    if (!ctx || !ref || !dis) return S2_ERR_INVALID_ARG;
    if (bits < 8 || bits > 16) return S2_ERR_INVALID_ARG;
    const size_t row = (size_t)ctx->w * 6;
    if (ref_pitch < row || dis_pitch < row) return S2_ERR_DIM_MISMATCH;
    const void *r = ref, *d = dis;
    size_t rp = ref_pitch, dp = dis_pitch;
    if (on_host) {
        s2_status st = stage_host(ctx, 0, ref, ref_pitch, row, ctx->h, stream, &r, &rp);
        if (st == S2_OK) st = stage_host(ctx, 1, dis, dis_pitch, row, ctx->h, stream, &d, &dp);
        if (st != S2_OK) return st;
    }
    s2_pair_desc desc = make_desc(ctx->w, ctx->h, S2_FMT_RGB16, r, rp, d, dp);
    desc.bits = bits;
    return ctx_run(ctx, desc, stream);
}

s2_status s2_get_result(s2_ctx *ctx, double *score, double stats[S2_NUM_STATS], double sums[S2_NUM_STATS]) {
    if (!ctx) return S2_ERR_INVALID_ARG;
    if (ctx->last_was_ref_build) return S2_ERR_NOT_READY;
    s2_status st = ctx->eng.wait();
    if (st != S2_OK) return st;
    const DevResult &r = ctx->eng.results_h[0];
    if (r.status != S2_OK) return (s2_status)r.status;
    if (score) *score = r.score;
    if (stats) memcpy(stats, r.stats, sizeof r.stats);
    if (sums) memcpy(sums, r.sums, sizeof r.sums);
    return S2_OK;
}

s2_status s2_compute_sync_linear_f32(s2_ctx *ctx, const float *ref, size_t ref_pitch, const float *dis,
                                     size_t dis_pitch, void *stream, double *score) {
    s2_status st = s2_compute_linear_f32(ctx, ref, ref_pitch, dis, dis_pitch, stream);
    if (st != S2_OK) return st;
    return s2_get_result(ctx, score, nullptr, nullptr);
}

// ---- cached reference ----------------------------------------------------
// set_reference converts the reference once and keeps its XYB planes of
// every scale on the device (set_reference_linear, ssimulacra2-cuda/src/
// lib.rs:440-546, keeps the reference's XYB, and also its blurred mu1_t and
// sigma11_t).  compute_with_reference converts only the distorted image and
// runs the same tile pass as a direct compute over the cached planes, so the
// scores equal the direct path's bit for bit.  The blurred reference moments
// are not kept: the tile pass blurs its planes as f32x2 pairs, so reading a
// cached mean saves no issue slot, and a candidate pass that did read it
// measured slower (3.50 against 3.23 ms per 63 1080p candidates).  Like the
// reference, set_reference returns after the device work is done.
static s2_status set_ref(s2_ctx *ctx, const s2_pair_desc &d, void *stream) {
    size_t off[kScales];
    const int ns = s2_num_scales_rule(ctx->w, ctx->h, ctx->eng.scale_rule);
    const size_t bytes = s2_image_levels_layout(ctx->w, ctx->h, ns, ctx->eng.esize(), off);
    if (ctx->ref_levels.n < bytes) {
        if (ctx->ref_levels.p) {
            S2_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
            cudaFree(ctx->ref_levels.p);
        }
        ctx->ref_levels.p = nullptr;
        ctx->ref_levels.n = 0;
        if (ctx->eng.budget && ctx->eng.allocated + bytes > ctx->eng.budget) {
            g_last_error = "reference cache over the HBM budget";
            return S2_ERR_OOM;
        }
        S2_CUDA(cudaMalloc(&ctx->ref_levels.p, bytes));
        ctx->ref_levels.n = bytes;
    }
    PairExtra build;
    build.prep_mask = 1;
    build.score = false;
    build.dssim = false;
    for (int s = 0; s < kScales; s++) build.ref_levels[s] = s < ns ? (char *)ctx->ref_levels.p + off[s] : nullptr;
    ctx->has_ref = false;
    s2_status st = ctx_run(ctx, d, stream, &build);
    if (st != S2_OK) return st;
    S2_CUDA(cudaEventSynchronize(ctx->eng.done));
    ctx->eng.pending = false;
    ctx->ref_extra = build;
    ctx->ref_extra.prep_mask = 2;
    ctx->ref_extra.score = true;
    ctx->has_ref = true;
    return S2_OK;
}

s2_status s2_set_reference_linear_f32(s2_ctx *ctx, const float *ref, size_t pitch, void *stream) {
    if (!ctx || !ref) return S2_ERR_INVALID_ARG;
    if (pitch < (size_t)ctx->w * 12) return S2_ERR_DIM_MISMATCH;
    return set_ref(ctx, make_desc(ctx->w, ctx->h, S2_FMT_LINEAR_F32, ref, pitch, nullptr, 0), stream);
}

s2_status s2_set_reference_srgb8(s2_ctx *ctx, const uint8_t *ref, size_t pitch, int32_t on_host, void *stream) {
    if (!ctx || !ref) return S2_ERR_INVALID_ARG;
    const size_t row = (size_t)ctx->w * 3;
    if (pitch < row) return S2_ERR_DIM_MISMATCH;
    const void *r = ref;
    size_t rp = pitch;
    if (on_host) {
        s2_status st = stage_host(ctx, 0, ref, pitch, row, ctx->h, stream, &r, &rp);
        if (st != S2_OK) return st;
    }
    return set_ref(ctx, make_desc(ctx->w, ctx->h, S2_FMT_SRGB8, r, rp, nullptr, 0), stream);
}

s2_status s2_compute_with_reference_linear_f32(s2_ctx *ctx, const float *dis, size_t pitch, void *stream) {
    if (!ctx || !dis) return S2_ERR_INVALID_ARG;
    if (!ctx->has_ref) return S2_ERR_NO_REFERENCE;
    if (pitch < (size_t)ctx->w * 12) return S2_ERR_DIM_MISMATCH;
    return ctx_run(ctx, make_desc(ctx->w, ctx->h, S2_FMT_LINEAR_F32, nullptr, 0, dis, pitch), stream,
                   &ctx->ref_extra);
}

s2_status s2_compute_with_reference_srgb8(s2_ctx *ctx, const uint8_t *dis, size_t pitch, int32_t on_host,
                                          void *stream) {
    if (!ctx || !dis) return S2_ERR_INVALID_ARG;
    if (!ctx->has_ref) return S2_ERR_NO_REFERENCE;
    const size_t row = (size_t)ctx->w * 3;
    if (pitch < row) return S2_ERR_DIM_MISMATCH;
    const void *d = dis;
    size_t dp = pitch;
    if (on_host) {
        s2_status st = stage_host(ctx, 1, dis, pitch, row, ctx->h, stream, &d, &dp);
        if (st != S2_OK) return st;
    }
    return ctx_run(ctx, make_desc(ctx->w, ctx->h, S2_FMT_SRGB8, nullptr, 0, d, dp), stream, &ctx->ref_extra);
}

s2_status s2_clear_reference(s2_ctx *ctx) {
    if (!ctx) return S2_ERR_INVALID_ARG;
    ctx->has_ref = false;
    return S2_OK;
}

int32_t s2_has_reference(const s2_ctx *ctx) { return ctx && ctx->has_ref ? 1 : 0; }

s2_status s2_error_maps(s2_ctx *ctx, int32_t scale, float *maps, size_t pitch, void *stream) {
    if (!ctx || !maps) return S2_ERR_INVALID_ARG;
    Engine &e = ctx->eng;
    Plan &P = ctx->plan;
    if (e.last_n != 1 || P.pairs.empty() || ctx->last_was_ref_build) return S2_ERR_NOT_READY;
    if (e.blur != S2_BLUR_FIR) return S2_ERR_INVALID_ARG;
    const DevPair &p = P.pairs[0];
    if (p.status != S2_OK || scale < 0 || scale >= p.nscales) return S2_ERR_INVALID_ARG;
    const size_t row = (size_t)p.w[scale] * sizeof(float);
    if (pitch < row || pitch % sizeof(float)) return S2_ERR_DIM_MISMATCH;
    // the last compute's descriptors and XYB planes are still in the
    // workspace; re-run its tile pass over this scale with the export on
    const int t0 = p.tile_base[scale], t1 = t0 + p.tile_cnt[scale];
    const size_t pb = s2_align_up(sizeof(DevPair), 256), bb = s2_align_up(sizeof(int), 256);
    char *dbase = (char *)e.pairs_d.p;
    cudaStream_t st = (cudaStream_t)stream;
    const long long mpitch = (long long)(pitch / sizeof(float));
    S2_CUDA(cudaMemsetAsync(e.counter_d.p, 0, Engine::kCounterBytes, st));
    S2_CUDA(launch_fused_export(e.storage, (const DevPair *)dbase, (const Seg *)(dbase + pb + bb),
                                (int)P.segs.size(), t0, t1, (int *)e.counter_d.p, tile_check(e.err_word()),
                                (double *)e.partials_d.p, maps, mpitch, mpitch * p.h[scale], e.num_sms * e.fused_bps,
                                st));
    // the tile pass's time-out word (set only if its row copies never landed)
    int err = 0;
    S2_CUDA(cudaMemcpyAsync(&err, e.err_word(), sizeof err, cudaMemcpyDeviceToHost, st));
    S2_CUDA(cudaStreamSynchronize(st));
    if (err) {
        g_last_error = "tile pass: row copies timed out";
        return S2_ERR_TIMEOUT;
    }
    return S2_OK;
}

// ---- batches -----------------------------------------------------------
s2_status s2_batch_create(const s2_config *cfg_in, uint32_t max_pairs, uint64_t max_pixels, s2_batch **out) {
    if (!out || max_pairs == 0) return S2_ERR_INVALID_ARG;
    *out = nullptr;
    s2_config cfg;
    if (cfg_in) cfg = *cfg_in;
    else s2_config_default(&cfg);
    s2_status st = check_cfg(&cfg);
    if (st != S2_OK) return st;
    s2_batch *b = new (std::nothrow) s2_batch();
    if (!b) return S2_ERR_OOM;
    b->max_pairs = max_pairs;
    b->max_pixels = max_pixels;
    b->cfg = cfg;
    st = b->open_slot(0);
    if (st != S2_OK) {
        delete b;
        return st;
    }
    *out = b;
    return S2_OK;
}

void s2_batch_destroy(s2_batch *b) {
    if (!b) return;
    for (int k = 0; k < 2; k++)
        if (b->ready[k]) b->eng[k].release();
    if (b->ref_buf.p) cudaFree(b->ref_buf.p);
    delete b;
}

s2_status s2_batch_submit(s2_batch *b, const s2_pair_desc *pairs, uint32_t n, void *stream) {
    if (!b || (!pairs && n)) return S2_ERR_INVALID_ARG;
    if (n > b->max_pairs) return S2_ERR_INVALID_ARG;
    const int k = b->take_slot(false);
    Engine &e = b->eng[k];
    s2_status st = e.plan(pairs, (int)n, b->plan[k]);
    if (st == S2_OK) st = e.tune(pairs, (int)n, b->plan[k], nullptr, (cudaStream_t)stream);
    if (st == S2_OK) st = e.enqueue(b->plan[k], (cudaStream_t)stream);
    if (st != S2_OK) return st;
    b->unread.push_back(k);
    b->last_slot = k;
    return S2_OK;
}

s2_status s2_batch_submit_host(s2_batch *b, const s2_pair_desc *pairs, uint32_t n, void *stream) {
    if (!b || (!pairs && n)) return S2_ERR_INVALID_ARG;
    if (n > b->max_pairs) return S2_ERR_INVALID_ARG;
    for (uint32_t i = 0; i < n; i++) {
        const size_t row = s2_row_bytes(pairs[i]);
        if (pairs[i].ref_pitch < row || pairs[i].dis_pitch < row) return S2_ERR_DIM_MISMATCH;
    }
    const int k = b->take_slot(true);
    s2_status st = b->open_slot(k);
    if (st != S2_OK) return st;
    Engine &e = b->eng[k];
    // S2_BLUR_IIR_REF runs its two passes over all pairs at once: one group
    const int ng = e.blur == S2_BLUR_IIR_REF ? 1 : std::min<int>(kMaxGroups, std::max<int>(1, (int)n / 4));
    st = e.plan(pairs, (int)n, b->plan[k], nullptr, ng);
    if (st == S2_OK) st = e.enqueue(b->plan[k], (cudaStream_t)stream, pairs);
    if (st != S2_OK) return st;
    b->unread.push_back(k);
    b->last_slot = k;
    return S2_OK;
}

// Cached reference of a batch: ssim2-gpu's Ssim2Batch::set_reference /
// compute_batch (crates/ssim2-gpu/src/pipeline_batch.rs:206-330), where every
// candidate of a submission is scored against one resident reference.  The
// reference's XYB pyramid is built once, on slot 0's engine, and kept in a
// buffer of the batch.
s2_status s2_batch_set_reference(s2_batch *b, const s2_pair_desc *ref, void *stream) {
    if (!b || !ref || !ref->ref) return S2_ERR_INVALID_ARG;
    if (!(b->metrics & S2_METRIC_SSIMULACRA2)) return S2_ERR_INVALID_ARG;
    Engine &e = b->eng[0];
    const uint32_t w = ref->width, h = ref->height;
    const int ns = s2_num_scales_rule(w, h, e.scale_rule);
    if (ns == 0 || w > (1u << 16) || h > (1u << 16)) return S2_ERR_INVALID_SIZE;
    if ((uint64_t)w * h > b->max_pixels) return S2_ERR_INVALID_SIZE;
    size_t off[kScales];
    const size_t bytes = s2_image_levels_layout(w, h, ns, e.esize(), off);
    b->has_ref = false;
    if (b->ref_buf.n < bytes) {
        S2_CUDA(cudaDeviceSynchronize());  // earlier submissions may still read the old cache
        if (b->ref_buf.p) cudaFree(b->ref_buf.p);
        b->ref_buf.p = nullptr;
        b->ref_buf.n = 0;
        if (e.budget && e.allocated + b->eng[1].allocated + bytes > e.budget) {
            g_last_error = "reference cache over the HBM budget";
            return S2_ERR_OOM;
        }
        S2_CUDA(cudaMalloc(&b->ref_buf.p, bytes));
        b->ref_buf.n = bytes;
    }
    PairExtra build;
    build.prep_mask = 1;
    build.score = false;
    build.dssim = false;
    for (int s = 0; s < kScales; s++) build.ref_levels[s] = s < ns ? (char *)b->ref_buf.p + off[s] : nullptr;
    s2_pair_desc d = *ref;
    d.dis = nullptr;
    d.dis_uv = nullptr;
    const int k = b->take_slot(false);
    s2_status st = e.plan(&d, 1, b->plan[k], &build);
    if (st == S2_OK && b->plan[k].pairs[0].status != S2_OK) st = (s2_status)b->plan[k].pairs[0].status;
    if (st == S2_OK) st = e.enqueue(b->plan[k], (cudaStream_t)stream);
    if (st == S2_OK) st = e.wait();
    if (st != S2_OK) return st;
    b->ref_extra = build;
    b->ref_extra.prep_mask = 2;
    b->ref_extra.score = true;
    b->ref_w = w;
    b->ref_h = h;
    b->has_ref = true;
    return S2_OK;
}

s2_status s2_batch_submit_with_reference(s2_batch *b, const s2_pair_desc *dis, uint32_t n, void *stream) {
    if (!b || (!dis && n)) return S2_ERR_INVALID_ARG;
    if (!b->has_ref) return S2_ERR_NO_REFERENCE;
    if (n > b->max_pairs || (uint64_t)n * b->ref_w * b->ref_h > b->max_pixels) return S2_ERR_INVALID_ARG;
    std::vector<s2_pair_desc> d(dis, dis + n);
    for (uint32_t i = 0; i < n; i++) {
        if (d[i].width != b->ref_w || d[i].height != b->ref_h) return S2_ERR_DIM_MISMATCH;
        if (!d[i].dis) return S2_ERR_INVALID_ARG;
        d[i].ref = nullptr;
        d[i].ref_uv = nullptr;
    }
    std::vector<PairExtra> ex(n, b->ref_extra);
    const int k = b->take_slot(false);
    Engine &e = b->eng[k];
    const int m = e.metrics;
    e.metrics = S2_METRIC_SSIMULACRA2;  // the cached reference keeps SSIMULACRA2's planes only
    s2_status st = e.plan(d.data(), (int)n, b->plan[k], ex.data());
    if (st == S2_OK) st = e.tune(d.data(), (int)n, b->plan[k], ex.data(), (cudaStream_t)stream);
    if (st == S2_OK) st = e.enqueue(b->plan[k], (cudaStream_t)stream);
    e.metrics = m;
    if (st != S2_OK) return st;
    b->unread.push_back(k);
    b->last_slot = k;
    return S2_OK;
}

s2_status s2_batch_clear_reference(s2_batch *b) {
    if (!b) return S2_ERR_INVALID_ARG;
    b->has_ref = false;
    return S2_OK;
}

int32_t s2_batch_has_reference(const s2_batch *b) { return b && b->has_ref ? 1 : 0; }

s2_status s2_batch_results(s2_batch *b, s2_result *out, uint32_t n) {
    if (!b || (!out && n)) return S2_ERR_INVALID_ARG;
    int k = b->last_slot;  // no unread submission: the last one again
    if (!b->unread.empty()) {
        k = b->unread.front();
        b->unread.pop_front();
    }
    Engine &e = b->eng[k];
    s2_status st = e.wait();
    if (st != S2_OK) return st;
    if ((int)n > e.last_n) return S2_ERR_INVALID_ARG;
    for (uint32_t i = 0; i < n; i++) {
        const DevResult &r = e.results_h[i];
        out[i].score = r.score;
        memcpy(out[i].stats, r.stats, sizeof r.stats);
        memcpy(out[i].sums, r.sums, sizeof r.sums);
        out[i].n_scales = r.n_scales;
        out[i].status = r.status;
        const bool ds = (b->plan[k].metrics & S2_METRIC_DSSIM) != 0;
        out[i].dssim = ds ? r.dssim : std::nan("");
        for (int s = 0; s < kDsLevels; s++) out[i].dssim_scale[s] = ds ? r.dssim_scale[s] : std::nan("");
    }
    return S2_OK;
}

s2_status s2_batch_mem_usage(const s2_batch *b, size_t *bytes) {
    if (!b || !bytes) return S2_ERR_INVALID_ARG;
    *bytes = b->eng[0].allocated + (b->ready[1] ? b->eng[1].allocated : 0) + b->ref_buf.n;
    return S2_OK;
}

s2_status s2_batch_set_profiling(s2_batch *b, int32_t enable) {
    if (!b) return S2_ERR_INVALID_ARG;
    b->profiling = enable != 0;
    for (int k = 0; k < 2; k++)
        if (b->ready[k]) {
            const s2_status st = b->eng[k].set_profiling(b->profiling);
            if (st != S2_OK) return st;
        }
    return S2_OK;
}

s2_status s2_batch_last_timings(s2_batch *b, float ms[3]) {
    if (!b || !ms) return S2_ERR_INVALID_ARG;
    return b->eng[b->last_slot].timings(ms);
}

s2_status s2_profile_enable(s2_ctx *ctx, int32_t enable) {
    if (!ctx) return S2_ERR_INVALID_ARG;
    return ctx->eng.set_profiling(enable != 0);
}

s2_status s2_profile_last(s2_ctx *ctx, float ms[3]) {
    if (!ctx || !ms) return S2_ERR_INVALID_ARG;
    return ctx->eng.timings(ms);
}

int32_t s2_fused_blocks_per_sm(int32_t storage) { return s2_global_init() == S2_OK ? fused_blocks_per_sm(storage) : 0; }

s2_status s2_batch_set_graphs(s2_batch *b, int32_t enable) {
    if (!b) return S2_ERR_INVALID_ARG;
    b->graphs = enable != 0;
    for (int k = 0; k < 2; k++)
        if (b->ready[k]) {
            b->eng[k].graphs = b->graphs;
            if (!b->graphs) b->eng[k].drop_graphs();
        }
    return S2_OK;
}

s2_status s2_set_graphs(s2_ctx *ctx, int32_t enable) {
    if (!ctx) return S2_ERR_INVALID_ARG;
    ctx->eng.graphs = enable != 0;
    if (!ctx->eng.graphs) ctx->eng.drop_graphs();
    return S2_OK;
}

// ---- DSSIM --------------------------------------------------------------
static bool metrics_ok(int32_t m) { return m >= 1 && m <= 3; }

s2_status s2_set_metrics(s2_ctx *ctx, int32_t metrics) {
    if (!ctx || !metrics_ok(metrics)) return S2_ERR_INVALID_ARG;
    if ((metrics & S2_METRIC_SSIMULACRA2) && s2_num_scales_rule(ctx->w, ctx->h, ctx->eng.scale_rule) == 0)
        return S2_ERR_INVALID_SIZE;
    if ((metrics & S2_METRIC_DSSIM) && (ctx->w < 8 || ctx->h < 8)) return S2_ERR_INVALID_SIZE;
    ctx->eng.metrics = metrics;
    return S2_OK;
}

s2_status s2_batch_set_metrics(s2_batch *b, int32_t metrics) {
    if (!b || !metrics_ok(metrics)) return S2_ERR_INVALID_ARG;
    b->metrics = metrics;
    for (int k = 0; k < 2; k++)
        if (b->ready[k]) b->eng[k].metrics = metrics;
    return S2_OK;
}

s2_status s2_batch_last_dssim_ms(s2_batch *b, float *ms) {
    if (!b || !ms) return S2_ERR_INVALID_ARG;
    float t[3];
    return b->eng[b->last_slot].timings(t, ms);
}

s2_status s2_get_dssim(s2_ctx *ctx, double *dssim, double scale_scores[5]) {
    if (!ctx) return S2_ERR_INVALID_ARG;
    if (ctx->last_was_ref_build) return S2_ERR_NOT_READY;
    s2_status st = ctx->eng.wait();
    if (st != S2_OK) return st;
    const Plan &P = ctx->plan;
    if (!(P.metrics & S2_METRIC_DSSIM) || P.ds.empty() || P.ds[0].status == -1) return S2_ERR_NOT_READY;
    const DevResult &r = ctx->eng.results_h[0];
    if (r.status != S2_OK) return (s2_status)r.status;
    if (dssim) *dssim = r.dssim;
    if (scale_scores)
        for (int s = 0; s < kDsLevels; s++) scale_scores[s] = r.dssim_scale[s];
    return S2_OK;
}

// s2_dssim: a context scoring DSSIM only.  A full compute leaves both
// images' Lab planes in the context's workspace at offsets fixed by its size;
// compute_dis_only converts the distorted image alone and reads the
// reference's planes from there.
struct s2_dssim {
    s2_ctx *ctx = nullptr;
    bool has_ref = false;
};

s2_status s2_dssim_create(int32_t device, uint32_t width, uint32_t height, s2_dssim **out) {
    if (!out) return S2_ERR_INVALID_ARG;
    *out = nullptr;
    s2_config cfg;
    s2_config_default(&cfg);
    cfg.device = device;
    s2_dssim *d = new (std::nothrow) s2_dssim();
    if (!d) return S2_ERR_OOM;
    s2_status st = ctx_create(&cfg, width, height, S2_METRIC_DSSIM, &d->ctx);
    if (st != S2_OK) {
        delete d;
        return st;
    }
    *out = d;
    return S2_OK;
}

void s2_dssim_destroy(s2_dssim *d) {
    if (!d) return;
    s2_destroy(d->ctx);
    delete d;
}

s2_status s2_dssim_compute_srgb8(s2_dssim *d, const uint8_t *ref, size_t ref_pitch, const uint8_t *dis,
                                 size_t dis_pitch, int32_t on_host, void *stream, double *dssim) {
    if (!d || !dssim) return S2_ERR_INVALID_ARG;
    d->has_ref = false;
    s2_status st = s2_compute_srgb8(d->ctx, ref, ref_pitch, dis, dis_pitch, on_host, stream);
    if (st == S2_OK) st = s2_get_dssim(d->ctx, dssim, nullptr);
    if (st == S2_OK) d->has_ref = true;
    return st;
}

s2_status s2_dssim_compute_dis_only_srgb8(s2_dssim *d, const uint8_t *dis, size_t dis_pitch, int32_t on_host,
                                          void *stream, double *dssim) {
    if (!d || !dis || !dssim) return S2_ERR_INVALID_ARG;
    if (!d->has_ref) return S2_ERR_NO_REFERENCE;
    s2_ctx *ctx = d->ctx;
    const size_t row = (size_t)ctx->w * 3;
    if (dis_pitch < row) return S2_ERR_DIM_MISMATCH;
    const void *dv = dis;
    size_t dp = dis_pitch;
    if (on_host) {
        s2_status st = stage_host(ctx, 1, dis, dis_pitch, row, ctx->h, stream, &dv, &dp);
        if (st != S2_OK) return st;
    }
    PairExtra ex;
    ex.prep_mask = 2;
    s2_status st = ctx_run(ctx, make_desc(ctx->w, ctx->h, S2_FMT_SRGB8, nullptr, 0, dv, dp), stream, &ex);
    if (st == S2_OK) st = s2_get_dssim(ctx, dssim, nullptr);
    return st;
}

s2_status s2_dssim_mem_usage(const s2_dssim *d, size_t *bytes) {
    if (!d) return S2_ERR_INVALID_ARG;
    return s2_mem_usage(d->ctx, bytes);
}

}  // extern "C"
