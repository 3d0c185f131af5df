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
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/ssim2b200.h"
#include "ssim2_launch.h"

using namespace s2;

// ---------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------
static thread_local std::string g_last_error;

static s2_status cuda_fail(cudaError_t e, const char *what) {
    char buf[256];
    snprintf(buf, sizeof buf, "%s: %s (%d)", what, cudaGetErrorString(e), (int)e);
    g_last_error = buf;
    return e == cudaErrorMemoryAllocation ? S2_ERR_OOM : S2_ERR_CUDA;
}
#define S2_CUDA(call)                                    \
    do {                                                 \
        cudaError_t e_ = (call);                         \
        if (e_ != cudaSuccess) return cuda_fail(e_, #call); \
    } while (0)

// ---------------------------------------------------------------------------
// constants shared by all engines
// ---------------------------------------------------------------------------
// sRGB8 -> linear table of the reference (ssimulacra2-cuda-kernel/src/srgb.rs:23-51).
// The entries follow the gamma-2.4 sRGB curve with a linear toe but were
// printed with 6-9 decimal digits; the table, not the formula, defines the
// reference's conversion, so the same numbers are used (hex-float spelling).
static const float kSrgb8Lut[256] = {
#include "srgb8_lut.inc"
};

static void kr_kb_from_primaries(const double prim[8], double *kr, double *kb) {
    // cuda-colorspace-kernel/src/lib.rs:205-221, in double
    double xyz[4][3];
    for (int i = 0; i < 4; i++) {
        double x = prim[2 * i], y = prim[2 * i + 1];
        xyz[i][0] = x / y;
        xyz[i][1] = 1.0;
        xyz[i][2] = (1.0 - x - y) / y;
    }
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

static ColorConsts make_color_consts() {
    static const double BT709[8] = {0.640, 0.330, 0.300, 0.600, 0.150, 0.060, 0.3127, 0.3290};
    static const double BT2020[8] = {0.708, 0.292, 0.170, 0.797, 0.131, 0.046, 0.3127, 0.3290};
    ColorConsts cc;
    double kr, kb;
    kr_kb_from_primaries(BT709, &kr, &kb);
    double kg = 1.0 - kr - kb;
    // cuda-colorspace-kernel/src/lib.rs:188-203, 8-bit limited range
    double c[5] = {1.0 / 219.0, 2.0 * (1.0 - kr) / 224.0, 2.0 * (1.0 - kb) / 224.0,
                   -2.0 * (1.0 - kb) * kb / kg / 224.0, -2.0 * (1.0 - kr) * kr / kg / 224.0};
    for (int i = 0; i < 5; i++) cc.nv12[i] = (float)c[i];
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

static s2_status global_init() {
    std::call_once(g_init_once, [] {
        if (!check_taps()) {
            g_last_error = "FIR taps compiled into the kernels do not match the derivation";
            g_init_status = S2_ERR_CUDA;
            return;
        }
        cudaError_t e = configure_kernels();
        if (e == cudaSuccess) e = upload_weights();
        if (e != cudaSuccess) g_init_status = cuda_fail(e, "kernel set-up");
    });
    return g_init_status;
}

// ---------------------------------------------------------------------------
// device buffers
// ---------------------------------------------------------------------------
struct DevBuf {
    void *p = nullptr;
    size_t n = 0;
};

static size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

static int num_scales_rule(uint32_t w, uint32_t h, int rule) {
    if (w < 1 || h < 1) return 0;
    if (rule == S2_SCALES_ALL6) return kScales;
    if (w < 8 || h < 8) return 0;
    int n = 0;
    uint64_t cw = w, ch = h;
    if (rule == S2_SCALES_MIN8) {
        while (n < kScales && cw >= 8 && ch >= 8) {
            n++;
            cw = (cw + 1) / 2;
            ch = (ch + 1) / 2;
        }
        return n;
    }
    // CPU crate: scale s > 0 is produced when scale s-1 is at least 8x8
    n = 1;
    for (int s = 1; s < kScales; s++) {
        if (cw < 8 || ch < 8) break;
        n++;
        cw = (cw + 1) / 2;
        ch = (ch + 1) / 2;
    }
    return n;
}

// One planned submission.
struct Plan {
    std::vector<DevPair> pairs;
    std::vector<int> blk_first;
    std::vector<Seg> segs;
    int total_blocks = 0;
    int total_tiles = 0;
    size_t level_bytes = 0;  // both images, all levels, all pairs
    int strip_rows = 63;
};

struct Engine {
    int device = 0;
    int storage = ST_F32;
    int scale_rule = S2_SCALES_CPU;
    int strip_rows_cfg = 0;
    int blur = S2_BLUR_FIR;
    uint64_t budget = 0;
    size_t allocated = 0;
    int num_sms = 148;
    int fused_bps = 1;
    ColorConsts cc;

    DevBuf pairs_d, blk_d, segs_d, counter_d, partials_d, results_d, levels_d, lut_d;
    void *pinned = nullptr;  // staging: pairs | blk_first | segs
    size_t pinned_n = 0;
    DevResult *results_h = nullptr;
    size_t results_cap = 0;
    cudaEvent_t done = nullptr;
    int last_n = -1;
    bool pending = false;
    bool profiling = false;
    cudaEvent_t prof[4] = {nullptr, nullptr, nullptr, nullptr};

    size_t esize() const { return storage == ST_F32 ? 4 : 2; }

    s2_status init(const s2_config *cfg) {
        s2_status st = global_init();
        if (st != S2_OK) return st;
        device = cfg->device;
        storage = cfg->storage;
        scale_rule = cfg->scale_rule;
        strip_rows_cfg = cfg->strip_rows;
        blur = cfg->blur;
        budget = cfg->hbm_budget;
        S2_CUDA(cudaSetDevice(device));
        S2_CUDA(cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, device));
        fused_bps = fused_blocks_per_sm(storage);
        cc = make_color_consts();
        S2_CUDA(cudaEventCreateWithFlags(&done, cudaEventDisableTiming));
        st = ensure(lut_d, sizeof kSrgb8Lut);
        if (st != S2_OK) return st;
        S2_CUDA(cudaMemcpy(lut_d.p, kSrgb8Lut, sizeof kSrgb8Lut, cudaMemcpyHostToDevice));
        st = ensure(counter_d, 256);
        return st;
    }

    s2_status set_profiling(bool on) {
        if (on && !prof[0])
            for (cudaEvent_t &e : prof) S2_CUDA(cudaEventCreate(&e));
        profiling = on;
        return S2_OK;
    }

    s2_status timings(float ms[3]) {
        if (!profiling || last_n < 0) return S2_ERR_NOT_READY;
        S2_CUDA(cudaEventSynchronize(prof[3]));
        for (int i = 0; i < 3; i++) S2_CUDA(cudaEventElapsedTime(&ms[i], prof[i], prof[i + 1]));
        return S2_OK;
    }

    void release() {
        if (device >= 0) cudaSetDevice(device);
        if (done) cudaEventSynchronize(done);
        for (cudaEvent_t &e : prof)
            if (e) cudaEventDestroy(e), e = nullptr;
        for (DevBuf *b : {&pairs_d, &blk_d, &segs_d, &counter_d, &partials_d, &results_d, &levels_d, &lut_d})
            if (b->p) cudaFree(b->p), b->p = nullptr, b->n = 0;
        if (pinned) cudaFreeHost(pinned), pinned = nullptr;
        if (results_h) cudaFreeHost(results_h), results_h = nullptr;
        if (done) cudaEventDestroy(done), done = nullptr;
        allocated = 0;
    }

    // Grow-only device allocation, checked against the budget.
    s2_status ensure(DevBuf &b, size_t bytes) {
        if (b.n >= bytes) return S2_OK;
        bytes = align_up(bytes, 4096);
        if (budget && allocated - b.n + bytes > budget) {
            g_last_error = "allocation over the HBM budget";
            return S2_ERR_OOM;
        }
        if (b.p) {
            if (done) cudaEventSynchronize(done);
            cudaFree(b.p);
            allocated -= b.n;
            b.p = nullptr;
            b.n = 0;
        }
        S2_CUDA(cudaMalloc(&b.p, bytes));
        b.n = bytes;
        allocated += bytes;
        return S2_OK;
    }

    s2_status ensure_pinned(size_t bytes, size_t nres) {
        if (pinned_n < bytes) {
            if (pinned) {
                if (done) cudaEventSynchronize(done);
                cudaFreeHost(pinned);
            }
            pinned = nullptr;
            bytes = align_up(bytes, 4096);
            S2_CUDA(cudaMallocHost(&pinned, bytes));
            pinned_n = bytes;
        }
        if (results_cap < nres) {
            if (results_h) {
                if (done) cudaEventSynchronize(done);
                cudaFreeHost(results_h);
            }
            results_h = nullptr;
            S2_CUDA(cudaMallocHost((void **)&results_h, nres * sizeof(DevResult)));
            results_cap = nres;
        }
        return S2_OK;
    }

    int choose_strip_rows(const std::vector<uint64_t> &tiles_at) const {
        if (strip_rows_cfg == 9 || strip_rows_cfg == 21 || strip_rows_cfg == 63) return strip_rows_cfg;
        // largest strip height that still gives ~4 waves of resident tiles
        const uint64_t resident = (uint64_t)num_sms * (uint64_t)fused_bps;
        if (tiles_at[0] >= 4 * resident) return 63;
        if (tiles_at[1] >= 4 * resident) return 21;
        return 9;
    }

    // Lay out the levels and tiles of n pairs.
    s2_status plan(const s2_pair_desc *d, int n, Plan &P) {
        P = Plan();
        P.pairs.resize(n);
        P.blk_first.resize(n);
        // tile counts at strip heights 64/32 for the strip choice
        std::vector<uint64_t> tiles_at(2, 0);
        std::vector<int> ns(n);
        for (int i = 0; i < n; i++) {
            ns[i] = num_scales_rule(d[i].width, d[i].height, scale_rule);
            uint64_t w = d[i].width, h = d[i].height;
            for (int s = 0; s < ns[i]; s++) {
                tiles_at[0] += ((w + kTileW - 1) / kTileW) * ((h + 62) / 63);
                tiles_at[1] += ((w + kTileW - 1) / kTileW) * ((h + 20) / 21);
                w = (w + 1) / 2;
                h = (h + 1) / 2;
            }
        }
        P.strip_rows = choose_strip_rows(tiles_at);
        size_t lvl_off = 0;
        int blk = 0;
        for (int i = 0; i < n; i++) {
            DevPair &p = P.pairs[i];
            memset(&p, 0, sizeof p);
            const s2_pair_desc &q = d[i];
            p.in[0] = q.ref;
            p.in[1] = q.dis;
            p.in_uv[0] = q.ref_uv;
            p.in_uv[1] = q.dis_uv;
            p.pitch[0] = (long long)q.ref_pitch;
            p.pitch[1] = (long long)q.dis_pitch;
            p.fmt = q.format;
            p.bits = q.bits;
            p.nscales = ns[i];
            p.status = S2_OK;
            if (ns[i] == 0 || q.width > (1u << 16) || q.height > (1u << 16)) {
                p.status = S2_ERR_INVALID_SIZE;
                p.nscales = 0;
                P.blk_first[i] = blk;
                continue;
            }
            if (q.format < 0 || q.format > 3 || !q.ref || !q.dis ||
                (q.format == S2_FMT_NV12 && (!q.ref_uv || !q.dis_uv || (q.width & 1) || (q.height & 1))) ||
                (q.format == S2_FMT_RGB16 && (q.bits < 8 || q.bits > 16))) {
                p.status = S2_ERR_INVALID_ARG;
                p.nscales = 0;
                P.blk_first[i] = blk;
                continue;
            }
            p.w[0] = (int)q.width;
            p.h[0] = (int)q.height;
            for (int s = 1; s < kScales; s++) {
                p.w[s] = (p.w[s - 1] + 1) / 2;
                p.h[s] = (p.h[s - 1] + 1) / 2;
            }
            for (int s = 0; s < p.nscales; s++) {
                p.lp[s] = (int)align_up((size_t)p.w[s], 64);
                size_t bytes = align_up((size_t)3 * p.lp[s] * p.h[s] * esize(), 256);
                p.lvl[0][s] = (void *)lvl_off;  // offsets, rebased at upload
                lvl_off += bytes;
                p.lvl[1][s] = (void *)lvl_off;
                lvl_off += bytes;
            }
            P.blk_first[i] = blk;
            {
                p.blk_x = (p.w[0] + kPyrBlk - 1) / kPyrBlk;
                p.blk_y = (p.h[0] + kPyrBlk - 1) / kPyrBlk;
                p.blk_base = blk;
                blk += p.blk_x * p.blk_y;
            }
        }
        P.total_blocks = blk;
        P.level_bytes = lvl_off;
        // tiles: all pairs' scale 0 first, then scale 1, ... (largest work first)
        int tile = 0;
        for (int s = 0; s < kScales; s++) {
            for (int i = 0; i < n; i++) {
                DevPair &p = P.pairs[i];
                if (p.status != S2_OK || s >= p.nscales) continue;
                Seg sg;
                sg.first_tile = tile;
                sg.pair = i;
                sg.scale = s;
                sg.tiles_x = (p.w[s] + kTileW - 1) / kTileW;
                sg.strip_rows = P.strip_rows;
                int ty = (p.h[s] + P.strip_rows - 1) / P.strip_rows;
                p.tile_base[s] = tile;
                p.tile_cnt[s] = sg.tiles_x * ty;
                tile += p.tile_cnt[s];
                P.segs.push_back(sg);
            }
        }
        P.total_tiles = tile;
        return S2_OK;
    }

    s2_status enqueue(Plan &P, cudaStream_t st) {
        const int n = (int)P.pairs.size();
        s2_status r;
        if ((r = ensure(levels_d, std::max<size_t>(P.level_bytes, 256))) != S2_OK) return r;
        if ((r = ensure(partials_d, std::max<size_t>((size_t)P.total_tiles * 18 * sizeof(double), 256))) != S2_OK) return r;
        if ((r = ensure(results_d, (size_t)n * sizeof(DevResult))) != S2_OK) return r;
        const size_t pb = align_up(n * sizeof(DevPair), 256), bb = align_up(n * sizeof(int), 256),
                     sb = align_up(std::max<size_t>(P.segs.size(), 1) * sizeof(Seg), 256);
        if ((r = ensure(pairs_d, pb + bb + sb)) != S2_OK) return r;
        if ((r = ensure_pinned(pb + bb + sb, n)) != S2_OK) return r;
        // the previous submission may still read the pinned staging
        if (pending) S2_CUDA(cudaEventSynchronize(done));
        char *h = (char *)pinned;
        DevPair *hp = (DevPair *)h;
        for (int i = 0; i < n; i++) {
            hp[i] = P.pairs[i];
            for (int s = 0; s < kScales; s++)
                for (int img = 0; img < 2; img++)
                    if (s < hp[i].nscales) hp[i].lvl[img][s] = (char *)levels_d.p + (size_t)hp[i].lvl[img][s];
                    else hp[i].lvl[img][s] = nullptr;
        }
        memcpy(h + pb, P.blk_first.data(), n * sizeof(int));
        if (!P.segs.empty()) memcpy(h + pb + bb, P.segs.data(), P.segs.size() * sizeof(Seg));
        char *dbase = (char *)pairs_d.p;
        const DevPair *dpairs = (const DevPair *)dbase;
        const int *dblk = (const int *)(dbase + pb);
        const Seg *dsegs = (const Seg *)(dbase + pb + bb);
        S2_CUDA(cudaMemcpyAsync(dbase, h, pb + bb + sb, cudaMemcpyHostToDevice, st));
        S2_CUDA(cudaMemsetAsync(counter_d.p, 0, sizeof(int), st));
        if (profiling) S2_CUDA(cudaEventRecord(prof[0], st));
        S2_CUDA(launch_pyramid(storage, dpairs, n, dblk, P.total_blocks, cc, (const float *)lut_d.p,
                               num_sms * 8, st));
        if (profiling) S2_CUDA(cudaEventRecord(prof[1], st));
        S2_CUDA(launch_fused(storage, dpairs, dsegs, (int)P.segs.size(), P.total_tiles, (int *)counter_d.p,
                             (double *)partials_d.p, cc, (const float *)lut_d.p, num_sms * fused_bps, st));
        if (profiling) S2_CUDA(cudaEventRecord(prof[2], st));
        S2_CUDA(launch_finalize(dpairs, n, (const double *)partials_d.p, (DevResult *)results_d.p, st));
        if (profiling) S2_CUDA(cudaEventRecord(prof[3], st));
        S2_CUDA(cudaMemcpyAsync(results_h, results_d.p, n * sizeof(DevResult), cudaMemcpyDeviceToHost, st));
        S2_CUDA(cudaEventRecord(done, st));
        last_n = n;
        pending = true;
        return S2_OK;
    }

    s2_status wait() {
        if (last_n < 0) return S2_ERR_NOT_READY;
        S2_CUDA(cudaEventSynchronize(done));
        pending = false;
        return S2_OK;
    }
};

// ---------------------------------------------------------------------------
// single-pair context
// ---------------------------------------------------------------------------
struct s2_ctx {
    Engine eng;
    uint32_t w = 0, h = 0;
    DevBuf stage[4];  // host-input staging: ref, dis (+ uv planes)
    bool has_ref = false;
    DevBuf ref_copy;  // cached reference input (packed, device)
    s2_pair_desc ref_desc;
    Plan plan;
};

struct s2_batch {
    Engine eng;
    uint32_t max_pairs = 0;
    uint64_t max_pixels = 0;
    Plan plan;
};

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

int s2_num_scales(uint32_t w, uint32_t h, int32_t rule) { return num_scales_rule(w, h, rule); }

static s2_status check_cfg(const s2_config *cfg) {
    if (!cfg || cfg->struct_size != sizeof(s2_config)) return S2_ERR_INVALID_ARG;
    if (cfg->blur != S2_BLUR_FIR && cfg->blur != S2_BLUR_IIR_REF) return S2_ERR_INVALID_ARG;
    if (cfg->storage < 0 || cfg->storage > 2) return S2_ERR_INVALID_ARG;
    if (cfg->scale_rule < 0 || cfg->scale_rule > 2) return S2_ERR_INVALID_ARG;
    if (cfg->strip_rows != 0 && cfg->strip_rows != 9 && cfg->strip_rows != 21 && cfg->strip_rows != 63)
        return S2_ERR_INVALID_ARG;
    return S2_OK;
}

s2_status s2_create(const s2_config *cfg_in, uint32_t width, uint32_t height, s2_ctx **out) {
    if (!out) return S2_ERR_INVALID_ARG;
    *out = nullptr;
    s2_config cfg;
    if (cfg_in) cfg = *cfg_in;
    else s2_config_default(&cfg);
    s2_status st = check_cfg(&cfg);
    if (st != S2_OK) return st;
    if (num_scales_rule(width, height, cfg.scale_rule) == 0 || width > 65536 || height > 65536)
        return S2_ERR_INVALID_SIZE;
    if (cfg.blur != S2_BLUR_FIR) {
        g_last_error = "S2_BLUR_IIR_REF is served by s2_iir_* entry points only";
        return S2_ERR_INVALID_ARG;
    }
    // pre-flight: levels (2 images, ~1/3 of scale 0) + partials + staging
    {
        size_t free_b = 0, total_b = 0;
        if (cudaSetDevice(cfg.device) != cudaSuccess) return cuda_fail(cudaGetLastError(), "cudaSetDevice");
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
    if (ctx->ref_copy.p) cudaFree(ctx->ref_copy.p);
    ctx->eng.release();
    delete ctx;
}

s2_status s2_mem_usage(const s2_ctx *ctx, size_t *bytes) {
    if (!ctx || !bytes) return S2_ERR_INVALID_ARG;
    size_t n = ctx->eng.allocated + ctx->ref_copy.n;
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

static s2_status ctx_run(s2_ctx *ctx, const s2_pair_desc &d, void *stream) {
    s2_status st = ctx->eng.plan(&d, 1, ctx->plan);
    if (st != S2_OK) return st;
    if (ctx->plan.pairs[0].status != S2_OK) return (s2_status)ctx->plan.pairs[0].status;
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

s2_status s2_compute_nv12(s2_ctx *ctx, const uint8_t *ref_y, const uint8_t *ref_uv, size_t ref_pitch,
                          const uint8_t *dis_y, const uint8_t *dis_uv, size_t dis_pitch, int32_t matrix,
                          int32_t range, int32_t on_host, void *stream) {
    if (!ctx || !ref_y || !ref_uv || !dis_y || !dis_uv) return S2_ERR_INVALID_ARG;
    if (matrix != S2_MATRIX_BT709 || range != S2_RANGE_LIMITED) return S2_ERR_INVALID_ARG;
    if ((ctx->w & 1) || (ctx->h & 1)) return S2_ERR_INVALID_SIZE;
    if (ref_pitch < ctx->w || dis_pitch < ctx->w) return S2_ERR_DIM_MISMATCH;
    const void *ry = ref_y, *ru = ref_uv, *dy = dis_y, *du = dis_uv;
    size_t rp = ref_pitch, dp = dis_pitch, tmp;
    if (on_host) {
        s2_status st = stage_host(ctx, 0, ref_y, ref_pitch, ctx->w, ctx->h, stream, &ry, &rp);
        if (st == S2_OK) st = stage_host(ctx, 1, dis_y, dis_pitch, ctx->w, ctx->h, stream, &dy, &dp);
        if (st == S2_OK) st = stage_host(ctx, 2, ref_uv, ref_pitch, ctx->w, ctx->h / 2, stream, &ru, &tmp);
        if (st == S2_OK) st = stage_host(ctx, 3, dis_uv, dis_pitch, ctx->w, ctx->h / 2, stream, &du, &tmp);
        if (st != S2_OK) return st;
    }
    s2_pair_desc d = make_desc(ctx->w, ctx->h, S2_FMT_NV12, ry, rp, dy, dp);
    d.ref_uv = ru;
    d.dis_uv = du;
    return ctx_run(ctx, d, stream);
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
// The context keeps a device copy of the reference input; candidates are
// scored against it without the caller re-supplying it.
static s2_status set_ref(s2_ctx *ctx, int fmt, const void *src, size_t pitch, size_t row, int32_t on_host,
                         void *stream) {
    DevBuf &b = ctx->ref_copy;
    size_t need = row * ctx->h;
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
    S2_CUDA(cudaMemcpy2DAsync(b.p, row, src, pitch, row, ctx->h,
                              on_host ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice, (cudaStream_t)stream));
    ctx->ref_desc = make_desc(ctx->w, ctx->h, fmt, b.p, row, nullptr, 0);
    ctx->has_ref = true;
    return S2_OK;
}

s2_status s2_set_reference_linear_f32(s2_ctx *ctx, const float *ref, size_t pitch, void *stream) {
    if (!ctx || !ref) return S2_ERR_INVALID_ARG;
    if (pitch < (size_t)ctx->w * 12) return S2_ERR_DIM_MISMATCH;
    return set_ref(ctx, S2_FMT_LINEAR_F32, ref, pitch, (size_t)ctx->w * 12, 0, stream);
}

s2_status s2_set_reference_srgb8(s2_ctx *ctx, const uint8_t *ref, size_t pitch, int32_t on_host, void *stream) {
    if (!ctx || !ref) return S2_ERR_INVALID_ARG;
    if (pitch < (size_t)ctx->w * 3) return S2_ERR_DIM_MISMATCH;
    return set_ref(ctx, S2_FMT_SRGB8, ref, pitch, (size_t)ctx->w * 3, on_host, stream);
}

s2_status s2_compute_with_reference_linear_f32(s2_ctx *ctx, const float *dis, size_t pitch, void *stream) {
    if (!ctx || !dis) return S2_ERR_INVALID_ARG;
    if (!ctx->has_ref) return S2_ERR_NO_REFERENCE;
    if (ctx->ref_desc.format != S2_FMT_LINEAR_F32) return S2_ERR_DIM_MISMATCH;
    if (pitch < (size_t)ctx->w * 12) return S2_ERR_DIM_MISMATCH;
    s2_pair_desc d = ctx->ref_desc;
    d.dis = dis;
    d.dis_pitch = pitch;
    return ctx_run(ctx, d, stream);
}

s2_status s2_compute_with_reference_srgb8(s2_ctx *ctx, const uint8_t *dis, size_t pitch, int32_t on_host,
                                          void *stream) {
    if (!ctx || !dis) return S2_ERR_INVALID_ARG;
    if (!ctx->has_ref) return S2_ERR_NO_REFERENCE;
    if (ctx->ref_desc.format != S2_FMT_SRGB8) return S2_ERR_DIM_MISMATCH;
    const size_t row = (size_t)ctx->w * 3;
    if (pitch < row) return S2_ERR_DIM_MISMATCH;
    const void *d = dis;
    size_t dp = pitch;
    if (on_host) {
        s2_status st = stage_host(ctx, 1, dis, pitch, row, ctx->h, stream, &d, &dp);
        if (st != S2_OK) return st;
    }
    s2_pair_desc desc = ctx->ref_desc;
    desc.dis = d;
    desc.dis_pitch = dp;
    return ctx_run(ctx, desc, stream);
}

s2_status s2_clear_reference(s2_ctx *ctx) {
    if (!ctx) return S2_ERR_INVALID_ARG;
    ctx->has_ref = false;
    return S2_OK;
}

int32_t s2_has_reference(const s2_ctx *ctx) { return ctx && ctx->has_ref ? 1 : 0; }

// ---- batches -----------------------------------------------------------
s2_status s2_batch_create(const s2_config *cfg_in, uint32_t max_pairs, uint64_t max_pixels, s2_batch **out) {
    if (!out || max_pairs == 0) return S2_ERR_INVALID_ARG;
    *out = nullptr;
    s2_config cfg;
    if (cfg_in) cfg = *cfg_in;
    else s2_config_default(&cfg);
    s2_status st = check_cfg(&cfg);
    if (st != S2_OK) return st;
    if (cfg.blur != S2_BLUR_FIR) return S2_ERR_INVALID_ARG;
    s2_batch *b = new (std::nothrow) s2_batch();
    if (!b) return S2_ERR_OOM;
    b->max_pairs = max_pairs;
    b->max_pixels = max_pixels;
    st = b->eng.init(&cfg);
    if (st == S2_OK) {
        // levels: < (1/3 + padding) of the scale-0 pixels, per image
        size_t lv = (size_t)(max_pixels * 3 * b->eng.esize() * 2) * 4 / 3 + (size_t)max_pairs * (1u << 20);
        st = b->eng.ensure(b->eng.levels_d, lv);
        if (st == S2_OK) st = b->eng.ensure(b->eng.results_d, (size_t)max_pairs * sizeof(DevResult));
    }
    if (st != S2_OK) {
        b->eng.release();
        delete b;
        return st;
    }
    *out = b;
    return S2_OK;
}

void s2_batch_destroy(s2_batch *b) {
    if (!b) return;
    b->eng.release();
    delete b;
}

s2_status s2_batch_submit(s2_batch *b, const s2_pair_desc *pairs, uint32_t n, void *stream) {
    if (!b || (!pairs && n)) return S2_ERR_INVALID_ARG;
    if (n > b->max_pairs) return S2_ERR_INVALID_ARG;
    s2_status st = b->eng.plan(pairs, (int)n, b->plan);
    if (st != S2_OK) return st;
    return b->eng.enqueue(b->plan, (cudaStream_t)stream);
}

s2_status s2_batch_results(s2_batch *b, s2_result *out, uint32_t n) {
    if (!b || (!out && n)) return S2_ERR_INVALID_ARG;
    s2_status st = b->eng.wait();
    if (st != S2_OK) return st;
    if ((int)n > b->eng.last_n) return S2_ERR_INVALID_ARG;
    for (uint32_t i = 0; i < n; i++) {
        const DevResult &r = b->eng.results_h[i];
        out[i].score = r.score;
        memcpy(out[i].stats, r.stats, sizeof r.stats);
        memcpy(out[i].sums, r.sums, sizeof r.sums);
        out[i].n_scales = r.n_scales;
        out[i].status = r.status;
    }
    return S2_OK;
}

s2_status s2_batch_mem_usage(const s2_batch *b, size_t *bytes) {
    if (!b || !bytes) return S2_ERR_INVALID_ARG;
    *bytes = b->eng.allocated;
    return S2_OK;
}

s2_status s2_batch_set_profiling(s2_batch *b, int32_t enable) {
    if (!b) return S2_ERR_INVALID_ARG;
    return b->eng.set_profiling(enable != 0);
}

s2_status s2_batch_last_timings(s2_batch *b, float ms[3]) {
    if (!b || !ms) return S2_ERR_INVALID_ARG;
    return b->eng.timings(ms);
}

s2_status s2_profile_enable(s2_ctx *ctx, int32_t enable) {
    if (!ctx) return S2_ERR_INVALID_ARG;
    return ctx->eng.set_profiling(enable != 0);
}

s2_status s2_profile_last(s2_ctx *ctx, float ms[3]) {
    if (!ctx || !ms) return S2_ERR_INVALID_ARG;
    return ctx->eng.timings(ms);
}

int32_t s2_fused_blocks_per_sm(int32_t storage) { return global_init() == S2_OK ? fused_blocks_per_sm(storage) : 0; }

s2_status s2_batch_set_graphs(s2_batch *b, int32_t enable) {
    if (!b) return S2_ERR_INVALID_ARG;
    (void)enable;
    return S2_OK;
}

}  // extern "C"
