// ssim2_engine_internal.h -- engine internals shared by the C-ABI units
// (ssim2_engine.cu, ssim2_server.cu): device buffers, submission plans and the
// Engine that lays pairs out into prep blocks and fused tiles and launches them.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/ssim2b200.h"
#include "ssim2_launch.h"

using namespace s2;

s2_status s2_cuda_fail(cudaError_t e, const char *what);
void s2_set_last_error(const char *msg);
s2_status s2_global_init();
ColorConsts s2_make_color_consts();
void s2_yuv_coeffs(int matrix, int range, int bits, float out[5], int *ymin, int *neutral);
extern const float s2_srgb8_lut[256];

// Tile-height autotuner cache (process-wide, thread-safe; ssim2_engine.cu).
// A workload class is the number of fused work items at the tallest strip,
// in half-octave buckets, with the storage type and the resident-CTA count.
uint64_t s2_tune_signature(uint64_t items63, int storage, int num_sms, int bps);
int s2_tuned_strip(uint64_t sig);  // 0 if not measured yet
void s2_set_tuned_strip(uint64_t sig, int strip);

#define S2_CUDA(call)                                          \
    do {                                                       \
        cudaError_t e_ = (call);                               \
        if (e_ != cudaSuccess) return s2_cuda_fail(e_, #call); \
    } while (0)

// ---------------------------------------------------------------------------
// device buffers
// ---------------------------------------------------------------------------
struct DevBuf {
    void *p = nullptr;
    size_t n = 0;
};

inline size_t s2_align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

inline int s2_num_scales_rule(uint32_t w, uint32_t h, int rule) {
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

// Per-pair options of a submission beyond s2_pair_desc: which images the
// prep pass converts, whether the pair is scored (tiles + result), and the
// reference's XYB planes when they were built earlier (a cached reference).
struct PairExtra {
    int prep_mask = 3;
    bool score = true;
    bool dssim = true;  // score DSSIM too when the engine's metrics include it
    void *ref_levels[kScales] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
};

// DSSIM level sizes (dssim-cuda/src/lib.rs:184-205): halved rounding up,
// never below 8.
inline void s2_dssim_dims(uint32_t w, uint32_t h, int dw[kDsLevels], int dh[kDsLevels]) {
    for (int s = 0; s < kDsLevels; s++) {
        dw[s] = (int)w;
        dh[s] = (int)h;
        w = std::max<uint32_t>((w + 1) / 2, 8);
        h = std::max<uint32_t>((h + 1) / 2, 8);
    }
}

// Host-side bytes of one image of a pair: its main plane (rows x row bytes)
// and, for NV12, the interleaved chroma plane (height / 2 rows of width bytes).
inline bool s2_is_yuv420(int format) { return format == S2_FMT_NV12 || format == S2_FMT_P016; }

inline size_t s2_row_bytes(const s2_pair_desc &q) {
    switch (q.format) {
    case S2_FMT_LINEAR_F32: return (size_t)q.width * 12;
    case S2_FMT_SRGB8: return (size_t)q.width * 3;
    case S2_FMT_NV12: return (size_t)q.width;
    case S2_FMT_P016: return (size_t)q.width * 2;
    default: return (size_t)q.width * 6;
    }
}

constexpr int kMaxGroups = 16;  // copy/compute groups of a host-input submission

// Byte layout of one image's XYB planes (all scored scales), as the plan lays
// them out: plane pitch rounded up to 64 elements, 256-byte aligned scales.
inline size_t s2_image_levels_layout(uint32_t w, uint32_t h, int ns, size_t esize, size_t off[kScales]) {
    size_t o = 0;
    uint64_t cw = w, ch = h;
    for (int s = 0; s < ns; s++) {
        off[s] = o;
        o += s2_align_up((size_t)3 * s2_align_up((size_t)cw, 64) * ch * esize, 256);
        cw = (cw + 1) / 2;
        ch = (ch + 1) / 2;
    }
    return o;
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
    // autotuning: the workload class of this plan, and whether the tile
    // height for it still has to be measured
    uint64_t tune_sig = 0;
    bool needs_tune = false;
    // groups: pairs [grp_pair[g], grp_pair[g+1]) own the tiles
    // [grp_tile[g], grp_tile[g+1]); one group unless the inputs are uploaded
    // from the host in pipelined groups
    std::vector<int> grp_pair, grp_tile;
    // S2_BLUR_IIR_REF: vertical / horizontal work runs, vertical output planes
    std::vector<IirSeg> vsegs, hsegs;
    int vtotal = 0, htotal = 0;
    size_t v_bytes = 0;
    // DSSIM (metrics include S2_METRIC_DSSIM): per-pair descriptors, tile
    // runs, and whether any pair needs the clamp pass
    int metrics = S2_METRIC_SSIMULACRA2;
    std::vector<DsPair> ds;
    std::vector<DsSeg> dsegs;
    int ds_tiles = 0;
    bool ds_clamp = false;

    // descriptor region: pairs | blk_first | segs | IIR vsegs | hsegs | DSSIM pairs | DSSIM segs
    struct Layout {
        size_t pb, bb, sb, vsb, hsb, dpb, dsb;
        size_t total() const { return pb + bb + sb + vsb + hsb + dpb + dsb; }
        size_t ds_pairs() const { return pb + bb + sb + vsb + hsb; }
        size_t ds_segs() const { return ds_pairs() + dpb; }
    };
    Layout layout() const {
        const size_t n = pairs.size();
        Layout L;
        L.pb = s2_align_up(n * sizeof(DevPair), 256);
        L.bb = s2_align_up(n * sizeof(int), 256);
        L.sb = s2_align_up(std::max<size_t>(segs.size(), 1) * sizeof(Seg), 256);
        L.vsb = s2_align_up(vsegs.size() * sizeof(IirSeg), 256);
        L.hsb = s2_align_up(hsegs.size() * sizeof(IirSeg), 256);
        const bool d = (metrics & S2_METRIC_DSSIM) != 0;
        L.dpb = d ? s2_align_up(n * sizeof(DsPair), 256) : 0;
        L.dsb = d ? s2_align_up(std::max<size_t>(dsegs.size(), 1) * sizeof(DsSeg), 256) : 0;
        return L;
    }
};

struct Engine {
    int device = 0;
    int storage = ST_F32;
    int scale_rule = S2_SCALES_CPU;
    int strip_rows_cfg = 0;
    int blur = S2_BLUR_FIR;
    int metrics = S2_METRIC_SSIMULACRA2;  // S2_METRIC_* bits scored by each submission
    uint64_t budget = 0;
    size_t allocated = 0;
    int num_sms = 148;
    int fused_bps = 1;
    ColorConsts cc;

    DevBuf pairs_d, blk_d, segs_d, counter_d, partials_d, results_d, levels_d, lut_d, iir_d;
    // counter_d: the tile groups' work counters (ints 0..), and at its last
    // int the tile pass's error word; all zeroed before every submission
    static constexpr size_t kCounterBytes = 256;
    int *err_word() const { return (int *)counter_d.p + kCounterBytes / sizeof(int) - 1; }
    DevBuf ds_d;  // DSSIM: per-tile SSIM sums, per-tile |avg - ssim| sums, per-level avg
    void *pinned = nullptr;  // staging: pairs | blk_first | segs
    size_t pinned_n = 0;
    DevResult *results_h = nullptr;
    size_t results_cap = 0;
    cudaEvent_t done = nullptr;
    int last_n = -1;
    bool pending = false;
    Plan plan_storage;  // a submission's plan, owned by whoever drives this engine
    bool profiling = false;
    // start, prep done, tile pass done, finalize done, DSSIM passes done
    cudaEvent_t prof[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    // host-input submissions: staging for the uploaded planes, the copy
    // stream and the prep stream (a group's prep runs beside the previous
    // group's tile launch, filling the SMs its last wave leaves idle), one
    // event per group for its planes having landed and one for its prep being
    // done, the submission's start, and the staging being free again (the
    // last group's prep has read it)
    // CUDA graphs of single-group device-input submissions, keyed by the
    // plan's shape (pair count, block / tile / segment counts); the buffers
    // the graph's nodes point at are fixed until a reallocation, which drops
    // every graph.  Captured on an engine-owned stream, launched on the
    // caller's.
    bool graphs = false;
    // Descriptor upload by a kernel reading the page-locked staging through
    // its device mapping instead of a copy-engine memcpy (the server: its copy
    // stream keeps the H2D engine busy with job images, and a small memcpy on
    // the compute stream would wait behind them).
    bool desc_kernel = false;
    void *pinned_dev = nullptr;  // device address of the pinned staging
    struct GraphEntry {
        uint64_t key[8];
        cudaGraphExec_t exec;
    };
    std::vector<GraphEntry> gcache;
    cudaStream_t cap_st = nullptr;
    DevBuf stage_d;
    cudaStream_t copy_st = nullptr, prep_st = nullptr;
    cudaEvent_t grp_copied[kMaxGroups] = {}, grp_prepped[kMaxGroups] = {};
    cudaEvent_t sub_start = nullptr, stage_free = nullptr;

    size_t esize() const { return storage == ST_F32 ? 4 : 2; }

    s2_status init(const s2_config *cfg) {
        s2_status st = s2_global_init();
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
        cc = s2_make_color_consts();
        S2_CUDA(cudaEventCreateWithFlags(&done, cudaEventDisableTiming));
        st = ensure(lut_d, sizeof s2_srgb8_lut);
        if (st != S2_OK) return st;
        S2_CUDA(cudaMemcpy(lut_d.p, s2_srgb8_lut, sizeof s2_srgb8_lut, cudaMemcpyHostToDevice));
        st = ensure(counter_d, kCounterBytes);
        return st;
    }

    s2_status set_profiling(bool on) {
        if (on && !prof[0])
            for (cudaEvent_t &e : prof) S2_CUDA(cudaEventCreate(&e));
        profiling = on;
        return S2_OK;
    }

    s2_status timings(float ms[3], float *ds_ms = nullptr) {
        if (!profiling || last_n < 0) return S2_ERR_NOT_READY;
        S2_CUDA(cudaEventSynchronize(prof[4]));
        for (int i = 0; i < 3; i++) S2_CUDA(cudaEventElapsedTime(&ms[i], prof[i], prof[i + 1]));
        if (ds_ms) S2_CUDA(cudaEventElapsedTime(ds_ms, prof[3], prof[4]));
        return S2_OK;
    }

    void release() {
        if (device >= 0) cudaSetDevice(device);
        if (done) cudaEventSynchronize(done);
        for (cudaEvent_t &e : prof)
            if (e) cudaEventDestroy(e), e = nullptr;
        drop_graphs();
        if (cap_st) cudaStreamDestroy(cap_st), cap_st = nullptr;
        if (copy_st) cudaStreamSynchronize(copy_st), cudaStreamDestroy(copy_st), copy_st = nullptr;
        if (prep_st) cudaStreamSynchronize(prep_st), cudaStreamDestroy(prep_st), prep_st = nullptr;
        for (cudaEvent_t &e : grp_copied)
            if (e) cudaEventDestroy(e), e = nullptr;
        for (cudaEvent_t &e : grp_prepped)
            if (e) cudaEventDestroy(e), e = nullptr;
        if (sub_start) cudaEventDestroy(sub_start), sub_start = nullptr;
        if (stage_free) cudaEventDestroy(stage_free), stage_free = nullptr;
        for (DevBuf *b : {&pairs_d, &blk_d, &segs_d, &counter_d, &partials_d, &results_d, &levels_d, &lut_d, &iir_d,
                          &stage_d, &ds_d})
            if (b->p) cudaFree(b->p), b->p = nullptr, b->n = 0;
        if (pinned) cudaFreeHost(pinned), pinned = nullptr;
        if (results_h) cudaFreeHost(results_h), results_h = nullptr;
        if (done) cudaEventDestroy(done), done = nullptr;
        allocated = 0;
    }

    void drop_graphs() {
        for (GraphEntry &g : gcache) cudaGraphExecDestroy(g.exec);
        gcache.clear();
    }

    // Grow-only device allocation, checked against the budget.
    s2_status ensure(DevBuf &b, size_t bytes) {
        if (b.n >= bytes) return S2_OK;
        drop_graphs();
        bytes = s2_align_up(bytes, 4096);
        if (budget && allocated - b.n + bytes > budget) {
            s2_set_last_error("allocation over the HBM budget");
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

    // Size every buffer for submissions of up to `pairs` pairs and `pixels`
    // scale-0 pixels, so that later submissions never reallocate (a cudaFree
    // synchronises the whole device, other streams' queued work included).
    s2_status reserve(size_t pairs, uint64_t pixels, bool one_image) {
        const size_t imgs = one_image ? 1 : 2;
        // XYB planes: 3 planes x esize x (4/3 of the pixels), plus row padding
        const size_t lv = imgs * (3 * esize() * (size_t)(pixels * 4 / 3) + pairs * (size_t(1) << 20));
        const size_t tiles = (size_t)(pixels * 3 / 2) / (kTileW * kStripMin) + pairs * 256;
        s2_status r;
        if ((r = ensure(levels_d, lv)) != S2_OK) return r;
        if ((r = ensure(partials_d, tiles * 18 * sizeof(double))) != S2_OK) return r;
        if ((r = ensure(results_d, pairs * sizeof(DevResult))) != S2_OK) return r;
        const size_t desc = s2_align_up(pairs * sizeof(DevPair), 256) + s2_align_up(pairs * sizeof(int), 256) +
                            s2_align_up(pairs * kScales * sizeof(Seg), 256);
        if ((r = ensure(pairs_d, desc)) != S2_OK) return r;
        return ensure_pinned(desc, pairs);
    }

    s2_status ensure_pinned(size_t bytes, size_t nres) {
        if (pinned_n < bytes || results_cap < nres) drop_graphs();
        if (pinned_n < bytes) {
            if (pinned) {
                if (done) cudaEventSynchronize(done);
                cudaFreeHost(pinned);
            }
            pinned = nullptr;
            bytes = s2_align_up(bytes, 4096);
            S2_CUDA(cudaHostAlloc(&pinned, bytes, cudaHostAllocMapped));
            S2_CUDA(cudaHostGetDevicePointer(&pinned_dev, pinned, 0));
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

    int force_strip = 0;  // a tuning trial's tile height (0 = none)

    // The fused pass's tile height (rows per strip): configured (16/32/64), a
    // tuning trial's, the autotuner's measured choice for this workload class,
    // or, until that is measured, the largest height that still gives ~4
    // waves of resident work items (three per tile: one per channel).
    int choose_strip_rows(const std::vector<uint64_t> &tiles_at, Plan &P) const {
        P.needs_tune = false;
        if (force_strip) return force_strip;
        if (tiles_at[0] == 0) return kStripMax;  // no tile pass (DSSIM only, or no valid pair)
        if (strip_rows_cfg == kStripMin || strip_rows_cfg == kStripMid || strip_rows_cfg == kStripMax)
            return strip_rows_cfg;
        const uint64_t resident = (uint64_t)num_sms * (uint64_t)fused_bps;
        if (blur == S2_BLUR_FIR) {
            P.tune_sig = s2_tune_signature(3 * tiles_at[0], storage, num_sms, fused_bps);
            const int tuned = s2_tuned_strip(P.tune_sig);
            if (tuned) return tuned;
            P.needs_tune = true;
        }
        if (3 * tiles_at[0] >= 4 * resident) return kStripMax;
        if (3 * tiles_at[1] >= 4 * resident) return kStripMid;
        return kStripMin;
    }

    // DSSIM layout of one valid pair (offsets into levels_d, rebased at
    // upload): Lab planes and SSIM map of each of the five levels; levels
    // whose DSSIM size equals the pyramid's ceil-halved size are written by
    // the prep pass, later ones (clamped to 8) by the clamp pass from the
    // kept linear RGB of the last equal level.
    static size_t plan_dssim(const s2_pair_desc &q, DevPair &p, DsPair &D, size_t off, const PairExtra *ex,
                             bool &clamp) {
        memset(&D, 0, sizeof D);
        D.prep_mask = p.prep_mask;
        D.clamp_from = kDsLevels;
        if (ex && (!ex->dssim || !ex->score)) {  // not scored by this submission
            D.status = -1;
            p.lab_levels = 0;
            p.prep_levels = p.nscales;
            return off;
        }
        int dw[kDsLevels], dh[kDsLevels];
        s2_dssim_dims(q.width, q.height, dw, dh);
        int ll = 0;
        while (ll < kDsLevels && dw[ll] == p.w[ll] && dh[ll] == p.h[ll]) ll++;
        p.lab_levels = ll;
        p.prep_levels = std::max(p.nscales, ll);
        for (int s = 0; s < p.prep_levels; s++) p.lp[s] = (int)s2_align_up((size_t)p.w[s], 64);
        for (int s = 0; s < kDsLevels; s++) {
            D.w[s] = dw[s];
            D.h[s] = dh[s];
            D.pitch[s] = (int)s2_align_up((size_t)dw[s], 64);
            const size_t plane = (size_t)D.pitch[s] * dh[s] * sizeof(float);
            for (int img = 0; img < 2; img++) {
                D.lab[img][s] = (float *)off;
                if (s < ll) p.lab[img][s] = D.lab[img][s];
                off += s2_align_up(3 * plane, 256);
            }
            D.map[s] = (float *)off;
            off += s2_align_up(plane, 256);
        }
        D.clamp_from = ll;
        if (ll < kDsLevels) {
            clamp = true;
            const int k = ll - 1;
            D.kw = p.w[k];
            D.kh = p.h[k];
            D.kpitch = p.lp[k];
            long long sp = 0;
            for (int s = ll; s < kDsLevels; s++) sp = std::max<long long>(sp, (long long)D.pitch[s] * dh[s]);
            D.splane = sp;
            for (int img = 0; img < 2; img++) {
                p.keep[img] = D.keep[img] = (float *)off;
                off += s2_align_up((size_t)3 * D.kpitch * D.kh * sizeof(float), 256);
                D.scratch[img] = (float *)off;
                off += s2_align_up((size_t)6 * sp * sizeof(float), 256);
            }
        }
        return off;
    }

    // Lay out the levels and tiles of n pairs.
    s2_status plan(const s2_pair_desc *d, int n, Plan &P, const PairExtra *ex = nullptr, int ngroups = 1) {
        P = Plan();
        P.metrics = metrics;
        const bool m_s2 = (metrics & S2_METRIC_SSIMULACRA2) != 0, m_ds = (metrics & S2_METRIC_DSSIM) != 0;
        P.pairs.resize(n);
        P.blk_first.resize(n);
        if (m_ds) P.ds.assign(n, DsPair());
        // tile counts at the two tallest strip heights for the strip choice
        std::vector<uint64_t> tiles_at(2, 0);
        std::vector<int> ns(n);
        for (int i = 0; i < n; i++) {
            ns[i] = m_s2 ? s2_num_scales_rule(d[i].width, d[i].height, scale_rule) : 0;
            uint64_t w = d[i].width, h = d[i].height;
            for (int s = 0; s < ns[i]; s++) {
                tiles_at[0] += ((w + kTileW - 1) / kTileW) * ((h + kStripMax - 1) / kStripMax);
                tiles_at[1] += ((w + kTileW - 1) / kTileW) * ((h + kStripMid - 1) / kStripMid);
                w = (w + 1) / 2;
                h = (h + 1) / 2;
            }
        }
        P.strip_rows = choose_strip_rows(tiles_at, P);
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
            p.prep_mask = ex ? ex[i].prep_mask : 3;
            const bool need_ref_in = (p.prep_mask & 1) != 0;
            const bool need_dis_in = (p.prep_mask & 2) != 0;
            if ((m_s2 && ns[i] == 0) || (m_ds && (q.width < 8 || q.height < 8)) || q.width > (1u << 16) ||
                q.height > (1u << 16)) {
                p.status = S2_ERR_INVALID_SIZE;
                p.nscales = 0;
                P.blk_first[i] = blk;
                continue;
            }
            const bool yuv = q.format == S2_FMT_NV12 || q.format == S2_FMT_P016;
            if (q.format < 0 || q.format > 4 || (need_ref_in && !q.ref) || (need_dis_in && !q.dis) ||
                (yuv && ((need_ref_in && !q.ref_uv) || (need_dis_in && !q.dis_uv) || (q.width & 1) ||
                         (q.height & 1) || q.matrix < S2_MATRIX_BT709 || q.matrix > S2_MATRIX_BT601_625 ||
                         (q.range != S2_RANGE_LIMITED && q.range != S2_RANGE_FULL))) ||
                (q.format == S2_FMT_RGB16 && (q.bits < 8 || q.bits > 16))) {
                p.status = S2_ERR_INVALID_ARG;
                p.nscales = 0;
                P.blk_first[i] = blk;
                continue;
            }
            if (yuv) s2_yuv_coeffs(q.matrix, q.range, q.format == S2_FMT_P016 ? 16 : 8, p.yuv, &p.yuv_min, &p.yuv_neutral);
            p.w[0] = (int)q.width;
            p.h[0] = (int)q.height;
            for (int s = 1; s < kScales; s++) {
                p.w[s] = (p.w[s - 1] + 1) / 2;
                p.h[s] = (p.h[s - 1] + 1) / 2;
            }
            const bool ref_ext = ex && ex[i].ref_levels[0] != nullptr;
            p.lvl_ext = ref_ext ? 1 : 0;
            for (int s = 0; s < p.nscales; s++) {
                p.lp[s] = (int)s2_align_up((size_t)p.w[s], 64);
                size_t bytes = s2_align_up((size_t)3 * p.lp[s] * p.h[s] * esize(), 256);
                if (ref_ext) {
                    p.lvl[0][s] = ex[i].ref_levels[s];
                } else {
                    p.lvl[0][s] = (void *)lvl_off;  // offsets, rebased at upload
                    lvl_off += bytes;
                }
                p.lvl[1][s] = (void *)lvl_off;
                lvl_off += bytes;
            }
            if (m_ds) lvl_off = plan_dssim(q, p, P.ds[i], lvl_off, ex ? &ex[i] : nullptr, P.ds_clamp);
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
        if (m_ds) {
            for (int i = 0; i < n; i++)
                if (P.pairs[i].status != S2_OK) P.ds[i].status = P.pairs[i].status;
            // DSSIM tiles: all pairs' level 0 first, then level 1, ...
            int dt = 0;
            for (int s = 0; s < kDsLevels; s++)
                for (int i = 0; i < n; i++) {
                    DsPair &D = P.ds[i];
                    if (D.status != 0) continue;
                    DsSeg sg;
                    sg.first_tile = dt;
                    sg.pair = i;
                    sg.level = s;
                    sg.tiles_x = (D.w[s] + 31) / 32;
                    D.tile_base[s] = dt;
                    D.tile_cnt[s] = sg.tiles_x * ((D.h[s] + 31) / 32);
                    dt += D.tile_cnt[s];
                    P.dsegs.push_back(sg);
                }
            P.ds_tiles = dt;
        }
        if (blur == S2_BLUR_IIR_REF) {
            P.grp_pair = {0, n};
            P.grp_tile = {0, 0};
            // one partial-sum record per row; vertical work items per column
            // (groups of 32) and plane, horizontal per row and channel
            int rec = 0;
            for (int i = 0; i < n; i++) {
                DevPair &p = P.pairs[i];
                if (p.status != S2_OK || (ex && !ex[i].score)) continue;
                for (int s = 0; s < p.nscales; s++) {
                    const size_t vb = s2_align_up((size_t)15 * p.lp[s] * p.h[s] * sizeof(float), 256);
                    IirSeg v;
                    v.first = P.vtotal;
                    v.pair = i;
                    v.scale = s;
                    v.rec_base = rec;
                    v.v = (float *)P.v_bytes;  // offset, rebased at upload
                    P.vsegs.push_back(v);
                    P.vtotal += ((p.w[s] + 31) / 32) * 32 * 15;
                    IirSeg h = v;
                    h.first = P.htotal;
                    P.hsegs.push_back(h);
                    P.htotal += 3 * p.h[s];
                    p.tile_base[s] = rec;
                    p.tile_cnt[s] = p.h[s];
                    rec += p.h[s];
                    P.v_bytes += vb;
                }
            }
            P.total_tiles = rec;
            return S2_OK;
        }
        int tile = 0;
        // groups of contiguous pairs, about equal scale-0 pixels except the
        // first, which gets half a share (its upload is the one that nothing
        // overlaps): group g ends where the running pixel count reaches
        // (g + 1/2) / (ngroups - 1/2) of the total
        P.grp_pair.assign(1, 0);
        if (ngroups > 1) {
            uint64_t total = 0, acc = 0;
            for (int i = 0; i < n; i++) total += (uint64_t)P.pairs[i].w[0] * P.pairs[i].h[0];
            for (int i = 0; i + 1 < n && (int)P.grp_pair.size() < ngroups; i++) {
                acc += (uint64_t)P.pairs[i].w[0] * P.pairs[i].h[0];
                if (acc * (2 * ngroups - 1) >= total * (2 * P.grp_pair.size() - 1)) P.grp_pair.push_back(i + 1);
            }
        }
        P.grp_pair.push_back(n);
        // tiles, per group: all its pairs' scale 0 first, then scale 1, ...
        // (largest work first)
        P.grp_tile.assign(1, tile);
        for (size_t g = 0; g + 1 < P.grp_pair.size(); g++) {
          for (int s = 0; s < kScales; s++) {
            for (int i = P.grp_pair[g]; i < P.grp_pair[g + 1]; i++) {
                DevPair &p = P.pairs[i];
                if (p.status != S2_OK || s >= p.nscales || (ex && !ex[i].score)) continue;
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
          P.grp_tile.push_back(tile);
        }
        P.total_tiles = tile;
        return S2_OK;
    }

    // Staging offsets of host-input planes: the images the prep pass reads,
    // packed rows, 256-byte aligned planes.  Rewrites the pairs' input
    // pointers to offsets into stage_d (rebased at upload) and returns the
    // bytes needed.
    static size_t plan_staging(Plan &P, const s2_pair_desc *d) {
        size_t off = 0;
        for (size_t i = 0; i < P.pairs.size(); i++) {
            DevPair &p = P.pairs[i];
            if (p.status != S2_OK) continue;
            const size_t row = s2_row_bytes(d[i]);
            for (int img = 0; img < 2; img++) {
                if (!((p.prep_mask >> img) & 1)) continue;
                p.in[img] = (const void *)off;
                p.pitch[img] = (long long)row;
                off += s2_align_up(row * d[i].height, 256);
                if (s2_is_yuv420(d[i].format)) {
                    p.in_uv[img] = (const void *)off;
                    off += s2_align_up(row * (d[i].height / 2), 256);
                }
            }
        }
        return off;
    }

    s2_status copy_plane(void *dst, const void *src, size_t pitch, size_t row, size_t rows) {
        if (pitch == row) S2_CUDA(cudaMemcpyAsync(dst, src, row * rows, cudaMemcpyHostToDevice, copy_st));
        else S2_CUDA(cudaMemcpy2DAsync(dst, row, src, pitch, row, rows, cudaMemcpyHostToDevice, copy_st));
        return S2_OK;
    }

    // The input format of every pair of a plan, or -1 when they differ: the
    // prep launch then runs a kernel compiled for that one format.
    static int uniform_fmt(const Plan &P) {
        if (P.pairs.empty()) return -1;
        const int f = P.pairs[0].fmt;
        for (const DevPair &q : P.pairs)
            if (q.fmt != f) return -1;
        return f;
    }

    // Enqueue a planned submission on `st`.  With `host` (the submission's
    // descriptors, planes in host memory), the planes are uploaded group by
    // group on the copy stream and each group's prep + fused launches wait
    // only for their own group's planes, so uploads overlap the compute of
    // the groups before them.
    s2_status enqueue(Plan &P, cudaStream_t st, const s2_pair_desc *host = nullptr) {
        const int n = (int)P.pairs.size();
        const int ng = (int)P.grp_pair.size() - 1;
        if (ng < 1 || ng > kMaxGroups) return S2_ERR_INVALID_ARG;
        s2_status r;
        if ((r = ensure(levels_d, std::max<size_t>(P.level_bytes, 256))) != S2_OK) return r;
        if ((r = ensure(partials_d, std::max<size_t>((size_t)P.total_tiles * 18 * sizeof(double), 256))) != S2_OK) return r;
        if ((r = ensure(results_d, (size_t)n * sizeof(DevResult))) != S2_OK) return r;
        const Plan::Layout L = P.layout();
        const size_t pb = L.pb, bb = L.bb, sb = L.sb, vsb = L.vsb;
        const bool m_s2 = (P.metrics & S2_METRIC_SSIMULACRA2) != 0, m_ds = (P.metrics & S2_METRIC_DSSIM) != 0;
        if (blur == S2_BLUR_IIR_REF && (r = ensure(iir_d, std::max<size_t>(P.v_bytes, 256))) != S2_OK) return r;
        if (m_ds && (r = ensure(ds_d, ds_bytes(P))) != S2_OK) return r;
        if ((r = ensure(pairs_d, L.total())) != S2_OK) return r;
        if ((r = ensure_pinned(L.total(), n)) != S2_OK) return r;
        if (host) {
            if ((r = ensure(stage_d, std::max<size_t>(plan_staging(P, host), 256))) != S2_OK) return r;
            if (!copy_st) {
                S2_CUDA(cudaStreamCreateWithFlags(&copy_st, cudaStreamNonBlocking));
                S2_CUDA(cudaStreamCreateWithFlags(&prep_st, cudaStreamNonBlocking));
                for (cudaEvent_t &e : grp_copied) S2_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
                for (cudaEvent_t &e : grp_prepped) S2_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
                S2_CUDA(cudaEventCreateWithFlags(&sub_start, cudaEventDisableTiming));
                S2_CUDA(cudaEventCreateWithFlags(&stage_free, cudaEventDisableTiming));
                S2_CUDA(cudaEventRecord(stage_free, st));
            }
        }
        // the previous submission may still read the pinned staging
        if (pending) S2_CUDA(cudaEventSynchronize(done));
        char *h = (char *)pinned;
        DevPair *hp = (DevPair *)h;
        char *const lb = (char *)levels_d.p;
        for (int i = 0; i < n; i++) {
            hp[i] = P.pairs[i];
            for (int s = 0; s < kScales; s++)
                for (int img = 0; img < 2; img++)
                    if (s >= hp[i].nscales) hp[i].lvl[img][s] = nullptr;
                    else if (!((hp[i].lvl_ext >> img) & 1))
                        hp[i].lvl[img][s] = (char *)levels_d.p + (size_t)hp[i].lvl[img][s];
            if (m_ds && hp[i].status == S2_OK) {
                for (int img = 0; img < 2; img++) {
                    for (int s = 0; s < kDsLevels; s++)
                        hp[i].lab[img][s] = s < hp[i].lab_levels ? (float *)(lb + (size_t)hp[i].lab[img][s]) : nullptr;
                    hp[i].keep[img] = hp[i].lab_levels > 0 && hp[i].lab_levels < kDsLevels
                                          ? (float *)(lb + (size_t)hp[i].keep[img])
                                          : nullptr;
                }
            }
            if (host && hp[i].status == S2_OK)
                for (int img = 0; img < 2; img++)
                    if ((hp[i].prep_mask >> img) & 1) {
                        hp[i].in[img] = (const char *)stage_d.p + (size_t)hp[i].in[img];
                        if (s2_is_yuv420(host[i].format))
                            hp[i].in_uv[img] = (const char *)stage_d.p + (size_t)hp[i].in_uv[img];
                    }
        }
        memcpy(h + pb, P.blk_first.data(), n * sizeof(int));
        if (!P.segs.empty()) memcpy(h + pb + bb, P.segs.data(), P.segs.size() * sizeof(Seg));
        {
            IirSeg *hv = (IirSeg *)(h + pb + bb + sb), *hh = (IirSeg *)(h + pb + bb + sb + vsb);
            for (size_t k = 0; k < P.vsegs.size(); k++) {
                hv[k] = P.vsegs[k];
                hv[k].v = (float *)((char *)iir_d.p + (size_t)P.vsegs[k].v);
            }
            for (size_t k = 0; k < P.hsegs.size(); k++) {
                hh[k] = P.hsegs[k];
                hh[k].v = (float *)((char *)iir_d.p + (size_t)P.hsegs[k].v);
            }
        }
        if (m_ds) {
            DsPair *hd = (DsPair *)(h + L.ds_pairs());
            for (int i = 0; i < n; i++) {
                hd[i] = P.ds[i];
                if (hd[i].status != 0) continue;
                for (int s = 0; s < kDsLevels; s++) {
                    for (int img = 0; img < 2; img++) hd[i].lab[img][s] = (float *)(lb + (size_t)hd[i].lab[img][s]);
                    hd[i].map[s] = (float *)(lb + (size_t)hd[i].map[s]);
                }
                for (int img = 0; img < 2; img++)
                    if (hd[i].clamp_from < kDsLevels) {
                        hd[i].keep[img] = (float *)(lb + (size_t)hd[i].keep[img]);
                        hd[i].scratch[img] = (float *)(lb + (size_t)hd[i].scratch[img]);
                    }
            }
            if (!P.dsegs.empty()) memcpy(h + L.ds_segs(), P.dsegs.data(), P.dsegs.size() * sizeof(DsSeg));
        }
        char *dbase = (char *)pairs_d.p;
        const DevPair *dpairs = (const DevPair *)dbase;
        const int *dblk = (const int *)(dbase + pb);
        const Seg *dsegs = (const Seg *)(dbase + pb + bb);
        const int pout = (m_s2 ? 1 : 0) | (m_ds ? 2 : 0);
        if (graphs && !host && !profiling && ng == 1) {
            const uint64_t key[8] = {(uint64_t)n | ((uint64_t)(uniform_fmt(P) + 1) << 40), (uint64_t)P.total_blocks,
                                     (uint64_t)P.total_tiles,
                                     P.segs.size(),
                                     P.vsegs.size(), P.hsegs.size(),
                                     ((uint64_t)(uint32_t)P.vtotal << 32) | (uint32_t)P.htotal,
                                     ((uint64_t)(uint32_t)P.ds_tiles << 32) | ((uint64_t)P.dsegs.size() << 3) |
                                         ((uint64_t)P.ds_clamp << 2) | (uint64_t)P.metrics};
            cudaGraphExec_t ex = nullptr;
            for (const GraphEntry &g : gcache)
                if (!memcmp(g.key, key, sizeof key)) ex = g.exec;
            if (!ex) ex = capture(P, key, L.total());
            if (ex) {
                S2_CUDA(cudaGraphLaunch(ex, st));
                S2_CUDA(cudaEventRecord(done, st));
                last_n = n;
                pending = true;
                return S2_OK;
            }
        }
        // Host submissions: the copy stream first waits until the previous
        // host submission's prep has read the staging, then uploads the
        // descriptors ahead of the planes, so preps (on the prep stream)
        // depend on copies only and may run beside another submission's tile
        // pass; the tile passes and finalize stay in order on `st`.
        const bool split = host && blur != S2_BLUR_IIR_REF;
        if (host) S2_CUDA(cudaStreamWaitEvent(copy_st, stage_free, 0));
        if (desc_kernel && !split)
            S2_CUDA(launch_desc_copy(dbase, pinned_dev, L.total(), st));
        else
            S2_CUDA(cudaMemcpyAsync(dbase, h, L.total(), cudaMemcpyHostToDevice, split ? copy_st : st));
        if (split) {
            S2_CUDA(cudaEventRecord(sub_start, copy_st));
            S2_CUDA(cudaStreamWaitEvent(st, sub_start, 0));
        }
        S2_CUDA(cudaMemsetAsync(counter_d.p, 0, kCounterBytes, st));
        if (profiling) S2_CUDA(cudaEventRecord(prof[0], st));
        cudaStream_t pst = split ? prep_st : st;
        for (int g = 0; g < ng; g++) {
            const int pa = P.grp_pair[g], pe = P.grp_pair[g + 1];
            if (host) {
                for (int i = pa; i < pe; i++) {
                    const DevPair &q = hp[i];
                    if (q.status != S2_OK) continue;
                    const size_t row = s2_row_bytes(host[i]);
                    const size_t hgt = host[i].height;
                    for (int img = 0; img < 2; img++) {
                        if (!((q.prep_mask >> img) & 1)) continue;
                        const void *src = img ? host[i].dis : host[i].ref;
                        const size_t sp = img ? host[i].dis_pitch : host[i].ref_pitch;
                        if ((r = copy_plane((void *)q.in[img], src, sp, row, hgt)) != S2_OK) return r;
                        if (s2_is_yuv420(host[i].format) &&
                            (r = copy_plane((void *)q.in_uv[img], img ? host[i].dis_uv : host[i].ref_uv, sp, row,
                                            hgt / 2)) != S2_OK)
                            return r;
                    }
                }
                S2_CUDA(cudaEventRecord(grp_copied[g], copy_st));
                S2_CUDA(cudaStreamWaitEvent(pst, grp_copied[g], 0));
            }
            const int b0 = pa < n ? P.blk_first[pa] : P.total_blocks;
            const int b1 = pe < n ? P.blk_first[pe] : P.total_blocks;
            S2_CUDA(launch_pyramid(storage, dpairs, n, dblk, b0, b1, cc, (const float *)lut_d.p, num_sms * 8, pst,
                                   pout, uniform_fmt(P)));
            if (host && g + 1 == ng) S2_CUDA(cudaEventRecord(stage_free, pst));
            if (split) {
                S2_CUDA(cudaEventRecord(grp_prepped[g], prep_st));
                S2_CUDA(cudaStreamWaitEvent(st, grp_prepped[g], 0));
            }
            if (profiling && ng == 1) S2_CUDA(cudaEventRecord(prof[1], st));
            if (!m_s2) continue;
            if (blur == S2_BLUR_IIR_REF)
                S2_CUDA(launch_iir(storage, dpairs, (const IirSeg *)(dbase + pb + bb + sb), (int)P.vsegs.size(),
                                   P.vtotal, (const IirSeg *)(dbase + pb + bb + sb + vsb), (int)P.hsegs.size(),
                                   P.htotal, (double *)partials_d.p, st));
            else
                S2_CUDA(launch_fused(storage, dpairs, dsegs, (int)P.segs.size(), P.grp_tile[g], P.grp_tile[g + 1],
                                     (int *)counter_d.p + g, tile_check(err_word()), (double *)partials_d.p, num_sms * fused_bps,
                                     st));
        }
        // several groups interleave prep and fused: the fused slot then holds both
        if (profiling && ng > 1) S2_CUDA(cudaEventRecord(prof[1], st));
        if (profiling) S2_CUDA(cudaEventRecord(prof[2], st));
        if (m_s2)
            S2_CUDA(launch_finalize(dpairs, n, (const double *)partials_d.p, err_word(), (DevResult *)results_d.p, st));
        if (profiling) S2_CUDA(cudaEventRecord(prof[3], st));
        if (m_ds) S2_CUDA(launch_ds(P, dbase, st));
        if (profiling) S2_CUDA(cudaEventRecord(prof[4], st));
        S2_CUDA(cudaMemcpyAsync(results_h, results_d.p, n * sizeof(DevResult), cudaMemcpyDeviceToHost, st));
        S2_CUDA(cudaEventRecord(done, st));
        last_n = n;
        pending = true;
        return S2_OK;
    }

    // DSSIM workspace: two f64 sums per tile, one f32 avg per (pair, level).
    static size_t ds_bytes(const Plan &P) {
        return s2_align_up((size_t)2 * std::max(P.ds_tiles, 1) * sizeof(double), 256) +
               P.pairs.size() * kDsLevels * sizeof(float);
    }

    cudaError_t launch_ds(const Plan &P, char *dbase, cudaStream_t st) {
        const Plan::Layout L = P.layout();
        const int n = (int)P.pairs.size();
        double *part = (double *)ds_d.p;
        float *avg = (float *)((char *)ds_d.p + s2_align_up((size_t)2 * std::max(P.ds_tiles, 1) * sizeof(double), 256));
        return launch_dssim((const DsPair *)(dbase + L.ds_pairs()), n, (const DsSeg *)(dbase + L.ds_segs()),
                            (int)P.dsegs.size(), P.ds_tiles, P.ds_clamp, part, avg, (DevResult *)results_d.p,
                            (P.metrics & S2_METRIC_SSIMULACRA2) == 0, num_sms, st);
    }

    // Record a single-group device-input submission of plan P (its
    // descriptors already in the pinned staging) as a graph: descriptor
    // upload, counter reset, prep, fused (or the two IIR passes), finalize,
    // result download.  nullptr if capture is not possible here (graphs are
    // then switched off for this engine and the launches go directly).
    cudaGraphExec_t capture(const Plan &P, const uint64_t key[8], size_t desc_bytes) {
        const int n = (int)P.pairs.size();
        const Plan::Layout L = P.layout();
        const size_t pb = L.pb, bb = L.bb, sb = L.sb, vsb = L.vsb;
        const bool m_s2 = (P.metrics & S2_METRIC_SSIMULACRA2) != 0, m_ds = (P.metrics & S2_METRIC_DSSIM) != 0;
        char *dbase = (char *)pairs_d.p;
        const DevPair *dpairs = (const DevPair *)dbase;
        if (!cap_st && cudaStreamCreateWithFlags(&cap_st, cudaStreamNonBlocking) != cudaSuccess) {
            graphs = false;
            return nullptr;
        }
        if (cudaStreamBeginCapture(cap_st, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
            graphs = false;
            return nullptr;
        }
        cudaError_t e = desc_kernel ? launch_desc_copy(dbase, pinned_dev, desc_bytes, cap_st)
                                    : cudaMemcpyAsync(dbase, pinned, desc_bytes, cudaMemcpyHostToDevice, cap_st);
        if (e == cudaSuccess) e = cudaMemsetAsync(counter_d.p, 0, kCounterBytes, cap_st);
        if (e == cudaSuccess)
            e = launch_pyramid(storage, dpairs, n, (const int *)(dbase + pb), 0, P.total_blocks, cc,
                               (const float *)lut_d.p, num_sms * 8, cap_st, (m_s2 ? 1 : 0) | (m_ds ? 2 : 0),
                               uniform_fmt(P));
        if (e == cudaSuccess && m_s2) {
            if (blur == S2_BLUR_IIR_REF)
                e = launch_iir(storage, dpairs, (const IirSeg *)(dbase + pb + bb + sb), (int)P.vsegs.size(), P.vtotal,
                               (const IirSeg *)(dbase + pb + bb + sb + vsb), (int)P.hsegs.size(), P.htotal,
                               (double *)partials_d.p, cap_st);
            else
                e = launch_fused(storage, dpairs, (const Seg *)(dbase + pb + bb), (int)P.segs.size(), 0,
                                 P.total_tiles, (int *)counter_d.p, tile_check(err_word()), (double *)partials_d.p,
                                 num_sms * fused_bps, cap_st);
        }
        if (e == cudaSuccess && m_s2)
            e = launch_finalize(dpairs, n, (const double *)partials_d.p, err_word(), (DevResult *)results_d.p, cap_st);
        if (e == cudaSuccess && m_ds) e = launch_ds(P, dbase, cap_st);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(results_h, results_d.p, n * sizeof(DevResult), cudaMemcpyDeviceToHost, cap_st);
        cudaGraph_t graph = nullptr;
        const cudaError_t ee = cudaStreamEndCapture(cap_st, &graph);
        cudaGraphExec_t exec = nullptr;
        if (e == cudaSuccess && ee == cudaSuccess && graph &&
            cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess) {
            if (gcache.size() >= 8) {
                cudaGraphExecDestroy(gcache.front().exec);
                gcache.erase(gcache.begin());
            }
            GraphEntry g;
            memcpy(g.key, key, sizeof g.key);
            g.exec = exec;
            gcache.push_back(g);
        } else {
            graphs = false;
            exec = nullptr;
            cudaGetLastError();  // clear a capture error; the direct path follows
        }
        if (graph) cudaGraphDestroy(graph);
        return exec;
    }

    s2_status wait() {
        if (last_n < 0) return S2_ERR_NOT_READY;
        S2_CUDA(cudaEventSynchronize(done));
        pending = false;
        return S2_OK;
    }

    // The autotuner: the first submission of a workload class runs once per
    // candidate tile height (16, 32, 64 rows) with the fused launch timed by
    // CUDA events, records the fastest for the class, and re-plans P with it.
    // The trials score the same pairs, so they need no inputs of their own;
    // later submissions of the class use the recorded height directly.
    s2_status tune(const s2_pair_desc *d, int n, Plan &P, const PairExtra *ex, cudaStream_t st) {
        if (!P.needs_tune) return S2_OK;
        const bool prof_was = profiling;
        s2_status r = set_profiling(true);
        if (r != S2_OK) return r;
        static const int cand[3] = {kStripMin, kStripMid, kStripMax};
        float best_ms = 0.0f;
        int best = 0;
        Plan T;
        for (int c : cand) {
            force_strip = c;
            r = plan(d, n, T, ex);
            if (r == S2_OK) r = enqueue(T, st);
            if (r == S2_OK) r = wait();
            float ms[3] = {0, 0, 0};
            if (r == S2_OK) r = timings(ms);
            if (r != S2_OK) break;
            if (!best || ms[1] < best_ms) best_ms = ms[1], best = c;
        }
        force_strip = 0;
        profiling = prof_was;
        if (r != S2_OK) return r;
        s2_set_tuned_strip(P.tune_sig, best);
        return plan(d, n, P, ex);
    }
};
