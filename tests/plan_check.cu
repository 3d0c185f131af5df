// plan_check.cu -- host-only check of the submission planner (Engine::plan in
// turbo-metrics_b200/csrc/ssim2_engine_internal.h) over random submissions:
// every device region a plan lays out (XYB levels, DSSIM Lab planes, SSIM
// maps, kept linear levels, clamp-pass scratch) lies inside the plan's level
// bytes, starts 256-byte aligned and overlaps no other; DSSIM level sizes
// follow dssim-cuda (halved rounding up, never below 8); the levels the prep
// pass converts and the clamp pass builds split where those sizes leave the
// ceil-halved pyramid; DSSIM tiles cover every level of every pair once;
// the copy/compute groups of host-input submissions split pairs and tiles
// contiguously; the staging of host planes is packed, aligned and disjoint;
// the reference-IIR mode's row records and vertical-walk planes are packed.
// plan() makes no CUDA call, so this runs without a GPU (built and run by
// tests/test_cpu_plan.py).
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <random>
#include <vector>

#include "../turbo-metrics_b200/csrc/ssim2_engine_internal.h"

static int fails = 0;
#define CHECK(c, ...)                              \
    do {                                           \
        if (!(c)) {                                \
            if (fails++ < 20) {                    \
                printf("FAIL %s:%d: ", __FILE__, __LINE__); \
                printf(__VA_ARGS__);               \
                printf("\n");                      \
            }                                      \
        }                                          \
    } while (0)

struct Region {
    size_t off, bytes;
};

int main(int argc, char **argv) {
    const int iters = argc > 1 ? atoi(argv[1]) : 400;
    std::mt19937_64 rng(0x5EED);
    auto dim = [&](void) -> uint32_t {
        switch (rng() % 4) {
        case 0: return 1 + (uint32_t)(rng() % 24);      // tiny: invalid or clamped levels
        case 1: return 8 + (uint32_t)(rng() % 120);     // small: clamped DSSIM levels
        case 2: return 64 + (uint32_t)(rng() % 1000);
        default: return 500 + (uint32_t)(rng() % 3500);
        }
    };
    size_t planned = 0, with_clamp = 0;
    for (int it = 0; it < iters; it++) {
        Engine e;  // not initialised: planning is host-only
        e.metrics = 1 + (int)(rng() % 3);
        e.scale_rule = (int)(rng() % 3);
        e.storage = (int)(rng() % 3);
        e.strip_rows_cfg = 21;
        e.blur = rng() % 4 == 0 ? S2_BLUR_IIR_REF : S2_BLUR_FIR;
        const int n = 1 + (int)(rng() % 12);
        std::vector<s2_pair_desc> d(n);
        for (auto &q : d) {
            memset(&q, 0, sizeof q);
            q.format = (int)(rng() % 5);
            q.width = dim();
            q.height = dim();
            if (q.format == S2_FMT_NV12 || q.format == S2_FMT_P016) q.width += q.width & 1, q.height += q.height & 1;
            q.bits = 10;
            q.ref = q.dis = q.ref_uv = q.dis_uv = (const void *)64;
            q.ref_pitch = q.dis_pitch = (size_t)q.width * 12;
        }
        Plan P;
        const int ngroups = 1 + (int)(rng() % 6);
        const s2_status st = e.plan(d.data(), n, P, nullptr, e.blur == S2_BLUR_FIR ? ngroups : 1);
        CHECK(st == S2_OK, "plan status %d", (int)st);
        const bool m_s2 = (e.metrics & S2_METRIC_SSIMULACRA2) != 0, m_ds = (e.metrics & S2_METRIC_DSSIM) != 0;
        std::vector<Region> regs;
        const size_t es = e.esize();
        for (int i = 0; i < n; i++) {
            const DevPair &p = P.pairs[i];
            const s2_pair_desc &q = d[i];
            const bool valid = (!m_s2 || s2_num_scales_rule(q.width, q.height, e.scale_rule) > 0) &&
                               (!m_ds || (q.width >= 8 && q.height >= 8));
            CHECK((p.status == S2_OK) == valid, "pair %d status %d for %ux%u metrics %d", i, p.status, q.width,
                  q.height, e.metrics);
            if (p.status != S2_OK) {
                if (m_ds) CHECK(P.ds[i].status == p.status, "DSSIM status of an invalid pair");
                continue;
            }
            planned++;
            CHECK(p.nscales == (m_s2 ? s2_num_scales_rule(q.width, q.height, e.scale_rule) : 0), "nscales");
            for (int s = 0; s < p.nscales; s++) {
                CHECK(p.lp[s] == (int)s2_align_up((size_t)p.w[s], 64), "XYB pitch");
                for (int img = 0; img < 2; img++)
                    regs.push_back({(size_t)p.lvl[img][s], s2_align_up((size_t)3 * p.lp[s] * p.h[s] * es, 256)});
            }
            if (!m_ds) {
                CHECK(p.lab_levels == 0, "Lab levels without DSSIM");
                continue;
            }
            const DsPair &D = P.ds[i];
            CHECK(D.status == 0, "DSSIM status %d", D.status);
            int dw[kDsLevels], dh[kDsLevels];
            uint32_t w = q.width, h = q.height;
            for (int s = 0; s < kDsLevels; s++) {
                dw[s] = (int)w, dh[s] = (int)h;
                w = std::max<uint32_t>((w + 1) / 2, 8), h = std::max<uint32_t>((h + 1) / 2, 8);
                CHECK(D.w[s] == dw[s] && D.h[s] == dh[s], "DSSIM size of level %d", s);
                CHECK(D.pitch[s] >= D.w[s] && D.pitch[s] % 64 == 0, "DSSIM pitch");
            }
            int ll = 0;
            while (ll < kDsLevels && dw[ll] == p.w[ll] && dh[ll] == p.h[ll]) ll++;
            CHECK(ll >= 1 && p.lab_levels == ll && D.clamp_from == ll, "Lab levels %d / %d", p.lab_levels, ll);
            CHECK(p.prep_levels == std::max(p.nscales, ll), "prep levels");
            for (int s = 0; s < p.prep_levels; s++) CHECK(p.lp[s] == (int)s2_align_up((size_t)p.w[s], 64), "pitch");
            for (int s = 0; s < kDsLevels; s++) {
                for (int img = 0; img < 2; img++) {
                    if (s < ll) CHECK(p.lab[img][s] == D.lab[img][s] && D.pitch[s] == p.lp[s], "prep Lab plane");
                    regs.push_back({(size_t)D.lab[img][s],
                                    s2_align_up((size_t)3 * D.pitch[s] * D.h[s] * sizeof(float), 256)});
                }
                regs.push_back({(size_t)D.map[s], s2_align_up((size_t)D.pitch[s] * D.h[s] * sizeof(float), 256)});
                CHECK(D.tile_cnt[s] == ((D.w[s] + 31) / 32) * ((D.h[s] + 31) / 32), "tile count");
            }
            if (ll < kDsLevels) {
                with_clamp++;
                CHECK(D.kw == p.w[ll - 1] && D.kh == p.h[ll - 1] && D.kpitch == p.lp[ll - 1], "kept level");
                for (int s = ll; s < kDsLevels; s++)
                    CHECK(D.splane >= (long long)D.pitch[s] * D.h[s], "scratch plane of level %d", s);
                for (int img = 0; img < 2; img++) {
                    CHECK(p.keep[img] == D.keep[img], "keep pointer");
                    regs.push_back({(size_t)D.keep[img], s2_align_up((size_t)3 * D.kpitch * D.kh * sizeof(float), 256)});
                    regs.push_back({(size_t)D.scratch[img], s2_align_up((size_t)6 * D.splane * sizeof(float), 256)});
                }
            }
        }
        std::sort(regs.begin(), regs.end(), [](const Region &a, const Region &b) { return a.off < b.off; });
        for (size_t k = 0; k < regs.size(); k++) {
            CHECK(regs[k].off % 256 == 0, "alignment");
            CHECK(regs[k].off + regs[k].bytes <= P.level_bytes, "region past the level bytes");
            if (k) CHECK(regs[k - 1].off + regs[k - 1].bytes <= regs[k].off, "overlapping regions");
        }
        if (m_ds) {
            int next = 0;
            for (const DsSeg &sg : P.dsegs) {
                CHECK(sg.first_tile == next, "DSSIM tiles not contiguous");
                const DsPair &D = P.ds[sg.pair];
                CHECK(D.tile_base[sg.level] == sg.first_tile && sg.tiles_x == (D.w[sg.level] + 31) / 32, "segment");
                next += D.tile_cnt[sg.level];
            }
            CHECK(next == P.ds_tiles, "DSSIM tile total");
        }
        if (e.blur == S2_BLUR_IIR_REF) {
            // the reference's recursion: one record per row of each scored
            // (pair, scale), its vertical-walk planes packed back to back
            int rec = 0;
            size_t vb = 0;
            CHECK(P.vsegs.size() == P.hsegs.size(), "IIR segments");
            for (size_t k = 0; k < P.vsegs.size(); k++) {
                const IirSeg &v = P.vsegs[k];
                const DevPair &p = P.pairs[v.pair];
                CHECK(v.rec_base == rec && p.tile_base[v.scale] == rec && p.tile_cnt[v.scale] == p.h[v.scale],
                      "IIR records");
                CHECK((size_t)v.v == vb && (size_t)P.hsegs[k].v == vb, "IIR planes");
                rec += p.h[v.scale];
                vb += s2_align_up((size_t)15 * p.lp[v.scale] * p.h[v.scale] * sizeof(float), 256);
            }
            CHECK(rec == P.total_tiles && vb == P.v_bytes, "IIR totals");
            continue;
        }
        // groups of a host-input submission: contiguous pairs and tiles, all covered
        const int ng = (int)P.grp_pair.size() - 1;
        CHECK(ng >= 1 && ng <= std::min(ngroups, n) && P.grp_pair.front() == 0 && P.grp_pair.back() == n,
              "group pairs");
        CHECK((int)P.grp_tile.size() == ng + 1 && P.grp_tile.front() == 0 && P.grp_tile.back() == P.total_tiles,
              "group tiles");
        for (int g = 0; g < ng; g++) {
            CHECK(P.grp_pair[g] < P.grp_pair[g + 1] && P.grp_tile[g] <= P.grp_tile[g + 1], "group order");
            for (int i = P.grp_pair[g]; i < P.grp_pair[g + 1]; i++)
                for (int sc = 0; sc < P.pairs[i].nscales && P.pairs[i].status == S2_OK; sc++)
                    CHECK(P.pairs[i].tile_base[sc] >= P.grp_tile[g] &&
                              P.pairs[i].tile_base[sc] + P.pairs[i].tile_cnt[sc] <= P.grp_tile[g + 1],
                          "a pair's tiles outside its group");
        }
        // staging of host planes: every plane the prep pass reads, packed, aligned, disjoint
        const size_t stage = Engine::plan_staging(P, d.data());
        std::vector<Region> st_regs;
        for (int i = 0; i < n; i++) {
            const DevPair &p = P.pairs[i];
            if (p.status != S2_OK) continue;
            const size_t row = s2_row_bytes(d[i]);
            for (int img = 0; img < 2; img++) {
                CHECK(p.pitch[img] == (long long)row, "staged pitch");
                st_regs.push_back({(size_t)p.in[img], s2_align_up(row * d[i].height, 256)});
                if (s2_is_yuv420(d[i].format))
                    st_regs.push_back({(size_t)p.in_uv[img], s2_align_up(row * (d[i].height / 2), 256)});
            }
        }
        std::sort(st_regs.begin(), st_regs.end(), [](const Region &a, const Region &b) { return a.off < b.off; });
        for (size_t k = 0; k < st_regs.size(); k++) {
            CHECK(st_regs[k].off % 256 == 0 && st_regs[k].off + st_regs[k].bytes <= stage, "staging bounds");
            if (k) CHECK(st_regs[k - 1].off + st_regs[k - 1].bytes <= st_regs[k].off, "overlapping staging");
        }
    }
    printf("%s fails=%d pairs=%zu clamped=%zu\n", fails ? "FAILED" : "OK", fails, planned, with_clamp);
    return fails ? 1 : 0;
}
