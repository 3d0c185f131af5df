// dssim_map_check.cu -- host-only check of the DSSIM tile pass's
// thread-to-item mapping (ds_item in turbo-metrics_b200/csrc/dssim_tile_map.h)
// for the three blur stages the pass runs: the threads of a block cover every
// (plane, row segment, column pair) of a stage exactly once, every item lies
// inside the stage, and each aligned half-warp of the main part reads one
// row segment of one plane at 16 consecutive column pairs (32 consecutive
// floats of a row: no shared-memory bank conflicts).  Built and run by
// tests/test_cpu_dssim_map.py; makes no CUDA call.
#include <cstdio>
#include <set>
#include <tuple>

#include "../turbo-metrics_b200/csrc/dssim_tile_map.h"

using namespace s2;

static int fails = 0;
#define CHECK(c, ...)                                               \
    do {                                                            \
        if (!(c)) {                                                 \
            if (fails++ < 20) {                                     \
                printf("FAIL %s:%d: ", __FILE__, __LINE__);         \
                printf(__VA_ARGS__);                                \
                printf("\n");                                       \
            }                                                       \
        }                                                           \
    } while (0)

template <int n, int planes, int S, int L>
static void check_stage(const char *name) {
    constexpr int half = n / 2;
    static_assert(planes * half * S <= kDsThreads && S * L >= n && L <= n && n % 2 == 0, "one run per thread");
    std::set<std::tuple<int, int, int>> seen;
    int items = 0;
    for (int t = 0; t < kDsThreads; t++) {
        int p, seg, c;
        if (!ds_item<half, S, planes>(t, p, seg, c)) continue;
        items++;
        CHECK(p >= 0 && p < planes && seg >= 0 && seg < S && c >= 0 && c < n && c % 2 == 0,
              "%s: thread %d -> (%d, %d, %d) outside the stage", name, t, p, seg, c);
        CHECK(seen.insert(std::make_tuple(p, seg, c)).second, "%s: (%d, %d, %d) twice", name, p, seg, c);
    }
    CHECK(items == planes * half * S, "%s: %d items, want %d", name, items, planes * half * S);
    // the main part: aligned half-warps of one (plane, segment), 16 consecutive pairs
    for (int h = 0; h < planes * S; h++) {
        int p0, s0, c0;
        ds_item<half, S, planes>(16 * h, p0, s0, c0);
        for (int l = 0; l < 16; l++) {
            int p, seg, c;
            ds_item<half, S, planes>(16 * h + l, p, seg, c);
            CHECK(p == p0 && seg == s0 && c == 2 * l, "%s: half-warp %d lane %d -> (%d, %d, %d)", name, h, l, p,
                  seg, c);
        }
    }
    printf("%s: %d items, %d threads\n", name, items, kDsThreads);
}

int main() {
    check_stage<kDsP, 2, kDsPre1S, kDsPre1L>("a/b pre-blur 1");
    check_stage<kDsX, 2, kDsPre2S, kDsPre2L>("a/b pre-blur 2");
    check_stage<kDsB, 5, kDsStatS, kDsStatL>("statistics blur");
    if (fails) {
        printf("%d failures\n", fails);
        return 1;
    }
    printf("OK\n");
    return 0;
}
