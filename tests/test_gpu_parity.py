"""GPU parity: the CUDA engine, through the C ABI, against the CPU oracle.

Two bars, on the same seeded inputs:
  * `fir32` -- the oracle's restatement of this engine's f32 arithmetic
    (same taps, shift anchors, FMA placement and 8-pixel f32 partial sums):
    every one of the 108 statistics within 2e-6 relative (or 1e-12 absolute
    for statistics that are ~0), score within 2e-6.  Differences come only
    from the error maps' division (the hardware reciprocal approximation and
    one correction on the GPU, an FMA-only Newton division in the oracle; both
    give the IEEE quotient outside rare near-halfway cases) and the f64
    summation order.
  * `fp64` -- the FP64 oracle: score within 1e-3 absolute (the metric's bar).
"""
import numpy as np
import pytest

import synth

pytestmark = pytest.mark.gpu

REL = 2e-6
ABS = 1e-12
SCORE_TOL = 2e-6
FP64_TOL = 1e-3


def dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def assert_stats_close(got, want, rel=REL, abs_=ABS, what=""):
    got, want = np.asarray(got), np.asarray(want)
    err = np.abs(got - want)
    bad = err > np.maximum(rel * np.abs(want), abs_)
    assert not bad.any(), "%s: stats %s differ: got %s want %s" % (
        what, np.nonzero(bad)[0][:8], got[bad][:8], want[bad][:8])


def run_srgb(tmb, torch, ref, dis, rule="cpu", storage="f32"):
    h, w = ref.shape[:2]
    s = tmb.Ssimulacra2(w, h, scale_rule=rule, storage=storage)
    s.compute_srgb(dev(torch, ref), dev(torch, dis))
    out = s.get_result()
    s.close()
    return out


@pytest.mark.parametrize("w,h,seed,step", [(512, 512, synth.pair_seed(0, 0), 16), (256, 256, 11, 2),
                                           (123, 45, 5, 8), (200, 150, 6, 16), (1024, 768, 9, 16),
                                           (300, 64, 10, 32)])
def test_srgb8_matches_oracle(tmb, oracle, cuda, w, h, seed, step):
    ref, dis = synth.srgb_pair(w, h, seed, step)
    score, stats, sums = run_srgb(tmb, cuda, ref, dis)
    mirror = oracle.ssim2_srgb8(ref, dis, "fir32")
    assert_stats_close(stats, mirror.stats, what="fir32 %dx%d" % (w, h))
    assert abs(score - mirror.score) < SCORE_TOL
    exact = oracle.ssim2_srgb8(ref, dis, "fp64")
    assert abs(score - exact.score) < FP64_TOL, (score, exact.score)


@pytest.mark.parametrize("rule", ["cpu", "min8", "all6"])
@pytest.mark.parametrize("w,h", [(16, 16), (8, 8), (9, 13), (64, 64), (33, 17), (8, 300)])
def test_small_sizes_and_scale_rules(tmb, oracle, cuda, rule, w, h):
    ref, dis = synth.synthetic_pair(w, h, 4)
    score, stats, _ = run_srgb(tmb, cuda, ref, dis, rule=rule)
    mirror = oracle.ssim2_srgb8(ref, dis, "fir32", rule)
    assert tmb.num_scales(w, h, rule) == mirror.n_scales == oracle.num_scales(w, h, rule)
    assert_stats_close(stats, mirror.stats, what="%dx%d %s" % (w, h, rule))
    assert abs(score - mirror.score) < SCORE_TOL
    # unscored scales hold zero
    for c in range(3):
        for s in range(mirror.n_scales, 6):
            assert not np.any(stats[c * 36 + s * 6: c * 36 + s * 6 + 6])


def test_16x16_two_or_three_scales(tmb, oracle, cuda):
    # ssim2-gpu/tests/parity_lock.rs:464-491: 16x16 -> 2 scales under its rule;
    # the CPU crate's rule (checked before downscaling) also scores 4x4.
    assert tmb.num_scales(16, 16, "min8") == 2
    assert tmb.num_scales(16, 16, "cpu") == 3
    assert tmb.num_scales(16, 16, "all6") == 6


def test_identical_scores_100(tmb, cuda):
    ref, _ = synth.srgb_pair(256, 192, 3)
    score, stats, _ = run_srgb(tmb, cuda, ref, ref.copy())
    assert score == 100.0
    assert not np.any(stats)


def test_linear_input_with_row_padding(tmb, oracle, cuda):
    ref8, dis8 = synth.srgb_pair(160, 96, 21)
    ref = oracle.srgb8_to_linear(ref8)
    dis = oracle.srgb8_to_linear(dis8)
    pad = cuda.zeros((96, 200, 3), dtype=cuda.float32, device="cuda")
    pad2 = cuda.zeros((96, 200, 3), dtype=cuda.float32, device="cuda")
    pad[:, :160] = cuda.from_numpy(ref).cuda()
    pad2[:, :160] = cuda.from_numpy(dis).cuda()
    s = tmb.Ssimulacra2(160, 96)
    s.compute_linear((pad.data_ptr(), 200 * 12), (pad2.data_ptr(), 200 * 12))
    score, stats, _ = s.get_result()
    mirror = oracle.ssim2_linear(ref, dis, "fir32")
    assert_stats_close(stats, mirror.stats)
    assert abs(score - mirror.score) < SCORE_TOL


def test_get_score_idempotent(tmb, cuda):
    ref, dis = synth.srgb_pair(128, 128, 4)
    s = tmb.Ssimulacra2(128, 128)
    s.compute_srgb(dev(cuda, ref), dev(cuda, dis))
    a = s.get_score()
    b = s.get_score()
    assert a == b


def test_host_srgb_path(tmb, oracle, cuda):
    ref, dis = synth.srgb_pair(320, 200, 8)
    s = tmb.Ssimulacra2(320, 200)
    score = s.compute_from_cpu_srgb_sync(ref, dis)
    assert abs(score - oracle.ssim2_srgb8(ref, dis, "fir32").score) < SCORE_TOL


def test_nv12_matches_oracle(tmb, oracle, cuda):
    (ry, ruv), (dy, duv) = synth.nv12_frame_pair(480, 272, 77)
    h, w = ry.shape
    s = tmb.Ssimulacra2(w, h)
    s.compute_nv12(dev(cuda, ry), dev(cuda, ruv), dev(cuda, dy), dev(cuda, duv))
    score, stats, _ = s.get_result()
    rl, dl = oracle.nv12_to_linear(ry, ruv), oracle.nv12_to_linear(dy, duv)
    mirror = oracle.ssim2_linear(rl, dl, "fir32")
    # powf differs between CUDA and glibc by <= 1-2 ulp
    assert_stats_close(stats, mirror.stats, rel=2e-5, abs_=1e-10)
    assert abs(score - mirror.score) < 2e-5
    exact = oracle.ssim2_linear(oracle.nv12_to_linear(ry, ruv, True), oracle.nv12_to_linear(dy, duv, True), "fp64")
    assert abs(score - exact.score) < FP64_TOL


def test_nv12_host_path(tmb, cuda):
    (ry, ruv), (dy, duv) = synth.nv12_frame_pair(256, 144, 78)
    s = tmb.Ssimulacra2(256, 144)
    s.compute_nv12(dev(cuda, ry), dev(cuda, ruv), dev(cuda, dy), dev(cuda, duv))
    a = s.get_score()
    s.compute_nv12(ry, ruv, dy, duv, on_host=True)
    assert s.get_score() == a


def test_rgb16_matches_oracle(tmb, oracle, cuda):
    ref, dis = synth.rgb10_pair(384, 216, 99)
    s = tmb.Ssimulacra2(384, 216)
    rt = dev(cuda, ref.view(np.int16))
    dt = dev(cuda, dis.view(np.int16))
    s.compute_rgb16((rt.data_ptr(), 384 * 6), (dt.data_ptr(), 384 * 6), bits=10)
    score, stats, _ = s.get_result()
    mirror = oracle.ssim2_linear(oracle.rgb16_to_linear(ref), oracle.rgb16_to_linear(dis), "fir32")
    assert_stats_close(stats, mirror.stats, rel=2e-5, abs_=1e-10)
    assert abs(score - mirror.score) < 2e-5


def test_error_paths(tmb, cuda):
    with pytest.raises(tmb.InvalidImageSize):
        tmb.Ssimulacra2(7, 100)
    with pytest.raises(tmb.InvalidImageSize):
        tmb.Ssimulacra2(100, 4)
    s = tmb.Ssimulacra2(64, 64)
    with pytest.raises(tmb.NoCachedReference):
        s.compute_with_reference_srgb(np.zeros((64, 64, 3), np.uint8), on_host=True)
    with pytest.raises(tmb.DimensionMismatch):
        s.compute_from_cpu_srgb_sync(np.zeros((64, 63, 3), np.uint8), np.zeros((64, 63, 3), np.uint8))
    a = cuda.zeros((64, 64, 3), dtype=cuda.uint8, device="cuda")
    with pytest.raises(tmb.DimensionMismatch):
        s.compute_srgb((a.data_ptr(), 100), (a.data_ptr(), 192))
    odd = tmb.Ssimulacra2(65, 64)
    y = cuda.zeros((64, 65), dtype=cuda.uint8, device="cuda")
    with pytest.raises(tmb.InvalidImageSize):
        odd.compute_nv12(y, y[:32], y, y[:32])


def test_cached_reference_equals_direct(tmb, oracle, cuda):
    """The cached path converts only the distorted image and runs the same
    tile pass over the cached reference planes: the score equals the direct
    path's bit for bit (the
    reference's own bar for cached == direct is 1e-4,
    ssim2-gpu/tests/parity_lock.rs:160-277), every statistic against the
    oracle's fir32 restatement."""
    ref, _ = synth.srgb_pair(200, 150, 31)
    s = tmb.Ssimulacra2(200, 150)
    assert not s.has_reference()
    s.set_reference_srgb(ref, on_host=True)
    assert s.has_reference()
    for q in (4, 16, 40):
        _, dis = synth.srgb_pair(200, 150, 31, q)
        direct = s.compute_from_cpu_srgb_sync(ref, dis)
        s.compute_with_reference_srgb(dis, on_host=True)
        cached, stats, _ = s.get_result()
        assert direct == cached
        mirror = oracle.ssim2_srgb8(ref, dis, "fir32")
        assert_stats_close(stats, mirror.stats, what="cached q%d" % q)
        assert abs(cached - mirror.score) < SCORE_TOL
    # the reference compared with itself through the cache scores exactly 100
    s.compute_with_reference_srgb(ref, on_host=True)
    assert s.get_score() == 100.0
    s.clear_reference()
    assert not s.has_reference()
    with pytest.raises(tmb.NoCachedReference):
        s.compute_with_reference_srgb(ref, on_host=True)


def test_batch_uneven_equals_single(tmb, cuda):
    sizes = [(64, 64), (123, 45), (517, 300), (1000, 61), (256, 256), (8, 8), (7, 50)]
    pairs, host = [], []
    for i, (w, h) in enumerate(sizes):
        r, d = synth.srgb_pair(w, h, 500 + i)
        host.append((r, d))
        pairs.append(tmb.PairDesc(dev(cuda, r), dev(cuda, d), "srgb8"))
    b = tmb.Ssim2Batch(16, 4 << 20)
    res = b.compute_batch(pairs)
    for (w, h), (r, d), out in zip(sizes, host, res):
        if w < 8 or h < 8:
            assert out[4] == 2  # S2_ERR_INVALID_SIZE
            continue
        assert out[4] == 0
        single = run_srgb(tmb, cuda, r, d)
        assert abs(out[0] - single[0]) < 1e-12
        assert_stats_close(out[1], single[1], rel=1e-12, abs_=1e-15)
    # repeated submission is deterministic
    res2 = b.compute_batch(pairs)
    assert [x[0] for x in res] == [x[0] for x in res2]


def test_batch_nv12_1080p_pair(tmb, oracle, cuda):
    (ry, ruv), (dy, duv) = synth.c1_pair(0)
    b = tmb.Ssim2Batch(2, 1920 * 1080 * 2)
    p = tmb.PairDesc(dev(cuda, ry), dev(cuda, dy), "nv12", dev(cuda, ruv), dev(cuda, duv))
    out = b.compute_batch([p, p])
    assert out[0][0] == out[1][0]
    exact = oracle.ssim2_linear(oracle.nv12_to_linear(ry, ruv, True), oracle.nv12_to_linear(dy, duv, True), "fp64")
    assert abs(out[0][0] - exact.score) < FP64_TOL, (out[0][0], exact.score)


def test_nv12_1080p_per_statistic(tmb, oracle, cuda):
    """The bench workload's size and format (one 1920x1080 NV12 BT.709
    limited pair of the 64): every statistic against fir32, the score against
    FP64."""
    (ry, ruv), (dy, duv) = synth.c1_pair(5)
    s = tmb.Ssimulacra2(1920, 1080)
    s.compute_nv12(dev(cuda, ry), dev(cuda, ruv), dev(cuda, dy), dev(cuda, duv))
    score, stats, _ = s.get_result()
    s.close()
    rl, dl = oracle.nv12_to_linear(ry, ruv), oracle.nv12_to_linear(dy, duv)
    mirror = oracle.ssim2_linear(rl, dl, "fir32")
    assert_stats_close(stats, mirror.stats, what="1080p nv12")
    assert abs(score - mirror.score) < SCORE_TOL
    exact = oracle.ssim2_linear(oracle.nv12_to_linear(ry, ruv, True), oracle.nv12_to_linear(dy, duv, True), "fp64")
    assert abs(score - exact.score) < FP64_TOL, (score, exact.score)


@pytest.mark.parametrize("w,h", [(2047, 1999), (1999, 64), (2048, 2047)])
def test_uneven_sizes_near_the_top_of_the_range(tmb, oracle, cuda, w, h):
    """Sizes near 2048 of the uneven-size workload (width and height in
    [64, 2048], not multiples of the tile): inside one batch with a small pair,
    every statistic against fir32 and the score against FP64."""
    i = 3000 + w + h
    ref, dis = synth.srgb_pair(w, h, synth.pair_seed(2, i), 24)
    small_r, small_d = synth.srgb_pair(97, 71, synth.pair_seed(2, i + 1), 8)
    b = tmb.Ssim2Batch(2, w * h + 97 * 71)
    out = b.compute_batch([tmb.PairDesc(dev(cuda, ref), dev(cuda, dis), "srgb8"),
                           tmb.PairDesc(dev(cuda, small_r), dev(cuda, small_d), "srgb8")])
    b.close()
    mirror = oracle.ssim2_srgb8(ref, dis, "fir32")
    assert_stats_close(out[0][1], mirror.stats, what="%dx%d" % (w, h))
    assert abs(out[0][0] - mirror.score) < SCORE_TOL
    exact = oracle.ssim2_srgb8(ref, dis, "fp64")
    assert abs(out[0][0] - exact.score) < FP64_TOL, (out[0][0], exact.score)
    small = oracle.ssim2_srgb8(small_r, small_d, "fir32")
    assert_stats_close(out[1][1], small.stats, what="97x71 beside %dx%d" % (w, h))


@pytest.mark.parametrize("storage", ["f16", "bf16"])
def test_reduced_precision_storage_refused(tmb, cuda, storage):
    """16-bit storage of the XYB planes is not offered (the passes are
    compute-bound, so it bought no time, and it cost up to 0.2 / 4 in
    score): a context asking for it is refused with S2_ERR_INVALID_ARG."""
    with pytest.raises(tmb.InvalidArgument):
        tmb.Ssimulacra2(64, 64, storage=storage)
    with pytest.raises(tmb.InvalidArgument):
        tmb.Ssim2Batch(2, 2 * 64 * 64, storage=storage)
