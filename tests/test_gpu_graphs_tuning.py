"""CUDA-graph replay and the tile-height autotuner.

Graph replay must pick up every submission's own pairs (pointers and sizes
travel in the uploaded descriptors): submissions of one shape with different
images, and a shape change, score exactly as with graphs off.  The autotuner
changes only how the work is cut into tiles, so its choice moves no score by
more than f64 summation order (1e-12), and once made it is kept."""
import numpy as np
import pytest

import synth

pytestmark = pytest.mark.gpu


def dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def batch_of(tmb, torch, sizes, seed):
    out = []
    for i, (w, h) in enumerate(sizes):
        r, d = synth.srgb_pair(w, h, seed + i)
        out.append(tmb.PairDesc(dev(torch, r), dev(torch, d), "srgb8"))
    return out


def test_graph_replay_follows_each_submission(tmb, cuda):
    shape = [(300, 200), (257, 131), (640, 360)]
    subs = [batch_of(tmb, cuda, shape, 700 + 10 * k) for k in range(3)]
    subs.append(batch_of(tmb, cuda, [(97, 333), (512, 512)], 800))  # another shape
    subs.append(subs[0])                                              # the first shape again
    g = tmb.Ssim2Batch(8, 4 << 20, strip_rows=32)
    plain = tmb.Ssim2Batch(8, 4 << 20, strip_rows=32)
    plain.set_graphs(False)
    for pairs in subs:
        a = g.compute_batch(pairs)
        b = plain.compute_batch(pairs)
        assert [x[0] for x in a] == [x[0] for x in b]
        for x, y in zip(a, b):
            assert np.array_equal(x[1], y[1])
    # different images of one shape give different scores (the replay did not reuse old inputs)
    s0 = [x[0] for x in g.compute_batch(subs[0])]
    s1 = [x[0] for x in g.compute_batch(subs[1])]
    assert s0 != s1


def test_single_pair_graphs_on_and_off(tmb, cuda):
    ref, dis = synth.srgb_pair(400, 300, 901)
    ref2, dis2 = synth.srgb_pair(400, 300, 902)
    s = tmb.Ssimulacra2(400, 300, strip_rows=16)
    t = tmb.Ssimulacra2(400, 300, strip_rows=16)
    t.set_graphs(False)
    for r, d in ((ref, dis), (ref2, dis2), (ref, dis)):
        s.compute_srgb(dev(cuda, r), dev(cuda, d))
        t.compute_srgb(dev(cuda, r), dev(cuda, d))
        assert s.get_score() == t.get_score()


def test_autotuned_tile_height_matches_fixed_heights(tmb, cuda):
    pairs = batch_of(tmb, cuda, [(1920, 1080), (1280, 720), (700, 500)], 950)
    auto = tmb.Ssim2Batch(4, 8 << 20)  # strip_rows 0: autotuned
    first = auto.compute_batch(pairs)
    again = auto.compute_batch(pairs)
    assert [x[0] for x in first] == [x[0] for x in again]  # the choice is kept
    for rows in (16, 32, 64):
        fixed = tmb.Ssim2Batch(4, 8 << 20, strip_rows=rows).compute_batch(pairs)
        for a, f in zip(first, fixed):
            assert abs(a[0] - f[0]) < 1e-12
            assert np.allclose(a[1], f[1], rtol=1e-12, atol=1e-15)


def nv12_batch_of(tmb, torch, sizes, seed):
    out = []
    for i, (w, h) in enumerate(sizes):
        (ry, ruv), (dy, duv) = synth.nv12_frame_pair(w, h, seed + i)
        out.append(tmb.PairDesc(dev(torch, ry), dev(torch, dy), "nv12", dev(torch, ruv), dev(torch, duv)))
    return out


def test_graph_replay_follows_the_input_format(tmb, cuda):
    """A submission whose pairs share one input format runs a prep kernel
    compiled for that format, so a replayed graph must be the one recorded
    for the same format: sRGB8, NV12 and a mix of both, all of one shape
    (same sizes, same tile plan), alternate on one batch with graphs on and
    score exactly as on a batch with graphs off."""
    shape = [(320, 180), (256, 144)]
    srgb = batch_of(tmb, cuda, shape, 1200)
    nv12 = nv12_batch_of(tmb, cuda, shape, 1300)
    mixed = [srgb[0], nv12[1]]
    g = tmb.Ssim2Batch(4, 1 << 20, strip_rows=32)
    plain = tmb.Ssim2Batch(4, 1 << 20, strip_rows=32)
    plain.set_graphs(False)
    for pairs in (srgb, nv12, mixed, srgb, mixed, nv12):
        a = g.compute_batch(pairs)
        b = plain.compute_batch(pairs)
        assert [x[0] for x in a] == [x[0] for x in b]
        for x, y in zip(a, b):
            assert np.array_equal(x[1], y[1])
    # the mixed submission scores each pair as its own-format submission does
    m = g.compute_batch(mixed)
    assert m[0][0] == g.compute_batch(srgb)[0][0]
    assert m[1][0] == g.compute_batch(nv12)[1][0]
