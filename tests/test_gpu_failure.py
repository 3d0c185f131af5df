"""Failure detection of the tile pass, without any GPU fault.

Every wait of the tile pass on its bulk row copies is bounded.  The hook
`s2_debug_tile_timeout(drop_item, wait_cycles)` makes the pass withhold the
row copies of one work item (the bytes are announced on the stage barrier,
nothing is copied), so that item's waits run out after `wait_cycles` SM
cycles.  The kernel records the time-out in a device word and returns; the
finalize pass then marks every pair of the submission S2_ERR_TIMEOUT.  The
tests check that status on the single-pair, batch and error-map paths, and
that the same context, hook reset, scores the pair exactly as before.
"""
import numpy as np
import pytest

import synth

pytestmark = pytest.mark.gpu

WAIT = 1 << 20  # SM cycles per bounded wait, about half a millisecond


def dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.fixture
def hook(tmb):
    def arm(item):
        assert tmb.lib.s2_debug_tile_timeout(item, WAIT) == 0
    yield arm
    assert tmb.lib.s2_debug_tile_timeout(-1, 0) == 0


@pytest.mark.parametrize("item", [0, 5])
def test_single_pair_timeout_then_recovers(tmb, cuda, oracle, hook, item):
    ref, dis = synth.srgb_pair(256, 192, 41, 8)
    s = tmb.Ssimulacra2(256, 192, strip_rows=64)
    s.set_graphs(False)  # a graph keeps the hook's values it was captured with
    r, d = dev(cuda, ref), dev(cuda, dis)
    s.compute_srgb(r, d)
    want = s.get_result()
    hook(item)
    s.compute_srgb(r, d)
    with pytest.raises(tmb.capi.Timeout):
        s.get_result()
    with pytest.raises(tmb.capi.Timeout):
        s.error_maps(0)
    tmb.lib.s2_debug_tile_timeout(-1, 0)
    cuda.cuda.synchronize()  # the context is still usable
    s.compute_srgb(r, d)
    got = s.get_result()
    assert got[0] == want[0]
    assert np.array_equal(got[1], want[1])
    assert abs(got[0] - oracle.ssim2_srgb8(ref, dis, "fir32").score) < 2e-6
    maps = s.error_maps(0)
    assert bool(cuda.isfinite(maps).all())
    s.close()


def test_batch_timeout_marks_every_pair(tmb, cuda, hook):
    pairs = [synth.srgb_pair(160 + 24 * i, 120 + 8 * i, 50 + i, 8) for i in range(3)]
    b = tmb.Ssim2Batch(8, 1 << 20, strip_rows=32)
    b.set_graphs(False)
    descs = [tmb.PairDesc(dev(cuda, r), dev(cuda, d), "srgb8") for r, d in pairs]
    want = b.compute_batch(descs)
    assert all(w[4] == 0 for w in want)
    hook(7)
    got = b.compute_batch(descs)
    assert [g[4] for g in got] == [tmb.capi.S2_ERR_TIMEOUT] * 3
    tmb.lib.s2_debug_tile_timeout(-1, 0)
    again = b.compute_batch(descs)
    for a, w in zip(again, want):
        assert a[4] == 0 and a[0] == w[0] and np.array_equal(a[1], w[1])
    b.close()
