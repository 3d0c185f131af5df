"""GPU tests of the continuous-batching server (s2_server_*): results equal
the single-pair context's, a job scores bit-identically alone and mixed with
other jobs, admission under the HBM budget, cancellation, bounded waits, and
the latency statistics."""
import numpy as np
import pytest

import synth

pytestmark = pytest.mark.gpu


def job_images(w, h, seed, k):
    ref, _ = synth.srgb_pair(w, h, seed)
    cands = [synth.srgb_pair(w, h, seed, step)[1] for step in (2.0, 6.0, 12.0, 24.0, 40.0)[:k]]
    return ref, cands


def test_server_matches_single_context(tmb, cuda):
    ref, cands = job_images(300, 200, synth.pair_seed(4, 1), 4)
    sv = tmb.Ssim2Server()
    jid = sv.submit(ref, cands)
    scores, st, lat = sv.wait(jid)
    assert list(st) == [0] * 4 and lat > 0
    # a job's candidates are scored against its cached reference: equal bit
    # for bit to a context's compute_with_reference and to the direct path
    ctx = tmb.Ssimulacra2(300, 200)
    ctx.set_reference_srgb(ref, on_host=True)
    for c, s in zip(cands, scores):
        assert abs(ctx.compute_with_reference_srgb(c, on_host=True) - s) < 1e-12
        assert ctx.compute_from_cpu_srgb_sync(ref, c) == s
    sv.close()


def test_server_alone_equals_mixed_bitwise(tmb, cuda):
    ref, cands = job_images(257, 131, synth.pair_seed(4, 2), 5)
    sv = tmb.Ssim2Server(max_batch_pairs=7, max_batch_pixels=1 << 20)
    alone, _, _ = sv.wait(sv.submit(ref, cands))
    others = []
    for i, (w, h) in enumerate([(128, 128), (640, 360), (97, 333), (1024, 576), (200, 150), (333, 97)]):
        r, c = job_images(w, h, synth.pair_seed(4, 10 + i), 3)
        others.append(sv.submit(r, c))
        if i == 2:
            mid = sv.submit(ref, cands)
    mixed, _, _ = sv.wait(mid)
    for o in others:
        sv.wait(o)
    assert np.array_equal(alone, mixed)
    rep = sv.stats()
    assert rep["jobs_done"] == 8 and rep["pairs_done"] == 5 + 5 + 6 * 3
    assert rep["rounds"] > 1 and 0 < rep["p50_ms"] <= rep["p99_ms"] <= rep["max_ms"]
    sv.close()


SMALL = dict(max_batch_pairs=8, max_batch_pixels=1 << 21)


def job_bytes(w, h, k):
    """Device bytes the server admits a job with: inputs + reference XYB
    pyramid (3 f32 planes per scale)."""
    up = lambda v, a: (v + a - 1) // a * a
    total = up(w * h * 3 * (1 + k), 256)
    for _ in range(tmb_num_scales(w, h)):
        total += up(3 * up(w, 64) * h * 4, 256)
        w, h = (w + 1) // 2, (h + 1) // 2
    return total


def tmb_num_scales(w, h):
    import conftest
    return conftest.load_package().num_scales(w, h)


def workspace(tmb, **cfg):
    probe = tmb.Ssim2Server(**(cfg or SMALL))
    ws = probe.stats()["hbm_in_use"]
    probe.close()
    return ws


def test_server_budget_admits_in_order(tmb, cuda):
    # a budget that holds about one job at a time: all still complete, in order
    ref, cands = job_images(512, 512, synth.pair_seed(4, 3), 3)
    sv = tmb.Ssim2Server(hbm_budget=workspace(tmb) + job_bytes(512, 512, 3) * 3 // 2, **SMALL)
    ids = [sv.submit(ref, cands) for _ in range(4)]
    res = [sv.wait(i) for i in ids]
    for r in res[1:]:
        assert np.array_equal(r[0], res[0][0])
    with pytest.raises(tmb.OutOfMemory):
        big = np.zeros((4096, 4096, 3), np.uint8)
        sv.submit(big, [big] * 4)
    sv.close()


def test_server_cancel_and_timeout(tmb, cuda):
    # 1440p jobs, admitted one at a time by the budget: the second job cannot
    # have finished right after the third is submitted (the first one's
    # uploads alone take longer than the calls in between)
    ref, cands = job_images(2560, 1440, synth.pair_seed(4, 4), 5)
    cfg = dict(max_batch_pairs=2, max_batch_pixels=1 << 22)
    sv = tmb.Ssim2Server(hbm_budget=workspace(tmb, **cfg) + job_bytes(2560, 1440, 5) * 3 // 2, **cfg)
    ids = [sv.submit(ref, cands) for _ in range(3)]
    with pytest.raises(tmb.S2Error) as e:
        sv.wait(ids[1], timeout_ms=0)
    assert e.value.status in (6,)  # S2_ERR_TIMEOUT (not done yet)
    sv.cancel(ids[2])  # still queued behind the budget
    with pytest.raises(tmb.S2Error) as e:
        sv.wait(ids[2])
    assert e.value.status == 10  # S2_ERR_CANCELLED
    a, _, _ = sv.wait(ids[0])
    b, _, _ = sv.wait(ids[1])
    assert np.array_equal(a, b)
    sv.close()
