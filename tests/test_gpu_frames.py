"""Frame-pair driver on the GPU: per-frame scores equal the single-pair
drop-in's, in frame order, with two submissions in flight."""
import numpy as np
import pytest

import synth

pytestmark = pytest.mark.gpu


def test_driver_scores_equal_per_frame_compute(tmb, cuda):
    ref = [synth.nv12_frame_pair(256, 144, 1700 + i)[0] for i in range(7)]
    dis = [synth.nv12_frame_pair(256, 144, 1700 + i)[1] for i in range(9)]
    sc = tmb.FramePairScorer(256, 144, "nv12", frames_per_submission=2)
    scores, stats = sc.compute_all(ref, dis, skip_dis=1, every=1)
    sc.close()
    assert len(scores) == 7
    s = tmb.Ssimulacra2(256, 144)
    want = []
    for (ry, ruv), (dy, duv) in zip(ref, dis[1:]):
        d = lambda a: cuda.from_numpy(np.ascontiguousarray(a)).cuda()
        s.compute_nv12(d(ry), d(ruv), d(dy), d(duv))
        want.append(s.get_score())
    assert np.allclose(scores, want, rtol=0, atol=1e-12)
    assert stats.mean == pytest.approx(np.mean(want)) and stats.min == min(scores)


def test_driver_srgb_every_and_limit(tmb, cuda):
    pairs = [synth.srgb_pair(160, 120, 1800 + i) for i in range(10)]
    sc = tmb.FramePairScorer(160, 120, "srgb8", frames_per_submission=3)
    scores, _ = sc.compute_all([p[0] for p in pairs], [p[1] for p in pairs], every=2, frames=4)
    sc.close()
    b = tmb.Ssim2Batch(4, 4 * 160 * 120)
    want = [r[0] for r in b.compute_batch([tmb.PairDesc(cuda.from_numpy(pairs[i][0]).cuda(),
                                                        cuda.from_numpy(pairs[i][1]).cuda(), "srgb8")
                                           for i in (0, 2)])]  # `frames` counts the skipped pairs too
    assert np.allclose(scores, want, rtol=0, atol=1e-12)
