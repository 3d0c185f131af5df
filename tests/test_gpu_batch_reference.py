"""The batch's cached reference (s2_batch_set_reference /
s2_batch_submit_with_reference), the semantics of ssim2-gpu's Ssim2Batch
(crates/ssim2-gpu/src/pipeline_batch.rs:206-330): one resident reference,
many distorted images per submission.  Candidates read the reference's
cached blurred mean: checked statistic by statistic against the oracle's
fir32 restatement, and equal bit for bit to the direct path."""
import numpy as np
import pytest

import synth

pytestmark = pytest.mark.gpu

REL, ABS = 2e-6, 1e-12


def dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def close(got, want):
    err = np.abs(np.asarray(got) - np.asarray(want))
    return np.all(err <= np.maximum(REL * np.abs(want), ABS))


def test_batch_reference_srgb_against_oracle_and_direct(tmb, oracle, cuda):
    w, h = 333, 217
    ref, _ = synth.srgb_pair(w, h, synth.pair_seed(0, 40))
    cands = [synth.srgb_pair(w, h, synth.pair_seed(0, 40), st)[1] for st in (3.0, 9.0, 27.0)]
    b = tmb.Ssim2Batch(4, 4 * w * h)
    assert not b.has_cached_reference()
    with pytest.raises(tmb.NoCachedReference):
        b.compute_batch_with_reference([dev(cuda, cands[0])])
    b.set_reference(dev(cuda, ref))
    assert b.has_cached_reference()
    out = b.compute_batch_with_reference([dev(cuda, c) for c in cands])
    direct = b.compute_batch([tmb.PairDesc(dev(cuda, ref), dev(cuda, c), "srgb8") for c in cands])
    for c, o, d in zip(cands, out, direct):
        assert o[4] == 0
        mirror = oracle.ssim2_srgb8(ref, c, "fir32")
        assert close(o[1], mirror.stats)
        assert abs(o[0] - mirror.score) < 2e-6
        assert o[0] == d[0]
    # a second submission against the same cache gives the same scores
    again = b.compute_batch_with_reference([dev(cuda, c) for c in cands])
    assert [x[0] for x in again] == [x[0] for x in out]
    # the reference itself scores 100
    assert b.compute_batch_with_reference([dev(cuda, ref)])[0][0] == 100.0
    b.close()


def test_batch_reference_errors(tmb, cuda):
    w, h = 64, 48
    ref, dis = synth.srgb_pair(w, h, 41)
    b = tmb.Ssim2Batch(2, 4 * w * h)
    b.set_reference(dev(cuda, ref))
    other = synth.srgb_pair(w + 2, h, 42)[1]
    with pytest.raises(tmb.DimensionMismatch):
        b.compute_batch_with_reference([dev(cuda, other)])
    with pytest.raises(tmb.S2Error):  # more than max_pairs (InvalidBatchSize in the reference)
        b.compute_batch_with_reference([dev(cuda, dis)] * 3)
    b.clear_reference()
    assert not b.has_cached_reference()
    with pytest.raises(tmb.NoCachedReference):
        b.compute_batch_with_reference([dev(cuda, dis)])
    b.close()


def test_batch_reference_nv12_frames(tmb, oracle, cuda):
    """An NV12 reference frame and NV12 candidates (the encoder's case)."""
    ref, _ = synth.nv12_frame_pair(320, 180, synth.pair_seed(1, 900))
    cands = [synth.nv12_candidate(ref, synth.c1_candidate_step(k)) for k in range(3)]
    b = tmb.Ssim2Batch(4, 4 * 320 * 180)
    b.set_reference(dev(cuda, ref[0]), "nv12", ref_uv=dev(cuda, ref[1]))
    out = b.compute_batch_with_reference([dev(cuda, c[0]) for c in cands], "nv12",
                                         dis_uv=[dev(cuda, c[1]) for c in cands])
    rl = oracle.nv12_to_linear(*ref)
    for c, o in zip(cands, out):
        mirror = oracle.ssim2_linear(rl, oracle.nv12_to_linear(*c), "fir32")
        assert close(o[1], mirror.stats)
        assert abs(o[0] - mirror.score) < 2e-6
    b.close()
