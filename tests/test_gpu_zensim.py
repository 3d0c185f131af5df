"""GPU zensim features (s2_zensim_*, tmb.Zensim) against the oracle's
restatement (oracle/zensim_oracle.c).  Every per-pixel value is the same f32
arithmetic on both sides, so the maxima are equal and the 17 f64 sums per
(scale, channel) differ only by their summation order; the 228 features are
checked within 1e-9 relative.  Parity with zensim itself is unpinned: no
published features or weights exist in the reference tree."""
import numpy as np
import pytest

import synth

pytestmark = pytest.mark.gpu


def dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("w,h,seed,step", [(200, 150, 71, 8), (64, 48, 72, 24), (333, 217, 73, 4),
                                           (517, 300, 74, 12), (15, 15, 75, 16)])
def test_zensim_matches_oracle(tmb, oracle, cuda, w, h, seed, step):
    ref, dis = synth.srgb_pair(w, h, seed, step)
    z = tmb.Zensim(w, h)
    feat = z.compute_features(dev(cuda, ref), dev(cuda, dis))
    acc, peaks = z.raw()
    want = oracle.zensim_features_srgb8(ref, dis)
    ns = want.n_scales
    assert z.n_scales == ns
    assert np.array_equal(peaks[:ns], want.peaks[:ns])
    np.testing.assert_allclose(acc[:ns], want.acc[:ns], rtol=1e-9, atol=1e-12)
    np.testing.assert_allclose(feat, want.features, rtol=1e-9, atol=1e-12)
    z.close()


def test_zensim_1080p(tmb, oracle, cuda):
    ref, dis = synth.srgb_pair(1920, 1080, 76, 10)
    z = tmb.Zensim(1920, 1080)
    feat = z.compute_features(ref, dis, on_host=True)
    want = oracle.zensim_features_srgb8(ref, dis)
    np.testing.assert_allclose(feat, want.features, rtol=1e-9, atol=1e-12)
    z.close()


def test_zensim_cached_reference(tmb, oracle, cuda):
    """set_reference once, then several candidates (Zensim::compute_with_reference)."""
    w, h = 160, 120
    ref, _ = synth.srgb_pair(w, h, 77)
    z = tmb.Zensim(w, h)
    assert not z.has_reference()
    with pytest.raises(tmb.NoCachedReference):
        z.compute_with_reference(dev(cuda, ref))
    z.set_reference(dev(cuda, ref))
    assert z.has_reference()
    for step in (2.0, 12.0, 40.0):
        _, dis = synth.srgb_pair(w, h, 77, step)
        got = z.compute_with_reference(dev(cuda, dis))
        np.testing.assert_allclose(got, oracle.zensim_features_srgb8(ref, dis).features, rtol=1e-9, atol=1e-12)
    # the same candidate twice gives the same features (fixed-order sums)
    a = z.compute_with_reference(dev(cuda, dis))
    b = z.compute_with_reference(dev(cuda, dis))
    assert np.array_equal(a, b)
    z.clear_reference()
    assert not z.has_reference()
    z.close()


def test_zensim_errors(tmb, cuda):
    with pytest.raises(tmb.InvalidImageSize):
        tmb.Zensim(7, 64)
    z = tmb.Zensim(64, 64)
    img = cuda.zeros((64, 65, 3), dtype=cuda.uint8, device="cuda")
    assert z.mem_usage() > 0
    z.close()
