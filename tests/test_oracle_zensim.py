"""CPU checks of the oracle's zensim restatement (oracle/zensim_oracle.c):
the SIMD-padded width rule and the scale-count rule of crates/zensim-cuda
(src/lib.rs:58-66, :222-233), the feature layout (lib.rs:686-819), and the
behaviour on identical images.  No zensim features are published in the
reference tree, so these pin the restatement's structure, not its values."""
import numpy as np
import pytest

import synth


@pytest.mark.parametrize("w,pw", [(8, 16), (200, 208), (496, 496), (500, 528), (512, 528), (527, 528), (529, 560), (545, 560), (561, 592), (1920, 1936),
                                  (3840, 3856), (1000, 1008)])
def test_simd_padded_width(oracle, w, pw):
    # aligned to 16; +16 when the aligned width is >= 512 and aligned / 16 is even
    assert oracle.zensim_padded_width(w) == pw


@pytest.mark.parametrize("w,h,ns", [(8, 8, 1), (15, 15, 2), (16, 16, 2), (31, 40, 3), (64, 64, 4), (200, 150, 4)])
def test_scale_count(oracle, w, h, ns):
    ref, dis = synth.srgb_pair(w, h, 3, 8)
    assert oracle.zensim_features_srgb8(ref, dis).n_scales == ns


def test_identical_images(oracle):
    ref, _ = synth.srgb_pair(96, 80, 4)
    r = oracle.zensim_features_srgb8(ref, ref)
    acc = r.acc[: r.n_scales]
    # no edge, MSE or high-frequency difference; the SSIM term only keeps
    # zensim's f32 cancellation (sigma terms of separately blurred squares)
    assert np.all(acc[:, :, 3:10] == 0) and np.all(acc[:, :, 15:17] == 0)
    assert np.all(acc[:, :, 10] == acc[:, :, 11]) and np.all(acc[:, :, 12] == acc[:, :, 13])
    assert np.max(r.features[: r.n_scales * 39].reshape(-1, 13)[:, 0]) < 1e-3


def test_feature_layout(oracle):
    ref, dis = synth.srgb_pair(40, 24, 5, 16)
    r = oracle.zensim_features_srgb8(ref, dis)
    assert r.n_scales == 2
    f = r.features
    # basic block: n_scales * 3 * 13, then peaks n_scales * 3 * 6, zeros after
    assert np.all(f[2 * 39 + 2 * 18:] == 0)
    n0 = oracle.zensim_padded_width(40) * 24
    assert f[0] == pytest.approx(abs(r.acc[0, 0, 0]) / n0)
    assert f[2 * 39] == pytest.approx(float(r.peaks[0, 0, 0]))
    assert f[2 * 39 + 3] == pytest.approx((r.acc[0, 0, 14] / n0) ** 0.125)
    # HF ratios: energy loss / gain are complementary around 1
    l2 = r.acc[0, 1, 11] / r.acc[0, 1, 10]
    assert f[13 + 10] == pytest.approx(max(1 - l2, 0)) and f[13 + 12] == pytest.approx(max(l2 - 1, 0))


def test_too_small(oracle):
    ref, dis = synth.srgb_pair(7, 9, 1)
    with pytest.raises(ValueError):
        oracle.zensim_features_srgb8(ref, dis)
