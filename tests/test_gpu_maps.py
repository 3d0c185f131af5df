"""Error-map export: the maps a compute pooled, written out per scale.  Each
map is compared pixel by pixel with the oracle's fir32 maps of the same
scale, and pooled again on the host (mean and fourth-power mean, f64) it
gives back the compute's 108 statistics (stat c*36 + scale*6 + norm*3 +
map)."""
import numpy as np
import pytest

import synth

pytestmark = pytest.mark.gpu


def test_exported_maps_pool_to_the_statistics(tmb, cuda):
    ref, dis = synth.srgb_pair(301, 203, 1900)
    s = tmb.Ssimulacra2(301, 203)
    s.compute_srgb(cuda.from_numpy(ref).cuda(), cuda.from_numpy(dis).cuda())
    score, stats, _ = s.get_result()
    n = tmb.num_scales(301, 203)
    for sc in range(n):
        m = s.error_maps(sc).double().cpu().numpy()  # (3, 3, h, w)
        assert m.min() >= 0.0
        for c in range(3):
            for k in range(3):
                l1 = m[c, k].mean()
                l4 = np.mean(m[c, k] ** 4) ** 0.25
                for got, want in ((l1, stats[c * 36 + sc * 6 + k]), (l4, stats[c * 36 + sc * 6 + 3 + k])):
                    assert abs(got - want) <= 1e-5 * abs(want) + 1e-9, (sc, c, k, got, want)
    # the export leaves the compute's result as it was
    assert s.get_result()[0] == score


@pytest.mark.parametrize("w,h,seed", [(301, 203, 1902), (250, 130, 1903)])
def test_exported_maps_match_oracle_maps(tmb, oracle, cuda, w, h, seed):
    """Element by element against the oracle's restatement
    (oracle.ssim2_maps_fir32): the two compute every value with the same f32
    operations except the division, whose results agree except in rare
    near-halfway cases (a difference of 1 ulp there)."""
    ref, dis = synth.srgb_pair(w, h, seed, 12)
    s = tmb.Ssimulacra2(w, h)
    s.compute_srgb(cuda.from_numpy(ref).cuda(), cuda.from_numpy(dis).cuda())
    s.get_score()
    rl, dl = oracle.srgb8_to_linear(ref), oracle.srgb8_to_linear(dis)
    for sc in range(tmb.num_scales(w, h)):
        got = s.error_maps(sc).cpu().numpy()  # (3, 3, h_s, w_s) float32
        want = oracle.ssim2_maps_fir32(rl, dl, sc)
        assert got.shape == want.shape
        ulp = np.spacing(np.maximum(np.abs(want), np.float32(1e-30)).astype(np.float32))
        diff = np.abs(got.astype(np.float64) - want.astype(np.float64))
        assert np.all(diff <= 2 * ulp + 1e-30), (sc, float((diff / ulp).max()))
        assert np.mean(got == want) > 0.999, (sc, float(np.mean(got == want)))


def test_error_maps_preconditions(tmb, cuda):
    s = tmb.Ssimulacra2(64, 64)
    with pytest.raises(tmb.S2Error):
        s.error_maps(0)  # no compute yet
    ref, dis = synth.srgb_pair(64, 64, 1901)
    s.compute_srgb(cuda.from_numpy(ref).cuda(), cuda.from_numpy(dis).cuda())
    s.get_score()
    with pytest.raises(tmb.S2Error):
        s.error_maps(tmb.num_scales(64, 64))  # no such scale
    t = tmb.Ssimulacra2(64, 64, blur="iir_ref")
    t.compute_srgb(cuda.from_numpy(ref).cuda(), cuda.from_numpy(dis).cuda())
    t.get_score()
    with pytest.raises(tmb.S2Error):
        t.error_maps(0)
