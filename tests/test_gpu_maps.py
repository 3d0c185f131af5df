"""Error-map export: the maps a compute pooled, written out per scale.  Pooled
again on the host (mean and fourth-power mean, f64), they give back the
compute's 108 statistics (stat c*36 + scale*6 + norm*3 + map)."""
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
