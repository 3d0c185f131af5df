"""GPU parity of DSSIM, the sibling metric scored from SSIMULACRA2's pyramid.

The device path (Lab planes written by the shared prep pass, the clamp pass,
the tile / mean / MAD / final kernels) is compared through the C ABI with the
oracle's f32 mirror of dssim-cuda (oracle/dssim_oracle.c): same LUT, same
pyramid, same f32 operations and the same cube root, so the SSIM maps agree
bit for bit and only the order of the f64 sums differs.  Bound:
|d_gpu - d_oracle| <= 1e-10 + 1e-8 * d_oracle, per-scale scores within 1e-10.
The published values of the reference (dssim-gpu PORT_STATUS.md:26-30) are
checked at the reference's own bounds.

Scoring both metrics from one prep pass must not change either: SSIMULACRA2
alone and with DSSIM are bit-identical, and so are DSSIM alone and with
SSIMULACRA2, single pairs and batches of mixed sizes and formats."""
import math

import numpy as np
import pytest

import synth
from test_oracle_dssim import PUB, add_noise, gradient, solid

pytestmark = pytest.mark.gpu

ABS, REL = 1e-10, 1e-8


def close(got, want):
    return abs(got - want) <= ABS + REL * abs(want)


def dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def test_published_cases(tmb, cuda, oracle):
    d = tmb.Dssim(64, 64)
    bw = d.compute_sync(dev(cuda, solid(64, 64, 0)), dev(cuda, solid(64, 64, 255)))
    assert close(bw, oracle.dssim_srgb8(solid(64, 64, 0), solid(64, 64, 255)).dssim)
    for want in PUB["black_white_64"].values():
        assert abs(bw - want) / want < 1e-3
    g = gradient(64, 64)
    ng = add_noise(g, 8)
    nz = d.compute_sync(dev(cuda, g), dev(cuda, ng))
    assert close(nz, oracle.dssim_srgb8(g, ng).dssim)
    for want in PUB["noisy_gradient_64"].values():
        assert abs(nz - want) / want < 1e-2
    d32 = tmb.Dssim(32, 32)
    g32 = dev(cuda, gradient(32, 32))
    assert d32.compute_sync(g32, g32) == 0.0


@pytest.mark.parametrize("w,h", [(8, 8), (16, 16), (37, 53), (123, 45), (200, 150), (9, 300), (700, 14),
                                 (512, 384), (1920, 1080)])
def test_srgb_sizes_match_oracle(tmb, cuda, oracle, w, h):
    """Odd sizes, sizes whose later levels are clamped to 8 (clamp pass), and
    a full frame."""
    r, d = synth.srgb_pair(w, h, 700 + w + h)
    want = oracle.dssim_srgb8(r, d, "cuda32")
    ctx = tmb.Ssimulacra2(w, h)
    ctx.set_metrics("dssim")
    ctx.compute_srgb(dev(cuda, r), dev(cuda, d))
    got, scales = ctx.get_dssim()
    assert close(got, want.dssim), (w, h, got, want.dssim)
    np.testing.assert_allclose(scales, want.level_scores, rtol=0, atol=1e-10)
    f64 = oracle.dssim_srgb8(r, d, "fp64").dssim
    assert abs(got - f64) <= 2e-3 * f64 + 1e-7


def test_both_metrics_share_the_pass_bit_identically(tmb, cuda):
    r, d = synth.srgb_pair(333, 211, 81)
    rt, dt = dev(cuda, r), dev(cuda, d)
    ctx = tmb.Ssimulacra2(333, 211)
    ctx.compute_srgb(rt, dt)
    s2_alone = ctx.get_result()
    ctx.set_metrics(("ssimulacra2", "dssim"))
    ctx.compute_srgb(rt, dt)
    both = ctx.get_result()
    ds_both = ctx.get_dssim()
    ctx.set_metrics("dssim")
    ctx.compute_srgb(rt, dt)
    ds_alone = ctx.get_dssim()
    assert both[0] == s2_alone[0] and np.array_equal(both[1], s2_alone[1])
    assert ds_both[0] == ds_alone[0] and np.array_equal(ds_both[1], ds_alone[1])
    assert math.isnan(ctx.get_score())  # DSSIM only: no SSIMULACRA2 score
    ctx.set_metrics("ssimulacra2")
    ctx.compute_srgb(rt, dt)
    with pytest.raises(tmb.S2Error):
        ctx.get_dssim()


def test_cached_reference_and_errors(tmb, cuda, oracle):
    r, d1 = synth.srgb_pair(96, 80, 3)
    _, d2 = synth.srgb_pair(96, 80, 4)
    ds = tmb.Dssim(96, 80)
    with pytest.raises(tmb.NoCachedReference):
        ds.compute_sync_dis_only(dev(cuda, d1))
    a = ds.compute_sync(dev(cuda, r), dev(cuda, d1))
    b = ds.compute_sync_dis_only(dev(cuda, d2))
    c = ds.compute_sync_dis_only(dev(cuda, d1))
    full = tmb.Dssim(96, 80).compute_sync(dev(cuda, r), dev(cuda, d2))
    assert c == a and b == full
    assert close(b, oracle.dssim_srgb8(r, d2).dssim)
    host = ds.compute_from_cpu_sync(r, d2)
    assert host == full
    assert ds.mem_usage() > 0
    with pytest.raises(tmb.InvalidImageSize):
        tmb.Dssim(7, 64)


def test_nv12_and_linear_inputs(tmb, cuda, oracle):
    (ry, ruv), (dy, duv) = synth.nv12_frame_pair(320, 180, 12)
    ctx = tmb.Ssimulacra2(320, 180)
    ctx.set_metrics("dssim")
    ctx.compute_nv12(dev(cuda, ry), dev(cuda, ruv), dev(cuda, dy), dev(cuda, duv))
    got = ctx.get_dssim()[0]
    rl = oracle.yuv420_to_linear(ry, ruv)
    dl = oracle.yuv420_to_linear(dy, duv)
    assert close(got, oracle.dssim_linear(rl, dl).dssim)
    ctx.compute_linear(dev(cuda, rl), dev(cuda, dl))
    assert close(ctx.get_dssim()[0], oracle.dssim_linear(rl, dl).dssim)


def _mixed(n, seed):
    out = []
    for i in range(n):
        if i % 3 == 1:
            (ry, ruv), (dy, duv) = synth.nv12_frame_pair(96 + 32 * i, 64 + 16 * i, seed + i)
            out.append(("nv12", ry, dy, ruv, duv))
        else:
            r, d = synth.srgb_pair(40 + 61 * i, 20 + 37 * i, seed + i)
            out.append(("srgb8", r, d))
    return out


def _desc(tmb, torch, p, host=False):
    conv = (lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory()) if host else (lambda a: dev(torch, a))
    if p[0] == "nv12":
        _, ry, dy, ruv, duv = p
        return tmb.PairDesc(conv(ry), conv(dy), "nv12", conv(ruv), conv(duv))
    return tmb.PairDesc(conv(p[1]), conv(p[2]), "srgb8")


def test_batch_matches_single_pairs_and_metric_sets(tmb, cuda):
    pairs = _mixed(10, 4400)
    # an undersized pair: its result says so, the others run
    small = synth.srgb_pair(7, 30, 1)
    pairs.insert(3, ("srgb8",) + small)
    descs = [_desc(tmb, cuda, p) for p in pairs]
    b = tmb.Ssim2Batch(16, 4 << 20)
    s2_only = b.compute_batch(descs)
    b.set_metrics(("ssimulacra2", "dssim"))
    both = b.compute_batch(descs)
    b.set_metrics("dssim")
    ds_only = b.compute_batch(descs)
    for i, p in enumerate(pairs):
        if i == 3:
            assert both[i][4] == ds_only[i][4] == 2  # S2_ERR_INVALID_SIZE
            continue
        assert both[i][0] == s2_only[i][0] and math.isnan(s2_only[i][5])
        assert both[i][5] == ds_only[i][5] and np.array_equal(both[i][6], ds_only[i][6])
        assert math.isnan(ds_only[i][0])
        # a pair's DSSIM does not depend on its batch
        w = p[1].shape[1]
        h = p[1].shape[0]
        ctx = tmb.Ssimulacra2(w, h)
        ctx.set_metrics("dssim")
        d = descs[i]
        if p[0] == "nv12":
            ctx.compute_nv12(d.ref, d.ref_uv, d.dis, d.dis_uv)
        else:
            ctx.compute_srgb(d.ref, d.dis)
        assert ctx.get_dssim()[0] == both[i][5], (i, p[0], w, h)


def test_host_batch_with_dssim(tmb, cuda):
    pairs = _mixed(12, 4600)
    b = tmb.Ssim2Batch(16, 8 << 20)
    b.set_metrics(("ssimulacra2", "dssim"))
    want = b.compute_batch([_desc(tmb, cuda, p) for p in pairs])
    b.submit_host([_desc(tmb, cuda, p, host=True) for p in pairs])
    got = b.results()
    assert [g[0] for g in got] == [w[0] for w in want]
    assert [g[5] for g in got] == [w[5] for w in want]
