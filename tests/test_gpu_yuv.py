"""The 4:2:0 YUV input family (cuda-colorspace/src/lib.rs:33-131): NV12
(8-bit) and P016 (16-bit samples) biplanar frames, BT.709 / BT.601-525 /
BT.601-625 matrices, limited and full range, converted inside the prep pass.

Each case runs through the C ABI and is checked against the oracle's
restatement of the same conversion (`fir32`, 2e-5 relative per statistic:
the power function's last ulp differs between the engine and glibc) and the
FP64 oracle (1e-3).  Parity with the reference itself is unpinned for these
inputs: its colour-space test has no assertions (cuda-colorspace/src/
kernel.rs:402-449) and full range is todo!() there."""
import numpy as np
import pytest

import synth

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-3


def dev(torch, a):
    if a.dtype == np.uint16:
        a = a.view(np.int16)
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def assert_close(got, want, rel=2e-5, abs_=1e-10):
    got, want = np.asarray(got), np.asarray(want)
    bad = np.abs(got - want) > np.maximum(rel * np.abs(want), abs_)
    assert not bad.any(), (np.nonzero(bad)[0][:8], got[bad][:8], want[bad][:8])


def check_pair(tmb, oracle, cuda, fmt, ref, dis, matrix, rng):
    (ry, ruv), (dy, duv) = ref, dis
    h, w = ry.shape
    s = tmb.Ssimulacra2(w, h)
    fn = s.compute_nv12 if fmt == "nv12" else s.compute_p016
    fn(dev(cuda, ry), dev(cuda, ruv), dev(cuda, dy), dev(cuda, duv), matrix=matrix, range=rng)
    score, stats, _ = s.get_result()
    full = rng == "full"
    rl = oracle.yuv420_to_linear(ry, ruv, matrix, full)
    dl = oracle.yuv420_to_linear(dy, duv, matrix, full)
    mirror = oracle.ssim2_linear(rl, dl, "fir32")
    assert_close(stats, mirror.stats)
    assert abs(score - mirror.score) < 2e-5
    exact = oracle.ssim2_linear(oracle.yuv420_to_linear(ry, ruv, matrix, full, True),
                                oracle.yuv420_to_linear(dy, duv, matrix, full, True), "fp64")
    assert abs(score - exact.score) < FP64_TOL
    return score


@pytest.mark.parametrize("matrix", ["bt709", "bt601_525", "bt601_625"])
@pytest.mark.parametrize("rng", ["limited", "full"])
def test_nv12_matrices_and_ranges(tmb, oracle, cuda, matrix, rng):
    ref, dis = synth.nv12_frame_pair(320, 184, 1200)
    check_pair(tmb, oracle, cuda, "nv12", ref, dis, matrix, rng)


@pytest.mark.parametrize("matrix,rng", [("bt709", "limited"), ("bt601_625", "limited"), ("bt601_525", "full")])
def test_p016_matches_oracle(tmb, oracle, cuda, matrix, rng):
    ref, dis = synth.p016_frame_pair(256, 144, 1300, bits=10)
    check_pair(tmb, oracle, cuda, "p016", ref, dis, matrix, rng)


def test_p016_of_shifted_nv12_equals_nv12(tmb, cuda):
    """16-bit samples holding 8-bit values << 8 give the 8-bit result exactly
    (the coefficients scale by the same power of two)."""
    (ry, ruv), (dy, duv) = synth.nv12_frame_pair(192, 108, 1400)
    w16 = lambda a: a.astype(np.uint16) << 8
    s = tmb.Ssimulacra2(192, 108)
    s.compute_nv12(dev(cuda, ry), dev(cuda, ruv), dev(cuda, dy), dev(cuda, duv), matrix="bt601_525")
    a = s.get_score()
    s.compute_p016(dev(cuda, w16(ry)), dev(cuda, w16(ruv)), dev(cuda, w16(dy)), dev(cuda, w16(duv)),
                   matrix="bt601_525")
    assert s.get_score() == a


def test_mixed_yuv_batch_equals_single_and_host(tmb, cuda):
    cases = [("nv12", synth.nv12_frame_pair(256, 144, 1500), "bt709", "limited"),
             ("p016", synth.p016_frame_pair(320, 180, 1501), "bt601_625", "limited"),
             ("nv12", synth.nv12_frame_pair(128, 96, 1502), "bt601_525", "full"),
             ("p016", synth.p016_frame_pair(200, 150, 1503, bits=12), "bt709", "full")]
    descs, hdescs, singles = [], [], []
    for fmt, ((ry, ruv), (dy, duv)), m, r in cases:
        descs.append(tmb.PairDesc(dev(cuda, ry), dev(cuda, dy), fmt, dev(cuda, ruv), dev(cuda, duv), matrix=m, range=r))
        hdescs.append(tmb.PairDesc(ry.view(np.int16) if ry.dtype == np.uint16 else ry,
                                   dy.view(np.int16) if dy.dtype == np.uint16 else dy, fmt,
                                   ruv.view(np.int16) if ruv.dtype == np.uint16 else ruv,
                                   duv.view(np.int16) if duv.dtype == np.uint16 else duv, matrix=m, range=r))
        h, w = ry.shape
        s = tmb.Ssimulacra2(w, h)
        fn = s.compute_nv12 if fmt == "nv12" else s.compute_p016
        fn(dev(cuda, ry), dev(cuda, ruv), dev(cuda, dy), dev(cuda, duv), matrix=m, range=r)
        singles.append(s.get_score())
    b = tmb.Ssim2Batch(8, 1 << 20)
    got = [x[0] for x in b.compute_batch(descs)]
    assert all(abs(g - s_) < 1e-12 for g, s_ in zip(got, singles)), (got, singles)
    b.submit_host(hdescs)
    assert [x[0] for x in b.results()] == got


def test_yuv_argument_errors(tmb, cuda):
    (ry, ruv), (dy, duv) = synth.nv12_frame_pair(64, 64, 1600)
    s = tmb.Ssimulacra2(64, 64)
    args = (dev(cuda, ry), dev(cuda, ruv), dev(cuda, dy), dev(cuda, duv))
    with pytest.raises(KeyError):
        s.compute_nv12(*args, matrix="bt2020")
    import ctypes
    r = tmb.lib.s2_compute_nv12(s._h, ctypes.c_void_p(args[0].data_ptr()), ctypes.c_void_p(args[1].data_ptr()), 64,
                                ctypes.c_void_p(args[2].data_ptr()), ctypes.c_void_p(args[3].data_ptr()), 64, 7, 0, 0,
                                None)
    assert r == 8  # S2_ERR_INVALID_ARG
