"""GPU tests of s2_batch_submit_host: batches whose planes are in host memory,
uploaded in groups on the batch's copy stream while earlier groups compute.

The arithmetic is the device-input batch's (same kernels, same per-pair tile
order), so the scores must be bit-identical to s2_batch_submit on the same
images, for every format, uneven sizes, padded host rows, pinned and pageable
memory, and back-to-back submissions that reuse the staging."""
import numpy as np
import pytest

import synth

pytestmark = pytest.mark.gpu


def dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def padded(a, extra):
    """The same image inside wider host rows (pitch > row bytes)."""
    h, w = a.shape[:2]
    big = np.zeros((h, w + extra) + a.shape[2:], a.dtype)
    big[:, :w] = a
    return big[:, :w]


def make_pairs(n, seed0):
    """Mixed formats and sizes: (format, host arrays...) per pair."""
    out = []
    for i in range(n):
        k = i % 4
        if k == 0:
            r, d = synth.srgb_pair(96 + 37 * i, 64 + 23 * i, seed0 + i)
            out.append(("srgb8", r, d))
        elif k == 1:
            (ry, ruv), (dy, duv) = synth.nv12_frame_pair(128 + 16 * i, 72 + 8 * i, seed0 + i)
            out.append(("nv12", ry, dy, ruv, duv))
        elif k == 2:
            r, d = synth.rgb10_pair(80 + 11 * i, 90 + 5 * i, seed0 + i)
            out.append(("rgb16", r, d))
        else:
            r, d = synth.srgb_pair(60 + 9 * i, 200 - 3 * i, seed0 + i, 6.0)
            out.append(("srgb8", padded(r, 13), padded(d, 5)))
    return out


def device_desc(tmb, torch, p):
    fmt = p[0]
    if fmt == "nv12":
        _, ry, dy, ruv, duv = p
        return tmb.PairDesc(dev(torch, ry), dev(torch, dy), "nv12", dev(torch, ruv), dev(torch, duv))
    _, r, d = p
    if fmt == "rgb16":
        return tmb.PairDesc(dev(torch, r.view(np.int16)), dev(torch, d.view(np.int16)), "rgb16", bits=10)
    return tmb.PairDesc(dev(torch, r), dev(torch, d), fmt)


def host_desc(tmb, torch, p, pinned):
    fmt = p[0]
    conv = (lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory()) if pinned else (lambda a: a)
    if fmt == "nv12":
        _, ry, dy, ruv, duv = p
        return tmb.PairDesc(conv(ry), conv(dy), "nv12", conv(ruv), conv(duv))
    _, r, d = p
    if fmt == "rgb16":
        if pinned:
            return tmb.PairDesc(conv(r.view(np.int16)), conv(d.view(np.int16)), "rgb16", bits=10)
        return tmb.PairDesc(r, d, "rgb16", bits=10)
    if pinned:
        return tmb.PairDesc(conv(r), conv(d), fmt)
    return tmb.PairDesc(r, d, fmt)  # numpy, padded rows kept as a strided view


@pytest.mark.parametrize("pinned", [True, False])
def test_host_batch_equals_device_batch(tmb, cuda, pinned):
    pairs = make_pairs(22, 9100)
    dd = [device_desc(tmb, cuda, p) for p in pairs]
    hd = [host_desc(tmb, cuda, p, pinned) for p in pairs]
    b = tmb.Ssim2Batch(32, 8 << 20)
    want = b.compute_batch(dd)
    b.submit_host(hd)
    got = b.results()
    for i, (g, w) in enumerate(zip(got, want)):
        assert g[4] == w[4] == 0, (i, g[4], w[4])
        assert g[0] == w[0], (i, pairs[i][0], g[0], w[0])
        assert np.array_equal(g[1], w[1])


def test_host_batch_back_to_back_and_invalid_pairs(tmb, cuda):
    b = tmb.Ssim2Batch(32, 8 << 20)
    dev_b = tmb.Ssim2Batch(32, 8 << 20)
    for rnd in range(3):
        pairs = make_pairs(9 + 5 * rnd, 9300 + 100 * rnd)
        # an undersized pair in the middle: its result says so, the rest run
        small = synth.srgb_pair(7, 50, 77)
        pairs.insert(4, ("srgb8",) + small)
        dd = [device_desc(tmb, cuda, p) for p in pairs]
        hd = [host_desc(tmb, cuda, p, rnd != 1) for p in pairs]
        want = dev_b.compute_batch(dd)
        b.submit_host(hd)
        got = b.results()
        assert got[4][4] == want[4][4] == 2  # S2_ERR_INVALID_SIZE
        assert [g[0] for g in got] == [w[0] for w in want]


def test_host_batch_rejects_short_pitch(tmb, cuda):
    r, d = synth.srgb_pair(64, 64, 5)
    b = tmb.Ssim2Batch(4, 1 << 20)
    short = np.lib.stride_tricks.as_strided(r, shape=r.shape, strides=(64 * 3 - 3, 3, 1))
    with pytest.raises(tmb.DimensionMismatch):
        b.submit_host([tmb.PairDesc(short, d, "srgb8")])


def test_two_host_submissions_in_flight(tmb, cuda):
    """Submission k+1 enqueued before k's results are read (the uploads and
    preps of k+1 overlap k's tile pass): results come back oldest first and
    equal the device-input batch's; a third submission with both slots
    pending drops the oldest one's results."""
    a = make_pairs(9, 9500)
    b = make_pairs(6, 9600)
    c = make_pairs(4, 9700)
    dev_b = tmb.Ssim2Batch(32, 8 << 20)
    want = [dev_b.compute_batch([device_desc(tmb, cuda, p) for p in x]) for x in (a, b, c)]
    bt = tmb.Ssim2Batch(32, 8 << 20)
    ha, hb, hc = ([host_desc(tmb, cuda, p, True) for p in x] for x in (a, b, c))
    bt.submit_host(ha)
    bt.submit_host(hb)
    got_a = bt.results()
    bt.submit_host(hc)
    got_b = bt.results()
    got_c = bt.results()
    for got, w in ((got_a, want[0]), (got_b, want[1]), (got_c, want[2])):
        assert [g[0] for g in got] == [x[0] for x in w]
    # three in flight: the first one's results are dropped, the other two come back in order
    bt.submit_host(ha)
    bt.submit_host(hb)
    bt.submit_host(hc)
    assert [g[0] for g in bt.results()] == [x[0] for x in want[1]]
    assert [g[0] for g in bt.results()] == [x[0] for x in want[2]]
