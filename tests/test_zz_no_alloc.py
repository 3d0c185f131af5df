"""GPU test of s2_compute_srgb8_noalloc, the entry point for callers that
cannot allocate device memory (their host framework owns the device memory
pool, or they must not grow the footprint or block on the allocator).

It is called through the C ABI twice in a row, on two different pairs, and
each result is checked against the allocating entry point (s2_compute_srgb8
via Ssimulacra2) within the tolerance of the other parity tests: 2e-6
relative on each of the 108 statistics (1e-12 absolute near zero) and 2e-6 on
the score.  The file is named to be collected last.
"""
import ctypes

import numpy as np
import pytest

import synth

pytestmark = pytest.mark.gpu

REL, ABS, SCORE_TOL = 2e-6, 1e-12, 2e-6


def test_noalloc_matches_allocating_entry_point(tmb, cuda):
    torch = cuda
    lib = tmb.lib
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    size = ctypes.sizeof(tmb.capi.Result)
    # 512x512 and 500x512 sit on the documented bound (width and height at most
    # 512 always fit); 317x200 has an odd width
    for (w, h, seed, step) in [(512, 384, synth.pair_seed(0, 11), 16), (317, 200, synth.pair_seed(0, 12), 8),
                               (512, 512, synth.pair_seed(0, 13), 12), (500, 512, synth.pair_seed(0, 14), 24)]:
        ref, dis = synth.srgb_pair(w, h, seed, step)
        rt = torch.from_numpy(ref).cuda()
        dt = torch.from_numpy(dis).cuda()
        out = torch.zeros(size, dtype=torch.uint8, device="cuda")
        st = lib.s2_compute_srgb8_noalloc(ctypes.c_void_p(rt.data_ptr()), w * 3, ctypes.c_void_p(dt.data_ptr()),
                                          w * 3, w, h, ctypes.c_void_p(out.data_ptr()), stream)
        assert st == 0, tmb.lib.s2_status_string(st)
        torch.cuda.synchronize()
        res = tmb.capi.Result.from_buffer_copy(out.cpu().numpy().tobytes())
        assert res.status == 0
        s = tmb.Ssimulacra2(w, h)
        s.compute_srgb(rt, dt)
        score, stats, _ = s.get_result()
        s.close()
        got = np.array(res.stats[:])
        err = np.abs(got - stats)
        assert np.all(err <= np.maximum(REL * np.abs(stats), ABS)), np.nonzero(err > np.maximum(REL * np.abs(stats), ABS))
        assert abs(res.score - score) < SCORE_TOL, (res.score, score)
        assert res.n_scales == tmb.num_scales(w, h)


def test_noalloc_rejects_pairs_over_its_array(tmb, cuda):
    torch = cuda
    w, h = 8, 32768  # padded rows need ~50 MB, over the 16 MiB array
    buf = torch.zeros((h, w, 3), dtype=torch.uint8, device="cuda")
    out = torch.zeros(ctypes.sizeof(tmb.capi.Result), dtype=torch.uint8, device="cuda")
    st = tmb.lib.s2_compute_srgb8_noalloc(ctypes.c_void_p(buf.data_ptr()), w * 3, ctypes.c_void_p(buf.data_ptr()),
                                          w * 3, w, h, ctypes.c_void_p(out.data_ptr()), None)
    assert st == 2  # S2_ERR_INVALID_SIZE
    # twice the documented bound: 1024x1024 needs about 34 MB
    w = h = 1024
    big = torch.zeros((h, w, 3), dtype=torch.uint8, device="cuda")
    st = tmb.lib.s2_compute_srgb8_noalloc(ctypes.c_void_p(big.data_ptr()), w * 3, ctypes.c_void_p(big.data_ptr()),
                                          w * 3, w, h, ctypes.c_void_p(out.data_ptr()), None)
    assert st == 2
    assert tmb.lib.s2_compute_srgb8_noalloc(None, 0, None, 0, 64, 64, None, None) == 8  # S2_ERR_INVALID_ARG
