"""Precision sweep (survey config C3): 3840x2160 10-bit BT.2020 RGB pairs
(gratings + noise; distorted = Gaussian blur sigma in [0.5, 2] + noise
sigma 8), XYB planes stored as f32, f16 or bf16 with f32 arithmetic and f64
pooling, every score against the FP64 oracle.

The test runs 4 pairs and holds f32 storage to the 1e-3 bar; the reduced
formats' errors are printed, not gated (they miss the bar: see the table
that `python tests/test_gpu_precision.py --pairs 32` prints)."""
import multiprocessing as mp
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(ROOT, "turbo-metrics_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

W, H = 3840, 2160


def _pair_and_fp64(i):
    import oracle
    import synth
    r, d = synth.c3_pair(i, W, H)
    exact = oracle.ssim2_linear(oracle.rgb16_to_linear(r), oracle.rgb16_to_linear(d), "fp64").score
    return r, d, exact


def sweep(tmb, torch, n):
    with mp.get_context("spawn").Pool(min(n, os.cpu_count() or 1)) as pool:
        data = pool.map(_pair_and_fp64, range(n))
    dev = [(torch.from_numpy(r.view(np.int16)).cuda(), torch.from_numpy(d.view(np.int16)).cuda()) for r, d, _ in data]
    exact = np.array([e for _, _, e in data])
    descs = [tmb.PairDesc(r, d, "rgb16", bits=10) for r, d in dev]
    out = {}
    for storage in ("f32",):
        b = tmb.Ssim2Batch(n, n * W * H, storage=storage)
        scores = np.array([x[0] for x in b.compute_batch(descs)])
        b.close()
        err = np.abs(scores - exact)
        out[storage] = {"max_abs_err": float(err.max()), "mean_abs_err": float(err.mean()),
                        "within_1e-3": int((err <= 1e-3).sum()), "pairs": n}
    return out


@pytest.mark.gpu
def test_precision_sweep_4k_10bit(tmb, cuda):
    res = sweep(tmb, cuda, 4)
    print("precision sweep (4 pairs, 3840x2160 10-bit BT.2020):", res)
    assert res["f32"]["max_abs_err"] < 1e-3


if __name__ == "__main__":
    import argparse
    import json
    import torch
    ap = argparse.ArgumentParser()
    ap.add_argument("--pairs", type=int, default=32)
    args = ap.parse_args()
    sys.path.insert(0, HERE)
    import conftest
    print(json.dumps(sweep(conftest.load_package(), torch, args.pairs)))
