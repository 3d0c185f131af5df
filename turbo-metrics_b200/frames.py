"""Frame-pair driver: SSIMULACRA2 over two frame sequences with per-frame
scores and summary statistics, as turbo-metrics' `TurboMetrics::compute_all`
does for this metric (crates/turbo-metrics/src/lib.rs:365-437; per-frame
`compute_one` :271-363), with the statistics of quick-stats' `full::Stats`
(crates/quick-stats/src/lib.rs:1-97).

Video decoding (the reference's NVDEC / AMF sources) is not part of this
engine: frames arrive as host arrays (a decoder's output), in any input
format the engine takes.  Frames are scored in submissions of several pairs
through `Ssim2Batch.submit_host`, two submissions in flight, so uploads
overlap the scoring of the previous frames.
"""
from __future__ import annotations

import dataclasses
import itertools
import math

import numpy as np

from .ssimulacra2 import PairDesc, Ssim2Batch


@dataclasses.dataclass
class Stats:
    """quick-stats full::Stats (quick-stats/src/lib.rs:3-19)."""
    min: float
    max: float
    mean: float
    var: float            # population variance
    sample_var: float
    stddev: float
    sample_stddev: float
    p1: float
    p5: float
    p50: float
    p95: float
    p99: float

    @staticmethod
    def compute(values) -> "Stats":
        """lib.rs:21-52: sorted copy, mean as sum / n, variances about the
        mean, percentiles by linear interpolation between ranks."""
        v = [float(x) for x in values]
        if not v:
            raise ValueError("no values")
        s = sorted(v)
        mean = sum(s) / len(v)
        var = _var(v, mean, False)
        sample_var = _var(v, mean, True)
        return Stats(s[0], s[-1], mean, var, sample_var, math.sqrt(var), math.sqrt(sample_var),
                     _percentile(s, 1.0), _percentile(s, 5.0), _percentile(s, 50.0), _percentile(s, 95.0),
                     _percentile(s, 99.0))


def _percentile(sorted_v, pct):
    """lib.rs:56-76: rank = pct / 100 * (n - 1), linear between its neighbours."""
    if len(sorted_v) == 1:
        return sorted_v[0]
    if pct == 100.0:
        return sorted_v[-1]
    rank = pct / 100.0 * (len(sorted_v) - 1)
    lrank = math.floor(rank)
    d = rank - lrank
    n = int(lrank)
    lo, hi = sorted_v[n], sorted_v[n + 1]
    return lo + (hi - lo) * d


def _var(values, mean, sample):
    """lib.rs:78-97: sum of squared deviations over n (population) or n - 1."""
    if len(values) < 2:
        return 0.0
    acc = 0.0
    for x in values:
        acc += (x - mean) * (x - mean)
    return acc / ((len(values) - 1) if sample else len(values))


def select_frames(frames_ref, frames_dis, skip=0, skip_ref=0, skip_dis=0, every=1, frames=0):
    """The frame pairs compute_all scores (lib.rs:385-413): skip `skip_ref +
    skip` reference and `skip_dis + skip` distorted frames, pair the rest in
    order while both sources last, keep the first decoded pair and then every
    `every`-th, stop after `frames` decoded pairs (0 = all)."""
    it_r = itertools.islice(iter(frames_ref), skip_ref + skip, None)
    it_d = itertools.islice(iter(frames_dis), skip_dis + skip, None)
    decode_count = 0
    for fr, fd in zip(it_r, it_d):
        if every > 1 and decode_count != 0 and decode_count % every != 0:
            decode_count += 1
            continue
        if frames > 0 and decode_count >= frames:
            break
        decode_count += 1
        yield fr, fd


class FramePairScorer:
    """SSIMULACRA2 of two frame sequences of one size and format.

    fmt: "nv12" / "p016" (frames are (y, uv) plane tuples), "srgb8",
    "linear_f32" or "rgb16" (frames are (H, W, 3) arrays); matrix / range
    apply to the YUV formats."""

    def __init__(self, width, height, fmt="nv12", matrix="bt709", range="limited", bits=10,
                 frames_per_submission=16, device=0, **batch_kw):
        self.width, self.height = int(width), int(height)
        self.fmt, self.matrix, self.range, self.bits = fmt, matrix, range, bits
        self.k = int(frames_per_submission)
        self.batch = Ssim2Batch(self.k, self.k * self.width * self.height, device=device, **batch_kw)

    def close(self):
        self.batch.close()

    def _desc(self, fr, fd):
        if self.fmt in ("nv12", "p016"):
            (ry, ruv), (dy, duv) = fr, fd
            return PairDesc(_plane(ry), _plane(dy), self.fmt, _plane(ruv), _plane(duv), matrix=self.matrix,
                            range=self.range)
        return PairDesc(_plane(fr), _plane(fd), self.fmt, bits=self.bits)

    def compute_all(self, frames_ref, frames_dis, **opts):
        """Per-frame scores (in frame order) and their Stats
        (None when no frame pair was scored)."""
        scores, in_flight, chunk = [], 0, []
        for fr, fd in select_frames(frames_ref, frames_dis, **opts):
            chunk.append(self._desc(fr, fd))
            if len(chunk) == self.k:
                in_flight = self._submit(chunk, in_flight, scores)
                chunk = []
        if chunk:
            in_flight = self._submit(chunk, in_flight, scores)
        while in_flight:
            scores.extend(r[0] for r in self.batch.results())
            in_flight -= 1
        return scores, (Stats.compute(scores) if scores else None)

    def _submit(self, chunk, in_flight, scores):
        self.batch.submit_host(chunk)
        in_flight += 1
        if in_flight == 2:  # read the older submission while the newer one runs
            scores.extend(r[0] for r in self.batch.results())
            in_flight -= 1
        return in_flight


def _plane(a):
    a = np.ascontiguousarray(a)
    return a.view(np.int16) if a.dtype == np.uint16 else a
