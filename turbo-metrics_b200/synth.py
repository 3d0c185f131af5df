"""Seeded synthetic image pairs for the five SSIMULACRA2 workloads.

The reference measures on real images and video; no dataset travels with this
repository, so every workload is generated here, deterministically, with the
shapes, bit depths and distortion types of the reference's benchmark configs:

  C0  one 512x512 sRGB8 pair: 8 random gratings per channel + uniform noise;
      distorted = + N(0, 4^2), then 8x8 block-DCT quantisation with step 16.
  C1  1920x1080 NV12 (BT.709 limited range) frame pairs: a smooth luma
      gradient + band-limited noise, chroma noise around 128; distorted =
      8x8 DCT quantisation of Y, U and V with a step from {4, 8, 16, 32}.
  C2  uneven sRGB8 pairs, width and height each uniform in [64, 2048].
  C3  3840x2160 10-bit BT.2020 RGB (uint16): gratings + noise; distorted =
      separable Gaussian blur (sigma in [0.5, 2]) + N(0, 8^2).
  C4  serving jobs: Poisson arrivals, log-uniform sizes 128^2..3840x2160,
      1..16 candidates per reference with a DCT step in [2, 48].

Randomness is a counter-based splitmix64 stream: element i of the stream
seeded s is splitmix64(s + (i + 1) * golden), so any slice can be drawn
without drawing what precedes it.  Per-pair seeds are
0x55AA0000 + config * 1_000_000 + pair_index.
"""
from __future__ import annotations

import math

import numpy as np

_GOLDEN = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def pair_seed(config: int, index: int) -> int:
    return 0x55AA0000 + config * 1_000_000 + index


class Stream:
    """Counter-based splitmix64 stream; `take(n)` returns the next n draws."""

    def __init__(self, seed: int):
        self.seed = np.uint64(seed & 0xFFFFFFFFFFFFFFFF)
        self.pos = 0

    def _u64(self, n: int) -> np.ndarray:
        idx = np.arange(self.pos + 1, self.pos + 1 + n, dtype=np.uint64)
        self.pos += n
        with np.errstate(over="ignore"):
            z = self.seed + idx * _GOLDEN
            z = (z ^ (z >> np.uint64(30))) * _M1
            z = (z ^ (z >> np.uint64(27))) * _M2
            z = z ^ (z >> np.uint64(31))
        return z

    def uniform(self, n: int, lo: float = 0.0, hi: float = 1.0) -> np.ndarray:
        u = (self._u64(n) >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)
        return lo + (hi - lo) * u

    def normal(self, n: int) -> np.ndarray:
        m = (n + 1) // 2
        u1 = self.uniform(m)
        u2 = self.uniform(m)
        r = np.sqrt(-2.0 * np.log(1.0 - u1))
        z = np.concatenate([r * np.cos(2 * math.pi * u2), r * np.sin(2 * math.pi * u2)])
        return z[:n]

    def scalar(self, lo: float = 0.0, hi: float = 1.0) -> float:
        return float(self.uniform(1, lo, hi)[0])

    def randint(self, lo: int, hi: int) -> int:
        """Uniform integer in [lo, hi]."""
        return lo + min(int(self.scalar() * (hi - lo + 1)), hi - lo)


# --------------------------------------------------------------------------
# building blocks
# --------------------------------------------------------------------------

def _dct_matrix() -> np.ndarray:
    k = np.arange(8)[:, None]
    n = np.arange(8)[None, :]
    d = np.sqrt(2.0 / 8.0) * np.cos(np.pi * (2 * n + 1) * k / 16.0)
    d[0, :] = np.sqrt(1.0 / 8.0)
    return d


_DCT = _dct_matrix()


def dct_quantize(plane: np.ndarray, step: float, centre: float, lo: float, hi: float) -> np.ndarray:
    """8x8 orthonormal DCT-II of (v - centre) with edge-replicated padding to a
    multiple of 8, coefficients rounded to multiples of `step`, inverse DCT,
    + centre, rounded and clamped to [lo, hi], cropped back."""
    h, w = plane.shape
    ph, pw = (-h) % 8, (-w) % 8
    p = np.pad(plane.astype(np.float64) - centre, ((0, ph), (0, pw)), mode="edge")
    H, W = p.shape
    blocks = p.reshape(H // 8, 8, W // 8, 8).transpose(0, 2, 1, 3)
    coef = np.einsum("ij,abjk,lk->abil", _DCT, blocks, _DCT, optimize=True)
    coef = np.round(coef / step) * step
    rec = np.einsum("ji,abjk,kl->abil", _DCT, coef, _DCT, optimize=True)
    out = rec.transpose(0, 2, 1, 3).reshape(H, W)[:h, :w] + centre
    return np.clip(np.round(out), lo, hi)


def gaussian_filter(plane: np.ndarray, sigma: float) -> np.ndarray:
    """Separable sampled Gaussian, radius ceil(3 sigma), reflect borders."""
    r = int(math.ceil(3.0 * sigma))
    x = np.arange(-r, r + 1, dtype=np.float64)
    k = np.exp(-0.5 * (x / sigma) ** 2)
    k /= k.sum()
    p = np.pad(plane.astype(np.float64), ((r, r), (0, 0)), mode="reflect")
    v = sum(k[i] * p[i:i + plane.shape[0], :] for i in range(2 * r + 1))
    p = np.pad(v, ((0, 0), (r, r)), mode="reflect")
    return sum(k[i] * p[:, i:i + plane.shape[1]] for i in range(2 * r + 1))


def gratings(st: Stream, w: int, h: int, centre: float, amp: float, noise: float,
             hi: float) -> np.ndarray:
    """Per channel: centre + sum of 8 gratings (orientation U[0,pi), period
    U[4,64] px, phase U[0,2pi), amplitude `amp`) + U[-noise, noise]; clamped
    to [0, hi] and rounded.  Returns (h, w, 3) float64."""
    yy, xx = np.mgrid[0:h, 0:w].astype(np.float64)
    out = np.empty((h, w, 3))
    for c in range(3):
        acc = np.full((h, w), centre)
        for _ in range(8):
            th = st.scalar(0.0, math.pi)
            per = st.scalar(4.0, 64.0)
            ph = st.scalar(0.0, 2 * math.pi)
            acc += amp * np.sin(2 * math.pi * (xx * math.cos(th) + yy * math.sin(th)) / per + ph)
        acc += st.uniform(h * w, -noise, noise).reshape(h, w)
        out[:, :, c] = acc
    return np.clip(np.round(out), 0, hi)


# --------------------------------------------------------------------------
# workloads
# --------------------------------------------------------------------------

def srgb_pair(w: int, h: int, seed: int, step: float = 16.0):
    """C0-style pair: (ref, dis), each (h, w, 3) uint8."""
    st = Stream(seed)
    ref = gratings(st, w, h, 128.0, 12.0, 16.0, 255.0)
    dis = np.clip(ref + 4.0 * st.normal(h * w * 3).reshape(h, w, 3), 0, 255)
    for c in range(3):
        dis[:, :, c] = dct_quantize(dis[:, :, c], step, 128.0, 0.0, 255.0)
    return ref.astype(np.uint8), dis.astype(np.uint8)


def c0_pair():
    return srgb_pair(512, 512, pair_seed(0, 0))


def _band_noise(st: Stream, w: int, h: int, sigma: float, amp: float) -> np.ndarray:
    n = gaussian_filter(st.normal(w * h).reshape(h, w), sigma)
    return n * (amp / max(np.abs(n).max(), 1e-12))


def nv12_frame_pair(w: int, h: int, seed: int):
    """C1-style pair of NV12 frames.  Returns (ref, dis), each a (y, uv) tuple:
    y (h, w) uint8, uv (h/2, w) uint8 interleaved Cb,Cr."""
    st = Stream(seed)
    phi = st.scalar(0.0, 2 * math.pi)
    yy, xx = np.mgrid[0:h, 0:w].astype(np.float64)
    g = xx * math.cos(phi) + yy * math.sin(phi)
    g = (g - g.min()) / max(g.max() - g.min(), 1e-12)
    Y = 16.0 + 219.0 * (0.25 + 0.5 * g) + _band_noise(st, w, h, 3.0, 20.0)
    Y = np.clip(np.round(Y), 16, 235)
    cw, ch = w // 2, h // 2
    U = np.clip(np.round(128.0 + _band_noise(st, cw, ch, 3.0, 20.0)), 16, 240)
    V = np.clip(np.round(128.0 + _band_noise(st, cw, ch, 3.0, 20.0)), 16, 240)
    step = [4.0, 8.0, 16.0, 32.0][min(int(st.scalar() * 4), 3)]
    Yd = dct_quantize(Y, step, 128.0, 16.0, 235.0)
    Ud = dct_quantize(U, step, 128.0, 16.0, 240.0)
    Vd = dct_quantize(V, step, 128.0, 16.0, 240.0)

    def pack(y, u, v):
        uv = np.empty((ch, cw * 2), dtype=np.uint8)
        uv[:, 0::2] = u
        uv[:, 1::2] = v
        return y.astype(np.uint8), uv

    return pack(Y, U, V), pack(Yd, Ud, Vd)


def p016_frame_pair(w: int, h: int, seed: int, bits: int = 10):
    """P016 version of nv12_frame_pair: the 8-bit samples scaled to `bits`
    bits (value * 2^(bits-8) plus seeded low-order noise), left-aligned in
    16-bit words as P010/P016 store them.  Returns (ref, dis) of (y, uv)
    uint16 planes."""
    ref, dis = nv12_frame_pair(w, h, seed)
    st = Stream(seed ^ 0x0F16)
    sh = bits - 8

    def widen(a):
        low = (st.uniform(a.size) * (1 << sh)).astype(np.uint32).reshape(a.shape) if sh else 0
        return (((a.astype(np.uint32) << sh) + low) << (16 - bits)).astype(np.uint16)

    return tuple(widen(p) for p in ref), tuple(widen(p) for p in dis)


def c1_pair(index: int, w: int = 1920, h: int = 1080):
    return nv12_frame_pair(w, h, pair_seed(1, index))


def nv12_candidate(ref, step: float):
    """A distorted version of an NV12 frame (y, uv): 8x8 DCT quantisation of
    Y, Cb and Cr at `step`, clamped to the limited range."""
    y, uv = ref
    u, v = uv[:, 0::2].astype(np.float64), uv[:, 1::2].astype(np.float64)
    yd = dct_quantize(y.astype(np.float64), step, 128.0, 16.0, 235.0)
    ud = dct_quantize(u, step, 128.0, 16.0, 240.0)
    vd = dct_quantize(v, step, 128.0, 16.0, 240.0)
    out = np.empty_like(uv)
    out[:, 0::2] = ud
    out[:, 1::2] = vd
    return yd.astype(np.uint8), out


def c1_candidate_step(k: int):
    """DCT step of cached-reference candidate k: spread over [2, 48]."""
    return 2.0 + 46.0 * ((k * 0.6180339887498949) % 1.0)


def c2_size(index: int):
    st = Stream(pair_seed(2, index) ^ 0x5A5A)
    return st.randint(64, 2048), st.randint(64, 2048)


def c2_pair(index: int):
    w, h = c2_size(index)
    return srgb_pair(w, h, pair_seed(2, index))


def rgb10_pair(w: int, h: int, seed: int):
    """C3-style pair of 10-bit BT.2020 RGB (h, w, 3) uint16 images."""
    st = Stream(seed)
    ref = gratings(st, w, h, 512.0, 48.0, 64.0, 1023.0)
    sigma = st.scalar(0.5, 2.0)
    dis = np.empty_like(ref)
    noise = 8.0 * st.normal(h * w * 3).reshape(h, w, 3)
    for c in range(3):
        dis[:, :, c] = gaussian_filter(ref[:, :, c], sigma)
    dis = np.clip(np.round(dis + noise), 0, 1023)
    return ref.astype(np.uint16), dis.astype(np.uint16)


def c3_pair(index: int, w: int = 3840, h: int = 2160):
    return rgb10_pair(w, h, pair_seed(3, index))


def c4_jobs(n_jobs: int, rate: float, seed_index: int = 0):
    """Serving workload: list of dicts {t, w, h, k, steps, seed}: arrival time
    (s, Poisson process of `rate` per second), size log-uniform between
    128x128 and 3840x2160, k in 1..16 candidates, DCT step per candidate."""
    st = Stream(pair_seed(4, seed_index))
    t = 0.0
    jobs = []
    for j in range(n_jobs):
        t += -math.log(1.0 - st.scalar()) / rate
        u = st.scalar()
        w = int(round(128 * 30.0 ** u))
        h = int(round(128 * 16.875 ** u))
        k = st.randint(1, 16)
        steps = [st.scalar(2.0, 48.0) for _ in range(k)]
        jobs.append({"t": t, "w": w, "h": h, "k": k, "steps": steps,
                     "seed": pair_seed(4, 1000 + j)})
    return jobs


C4_POOL_W, C4_POOL_H, C4_POOL_CANDS = 3840, 2160, 16


def c4_pool_reference():
    """The serving pool's reference: a 3840x2160 sRGB8 image with C0 content
    (gratings + noise).  Jobs crop their reference from it."""
    st = Stream(pair_seed(4, 500))
    return gratings(st, C4_POOL_W, C4_POOL_H, 128.0, 12.0, 16.0, 255.0).astype(np.uint8)


def c4_pool_step(i):
    """DCT step of pool candidate i: the midpoints of 16 equal bins of [2, 48]."""
    return 2.0 + 46.0 * (i + 0.5) / C4_POOL_CANDS


def c4_pool_candidate(ref, i):
    """Pool candidate i: the reference plus Gaussian noise (sigma 4), 8x8 DCT
    quantisation at step c4_pool_step(i), rounded to uint8."""
    st = Stream(pair_seed(4, 600 + i))
    h, w, _ = ref.shape
    d = np.clip(ref.astype(np.float64) + 4.0 * st.normal(h * w * 3).reshape(h, w, 3), 0, 255)
    for c in range(3):
        d[:, :, c] = dct_quantize(d[:, :, c], c4_pool_step(i), 128.0, 0.0, 255.0)
    return d.astype(np.uint8)


def c4_job_crop(job):
    """Crop offset (x, y) of a job inside the pool images and the pool
    candidate of each of its DCT steps (the bin that holds the step)."""
    st = Stream(job["seed"])
    ox = min(int(st.scalar() * (C4_POOL_W - job["w"] + 1)), C4_POOL_W - job["w"])
    oy = min(int(st.scalar() * (C4_POOL_H - job["h"] + 1)), C4_POOL_H - job["h"])
    idx = [min(C4_POOL_CANDS - 1, int((s - 2.0) / 46.0 * C4_POOL_CANDS)) for s in job["steps"]]
    return ox, oy, idx


def serving_job_images(job):
    """Reference + candidates (uint8 HxWx3) for a serving job."""
    st = Stream(job["seed"])
    w, h = job["w"], job["h"]
    ref = gratings(st, w, h, 128.0, 12.0, 16.0, 255.0)
    cands = []
    for step in job["steps"]:
        d = np.clip(ref + 4.0 * st.normal(h * w * 3).reshape(h, w, 3), 0, 255)
        for c in range(3):
            d[:, :, c] = dct_quantize(d[:, :, c], step, 128.0, 0.0, 255.0)
        cands.append(d.astype(np.uint8))
    return ref.astype(np.uint8), cands


def synthetic_pair(width: int, height: int, mag: int):
    """The reference test suite's deterministic pair (gradient RGB and a +/-mag
    8x8 checkerboard perturbation; ssim2-gpu/tests/parity_lock.rs:77-102)."""
    y, x = np.mgrid[0:height, 0:width]
    r = (x * 220 // max(width, 1)) & 0xFF
    g = (y * 220 // max(height, 1)) & 0xFF
    b = ((x + y) * 200 // max(width + height, 1)) & 0xFF
    a = np.stack([r, g, b], axis=-1).astype(np.int32)
    pert = np.where(((x // 8) ^ (y // 8)) & 1 == 0, mag, -mag)[..., None]
    d = np.clip(a + pert, 0, 255)
    return a.astype(np.uint8), d.astype(np.uint8)
