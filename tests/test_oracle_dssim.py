"""The DSSIM oracle (oracle/dssim_oracle.c) pinned against the values the
reference publishes for its DSSIM path.

crates/dssim-gpu/PORT_STATUS.md:26-30 lists dssim-core 3.4 (CPU) and GPU
scores of the crates/dssim-gpu/tests/parity_lock.rs cases; the generators
below restate that file's `solid`, `gradient` and `add_noise` (:54-88).  The
bounds are the reference's own: 0.1 % for black vs white
(crates/dssim-cuda/tests/accuracy.rs:241-255), 1 % for a small distortion
(accuracy.rs:195-204), 5 % for the JPEG corpus (parity_lock.rs:240-250),
which PIL decodes here instead of the `image` crate."""
import json
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = json.load(open(os.path.join(HERE, "golden", "reference_tables.json")))["dssim"]
PUB = GOLD["published"]
REF_TREE = os.environ.get("TURBO_METRICS_REF", "/root/reference")


def solid(w, h, v):
    return np.full((h, w, 3), v, np.uint8)


def gradient(w, h):
    x = (np.arange(w) * 255) // w
    return np.repeat(np.repeat(x[None, :, None].astype(np.uint8), h, 0), 3, 2)


def add_noise(a, amount):
    """parity_lock.rs:77-88: LCG seed 12345, the high half taken as i16, Rust's
    truncating remainder."""
    flat = a.reshape(-1)
    out = np.empty_like(flat)
    seed = 12345
    m = amount * 2 + 1
    for i, v in enumerate(flat):
        seed = (seed * 1103515245 + 12345) & 0xFFFFFFFF
        n = (seed >> 16) - 65536 if (seed >> 16) >= 32768 else (seed >> 16)
        r = int(np.fmod(n, m))
        out[i] = min(255, max(0, int(v) + r - amount))
    return out.reshape(a.shape)


@pytest.mark.parametrize("mode", ["cuda32", "fp64"])
def test_identical_is_zero(oracle, mode):
    g = gradient(32, 32)
    assert oracle.dssim_srgb8(g, g, mode).dssim == 0.0 == PUB["identical_32"]["dssim_core_cpu"]


@pytest.mark.parametrize("mode", ["cuda32", "fp64"])
def test_black_vs_white(oracle, mode):
    got = oracle.dssim_srgb8(solid(64, 64, 0), solid(64, 64, 255), mode).dssim
    for want in PUB["black_white_64"].values():
        assert abs(got - want) / want < 1e-3, (got, want)


@pytest.mark.parametrize("mode", ["cuda32", "fp64"])
def test_noisy_gradient(oracle, mode):
    g = gradient(64, 64)
    got = oracle.dssim_srgb8(g, add_noise(g, 8), mode).dssim
    for want in PUB["noisy_gradient_64"].values():
        assert abs(got - want) / want < 1e-2, (got, want)


def test_noise_generator_range():
    """The i16 cast makes the noise span [-3a, a]: the generator is the
    reference's, not a symmetric one."""
    z = np.full((1, 4096, 3), 128, np.uint8)
    d = add_noise(z, 8).astype(int) - 128
    assert d.min() == -24 and d.max() == 8


def test_level_dims_clamped_to_8(oracle):
    """dssim-cuda/src/lib.rs:184-205: halve rounding up, never below 8."""
    assert oracle.dssim_level_dims(64, 64) == [(64, 64), (32, 32), (16, 16), (8, 8), (8, 8)]
    assert oracle.dssim_level_dims(21, 1000) == [(21, 1000), (11, 500), (8, 250), (8, 125), (8, 63)]
    with pytest.raises(ValueError):
        oracle.dssim_linear(np.zeros((7, 9, 3), np.float32), np.zeros((7, 9, 3), np.float32))


def test_f32_mirror_close_to_f64(oracle):
    rng = np.random.default_rng(5)
    for w, h in ((96, 80), (37, 53), (200, 150)):
        a = rng.integers(0, 256, (h, w, 3), dtype=np.uint8)
        b = np.clip(a.astype(int) + rng.integers(-12, 13, a.shape), 0, 255).astype(np.uint8)
        f32 = oracle.dssim_srgb8(a, b, "cuda32")
        f64 = oracle.dssim_srgb8(a, b, "fp64")
        assert abs(f32.dssim - f64.dssim) <= 2e-3 * f64.dssim + 1e-7, (w, h, f32.dssim, f64.dssim)
        assert np.max(np.abs(f32.level_scores - f64.level_scores)) < 1e-5


def test_lab_white_and_black(oracle):
    """lab.rs:42-86: white maps to L = (1 - 16/116) * 1.05 and the a/b offsets,
    black to L = 0 (linear branch of lab_f)."""
    import ctypes
    o = (ctypes.c_float * 3)()
    oracle._lib.or_dssim_lab_f32(ctypes.c_float(1.0), ctypes.c_float(1.0), ctypes.c_float(1.0), o)
    np.testing.assert_allclose(list(o), [(1 - 16 / 116) * 1.05, 86.2 / 220, 107.9 / 220], rtol=1e-6)
    oracle._lib.or_dssim_lab_f32(ctypes.c_float(0.0), ctypes.c_float(0.0), ctypes.c_float(0.0), o)
    np.testing.assert_allclose(list(o), [0.0, 86.2 / 220, 107.9 / 220], atol=1e-7)


def _load_rgb(path):
    from PIL import Image
    return np.asarray(Image.open(path).convert("RGB"), np.uint8)


@pytest.mark.skipif(not os.path.isdir(REF_TREE), reason="reference tree not mounted")
@pytest.mark.parametrize("q", [70, 90])
def test_corpus(oracle, q):
    d = os.path.join(REF_TREE, "crates", "dssim-cuda", "test_data")
    src = _load_rgb(os.path.join(d, "source.png"))
    dis = _load_rgb(os.path.join(d, "q%d.jpg" % q))
    got = oracle.dssim_srgb8(src, dis, "cuda32").dssim
    for want in PUB["q%d" % q].values():
        assert abs(got - want) / want < 0.05, (q, got, want)
