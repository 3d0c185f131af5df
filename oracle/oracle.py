"""ctypes wrapper of the CPU oracle (oracle/ssim2_oracle.c).

TEST INFRASTRUCTURE ONLY: the parity tests, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py use it as the checker.  The product path never
imports it.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "libssim2_oracle.so")

MODE = {"fp64": 0, "cuda32": 1, "cpu32": 2, "fir32": 3}
RULE = {"cpu": 0, "min8": 1, "all6": 2}


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB


if not os.path.exists(LIB):
    build()
_lib = ctypes.CDLL(LIB)
_P = ctypes.POINTER
_F = _P(ctypes.c_float)
_D = _P(ctypes.c_double)
_U8 = _P(ctypes.c_uint8)
_U16 = _P(ctypes.c_uint16)
_lib.or_score_from_stats.restype = ctypes.c_double
_lib.or_ssim2_linear.restype = ctypes.c_int
_lib.or_ssim2_linear_f64.restype = ctypes.c_int
_lib.or_num_scales.restype = ctypes.c_int
_lib.or_blur_constants.restype = ctypes.c_int


def _f(a):
    return a.ctypes.data_as(_F)


def _d(a):
    return a.ctypes.data_as(_D)


def srgb8_lut():
    a = np.zeros(256, np.float32)
    _lib.or_srgb8_lut(_f(a))
    return a


def weights():
    w = np.zeros(108)
    _lib.or_weights(_d(w))
    return w


def blur_constants():
    arrs = [np.zeros(3, np.float32) for _ in range(5)]
    taps = np.zeros(5)
    radius = _lib.or_blur_constants(*[_f(a) for a in arrs], _d(taps))
    names = ["mul_in", "mul_prev", "mul_prev2", "vert_mul_in", "vert_mul_prev"]
    out = dict(zip(names, arrs))
    out["radius"] = radius
    out["fir_taps"] = taps
    return out


def num_scales(w, h, rule="cpu"):
    return _lib.or_num_scales(w, h, RULE[rule])


def score_from_stats(stats):
    s = np.ascontiguousarray(stats, np.float64)
    return _lib.or_score_from_stats(_d(s))


def srgb8_to_linear(img, f64=False):
    a = np.ascontiguousarray(img, np.uint8)
    if f64:
        out = np.empty(a.shape, np.float64)
        _lib.or_srgb8_to_linear_f64(a.ctypes.data_as(_U8), ctypes.c_size_t(a.size), _d(out))
    else:
        out = np.empty(a.shape, np.float32)
        _lib.or_srgb8_to_linear(a.ctypes.data_as(_U8), ctypes.c_size_t(a.size), _f(out))
    return out


def nv12_to_linear(y, uv, f64=False):
    y = np.ascontiguousarray(y, np.uint8)
    uv = np.ascontiguousarray(uv, np.uint8)
    h, w = y.shape
    assert uv.shape == (h // 2, w)
    if f64:
        out = np.empty((h, w, 3), np.float64)
        _lib.or_nv12_to_linear_f64(y.ctypes.data_as(_U8), uv.ctypes.data_as(_U8), ctypes.c_size_t(w), w, h, _d(out))
    else:
        out = np.empty((h, w, 3), np.float32)
        _lib.or_nv12_to_linear(y.ctypes.data_as(_U8), uv.ctypes.data_as(_U8), ctypes.c_size_t(w), w, h, _f(out))
    return out


MATRIX = {"bt709": 0, "bt601_525": 1, "bt601_625": 2}


def yuv420_to_linear(y, uv, matrix="bt709", full=False, f64=False):
    """4:2:0 biplanar YUV -> linear RGB: uint8 planes (NV12) or uint16 planes
    (P016); y (H, W), uv (H/2, W) interleaved CbCr."""
    bits = 8 if y.dtype == np.uint8 else 16
    y = np.ascontiguousarray(y)
    uv = np.ascontiguousarray(uv, y.dtype)
    h, w = y.shape
    assert uv.shape == (h // 2, w)
    pitch = ctypes.c_size_t(w * y.itemsize)
    args = (y.ctypes.data_as(ctypes.c_void_p), uv.ctypes.data_as(ctypes.c_void_p), pitch, w, h, bits,
            MATRIX[matrix], 1 if full else 0)
    if f64:
        out = np.empty((h, w, 3), np.float64)
        _lib.or_yuv420_to_linear_f64(*args, _d(out))
    else:
        out = np.empty((h, w, 3), np.float32)
        _lib.or_yuv420_to_linear(*args, _f(out))
    return out


def yuv_coeffs_ref_f32(matrix="bt709", full=False, bits=8):
    """The reference's f32 derivation (cuda-colorspace-kernel/src/lib.rs:188-221)
    of y_coeff, r_coeff, b_coeff, g_coeff1, g_coeff2, with the luma minimum and
    chroma neutral value."""
    c = np.zeros(5, np.float32)
    ymin, neu = ctypes.c_int(), ctypes.c_int()
    _lib.or_yuv_coeffs_ref_f32(MATRIX[matrix], 1 if full else 0, bits, _f(c), ctypes.byref(ymin), ctypes.byref(neu))
    return c, ymin.value, neu.value


def bt709_eotf_consts():
    """alpha - 1, 1 / alpha, threshold, 1 / 4.5 as the f32 conversion uses them."""
    c = np.zeros(4, np.float32)
    _lib.or_bt709_eotf_consts(_f(c))
    return c


def rgb16_to_linear(img, bits=10, f64=False):
    a = np.ascontiguousarray(img, np.uint16)
    n = a.size // 3
    if f64:
        out = np.empty(a.shape, np.float64)
        _lib.or_rgb16_bt2020_to_linear_f64(a.ctypes.data_as(_U16), ctypes.c_size_t(n), bits, _d(out))
    else:
        out = np.empty(a.shape, np.float32)
        _lib.or_rgb16_bt2020_to_linear(a.ctypes.data_as(_U16), ctypes.c_size_t(n), bits, _f(out))
    return out


def downscale(lin):
    a = np.ascontiguousarray(lin, np.float32)
    h, w, _ = a.shape
    out = np.empty(((h + 1) // 2, (w + 1) // 2, 3), np.float32)
    _lib.or_downscale_f32(_f(a), w, h, _f(out))
    return out


def linear_to_xyb(lin):
    a = np.ascontiguousarray(lin, np.float32)
    out = np.empty_like(a)
    _lib.or_linear_to_xyb_f32(_f(a), ctypes.c_size_t(a.size // 3), _f(out))
    return out


def blur_plane(plane, mode="cuda32"):
    a = np.ascontiguousarray(plane, np.float32)
    h, w = a.shape
    out = np.empty_like(a)
    _lib.or_blur_plane_f32(_f(a), w, h, MODE[mode], _f(out))
    return out


def blur_plane_f64(plane):
    a = np.ascontiguousarray(plane, np.float64)
    h, w = a.shape
    out = np.empty_like(a)
    _lib.or_blur_plane_f64(_d(a), w, h, _d(out))
    return out


class Result:
    def __init__(self, score, stats, sums, n_scales):
        self.score, self.stats, self.sums, self.n_scales = score, stats, sums, n_scales


def ssim2_linear(ref, dis, mode="fp64", rule="cpu"):
    """Full metric from linear RGB (H, W, 3).  mode: fp64 | cuda32 | cpu32 | fir32."""
    h, w = ref.shape[:2]
    st = np.zeros(108)
    su = np.zeros(108)
    sc = ctypes.c_double()
    ns = ctypes.c_int()
    if mode == "fp64":
        r = np.ascontiguousarray(ref, np.float64)
        d = np.ascontiguousarray(dis, np.float64)
        rc = _lib.or_ssim2_linear_f64(_d(r), _d(d), w, h, RULE[rule], _d(st), _d(su), ctypes.byref(sc),
                                      ctypes.byref(ns))
    else:
        r = np.ascontiguousarray(ref, np.float32)
        d = np.ascontiguousarray(dis, np.float32)
        rc = _lib.or_ssim2_linear(_f(r), _f(d), w, h, MODE[mode], RULE[rule], _d(st), _d(su), ctypes.byref(sc),
                                  ctypes.byref(ns))
    if rc != 0:
        raise ValueError("invalid image size %dx%d" % (w, h))
    return Result(sc.value, st, su, ns.value)


def ssim2_maps_fir32(ref, dis, scale, rule="cpu"):
    """The fir32 error maps of one scale from linear RGB (H, W, 3): an array
    (3 channels, 3 maps [ssim error, artifact, detail loss], h_s, w_s)."""
    h, w = ref.shape[:2]
    hs, ws = h, w
    for _ in range(scale):
        hs, ws = (hs + 1) // 2, (ws + 1) // 2
    r = np.ascontiguousarray(ref, np.float32)
    d = np.ascontiguousarray(dis, np.float32)
    out = np.zeros((3, 3, hs, ws), np.float32)
    if _lib.or_ssim2_maps_fir32(_f(r), _f(d), w, h, RULE[rule], scale, _f(out)) != 0:
        raise ValueError("scale %d is not scored for %dx%d" % (scale, w, h))
    return out


def ssim2_srgb8(ref, dis, mode="fp64", rule="cpu"):
    f64 = mode == "fp64"
    return ssim2_linear(srgb8_to_linear(ref, f64), srgb8_to_linear(dis, f64), mode, rule)


# ---- DSSIM (dssim_oracle.c): crates/dssim-cuda's metric ----------------------
DSSIM_MODE = {"fp64": 0, "cuda32": 1}
_lib.or_dssim_linear.restype = ctypes.c_int


class DssimResult:
    def __init__(self, dssim, level_scores, level_means):
        self.dssim, self.level_scores, self.level_means = dssim, level_scores, level_means


def dssim_level_dims(w, h):
    dw = (ctypes.c_int * 5)()
    dh = (ctypes.c_int * 5)()
    _lib.or_dssim_level_dims(w, h, dw, dh)
    return list(zip(dw, dh))


def dssim_linear(ref, dis, mode="cuda32"):
    """DSSIM from linear RGB (H, W, 3).  mode: cuda32 (the reference GPU's
    f32 arithmetic) | fp64."""
    h, w = ref.shape[:2]
    r = np.ascontiguousarray(ref, np.float32)
    d = np.ascontiguousarray(dis, np.float32)
    sc = np.zeros(5)
    mn = np.zeros(5)
    out = ctypes.c_double()
    if _lib.or_dssim_linear(_f(r), _f(d), w, h, DSSIM_MODE[mode], _d(sc), _d(mn), ctypes.byref(out)) != 0:
        raise ValueError("invalid image size %dx%d" % (w, h))
    return DssimResult(out.value, sc, mn)


def dssim_srgb8(ref, dis, mode="cuda32"):
    """DSSIM of two sRGB8 images (H, W, 3): the reference's 256-entry LUT,
    then dssim_linear (dssim-cuda's srgb_to_linear, srgb.rs:23-73)."""
    return dssim_linear(srgb8_to_linear(ref), srgb8_to_linear(dis), mode)


_lib.zs_features_srgb8.restype = ctypes.c_int
_lib.zs_padded_width.restype = ctypes.c_int


class ZensimResult:
    def __init__(self, features, acc, peaks, n_scales):
        self.features, self.acc, self.peaks, self.n_scales = features, acc, peaks, n_scales


def zensim_padded_width(w):
    return _lib.zs_padded_width(w)


def zensim_features_srgb8(ref, dis):
    """zensim's 228 features of two sRGB8 images (H, W, 3) (restatement of
    crates/zensim-cuda; see zensim_oracle.c).  acc: (4, 3, 17) f64 sums,
    peaks: (4, 3, 3) maxima (f32), features: 228."""
    h, w = ref.shape[:2]
    r = np.ascontiguousarray(ref, np.uint8)
    d = np.ascontiguousarray(dis, np.uint8)
    acc = np.zeros((4, 3, 17))
    peaks = np.zeros((4, 3, 3), np.uint32)
    feat = np.zeros(228)
    ns = _lib.zs_features_srgb8(r.ctypes.data_as(_U8), d.ctypes.data_as(_U8), w, h, ctypes.c_size_t(3 * w),
                                _d(acc), peaks.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)), _d(feat))
    if ns < 0:
        raise ValueError("zensim needs at least 8x8, got %dx%d" % (w, h))
    return ZensimResult(feat, acc, peaks.view(np.float32), ns)
