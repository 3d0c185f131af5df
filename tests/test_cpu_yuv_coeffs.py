"""The 4:2:0 YUV conversion constants, pinned to the reference's own f32
derivation (no GPU needed).

The reference computes Kr / Kb from the primaries in f32 const arithmetic
(constants_from_primaries, crates/cuda-colorspace-kernel/src/lib.rs:205-221,
with the Vec2 / Vec3 algebra of const_algebra.rs) and the five conversion
coefficients from them in f32 (MatrixCoefficients::coefficients,
lib.rs:188-203).  The oracle restates that derivation operation for
operation; the engine's coefficients (s2_yuv_coefficients, the values the
prep kernel is given) must equal it to the bit for every matrix, range and
depth.  The f64 derivation rounded once differs from it by a few ulp, which
is why the derivation itself is restated."""
import ctypes

import numpy as np
import pytest

MATS = ["bt709", "bt601_525", "bt601_625"]


def engine_coeffs(tmb, matrix, full, bits):
    c = (ctypes.c_float * 5)()
    ymin, neu = ctypes.c_int32(), ctypes.c_int32()
    st = tmb.lib.s2_yuv_coefficients(tmb.capi.MATRIX[matrix], 1 if full else 0, bits, c, ctypes.byref(ymin),
                                     ctypes.byref(neu))
    assert st == 0
    return np.array(c[:], np.float32), ymin.value, neu.value


def f32_ref_derivation(matrix, full, bits):
    """The same derivation in numpy float32 scalars (each operation rounded)."""
    f = np.float32
    prim = {"bt709": (0.640, 0.330, 0.300, 0.600, 0.150, 0.060),
            "bt601_525": (0.630, 0.340, 0.310, 0.595, 0.155, 0.070),
            "bt601_625": (0.640, 0.330, 0.290, 0.600, 0.150, 0.060)}[matrix] + (0.3127, 0.3290)
    p = [f(v) for v in prim]

    def xyz(x, y):
        return (x / y, f(1.0), ((f(1.0) - x) - y) / y)

    def dot(a, b):
        return (a[0] * b[0] + a[1] * b[1]) + a[2] * b[2]

    def cross(a, b):
        return (a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0])

    r, g, b, w = xyz(p[0], p[1]), xyz(p[2], p[3]), xyz(p[4], p[5]), xyz(p[6], p[7])
    mul = f(1.0) / dot((r[0], g[0], b[0]), cross((r[1], g[1], b[1]), (r[2], g[2], b[2])))
    kr = dot(w, cross(g, b)) * mul
    kb = dot(w, cross(r, g)) * mul
    sh = bits - 8
    lr = f((1 << bits) - 1 if full else (235 - 16) << sh)
    cr = f((1 << bits) - 1 if full else (240 - 16) << sh)
    kg = (f(1.0) - kr) - kb
    return np.array([f(1.0) / lr, f(2.0) * (f(1.0) - kr) * f(1.0) / cr, f(2.0) * (f(1.0) - kb) * f(1.0) / cr,
                     f(-2.0) * (f(1.0) - kb) * kb / kg * f(1.0) / cr,
                     f(-2.0) * (f(1.0) - kr) * kr / kg * f(1.0) / cr], np.float32)


@pytest.mark.parametrize("matrix", MATS)
@pytest.mark.parametrize("full", [False, True])
@pytest.mark.parametrize("bits", [8, 16])
def test_engine_coefficients_are_the_reference_f32_derivation(tmb, oracle, matrix, full, bits):
    eng, ymin, neu = engine_coeffs(tmb, matrix, full, bits)
    ref, rymin, rneu = oracle.yuv_coeffs_ref_f32(matrix, full, bits)
    assert eng.tobytes() == ref.tobytes(), (eng, ref)
    assert eng.tobytes() == f32_ref_derivation(matrix, full, bits).tobytes()
    assert (ymin, neu) == (rymin, rneu) == ((0 if full else 16 << (bits - 8)), 1 << (bits - 1))


def test_bt709_limited_kr_kb_are_the_textbook_values(oracle):
    """Sanity: BT.709 from its primaries gives Kr 0.2126, Kb 0.0722 (4 digits)."""
    c, _, _ = oracle.yuv_coeffs_ref_f32("bt709", False, 8)
    kr = 1.0 - float(c[1]) * 224.0 / 2.0
    kb = 1.0 - float(c[2]) * 224.0 / 2.0
    assert abs(kr - 0.2126) < 1e-4 and abs(kb - 0.0722) < 1e-4


def test_f64_derivation_differs_by_ulps_only(oracle):
    """The f64 derivation rounded once (what the engine used before) is within
    4 ulp of the reference's f32 values: the difference the pinning removes."""
    for m in MATS:
        ref, _, _ = oracle.yuv_coeffs_ref_f32(m, False, 8)
        prim = {"bt709": (0.640, 0.330, 0.300, 0.600, 0.150, 0.060),
                "bt601_525": (0.630, 0.340, 0.310, 0.595, 0.155, 0.070),
                "bt601_625": (0.640, 0.330, 0.290, 0.600, 0.150, 0.060)}[m] + (0.3127, 0.3290)
        xyz = [np.array([x / y, 1.0, (1 - x - y) / y]) for x, y in zip(prim[0::2], prim[1::2])]
        M = np.stack(xyz[:3], 1)
        s = np.linalg.solve(M, xyz[3])
        kr, kb = s[0] * M[1, 0], s[2] * M[1, 2]
        kg = 1 - kr - kb
        d64 = np.array([1 / 219, 2 * (1 - kr) / 224, 2 * (1 - kb) / 224, -2 * (1 - kb) * kb / kg / 224,
                        -2 * (1 - kr) * kr / kg / 224]).astype(np.float32)
        ulps = np.abs(d64.view(np.int32).astype(np.int64) - ref.view(np.int32).astype(np.int64))
        assert ulps.max() <= 4, (m, ulps)


def test_eotf_constants_follow_the_reference_f32_consts(oracle):
    """BT709::eotf (lib.rs:223-238): BETA, ALPHA = 1 + 5.5 BETA and THRESHOLD
    are f32 consts; value + (ALPHA - 1) is what the engine adds, and it
    multiplies by the f32 reciprocals of ALPHA and 4.5 where the reference
    divides (<= 1 ulp from the quotient)."""
    f = np.float32
    beta = f(0.018053968510807)
    alpha = f(1.0) + f(5.5) * beta
    c = oracle.bt709_eotf_consts()
    assert c[0] == alpha - f(1.0)
    assert c[1] == f(1.0 / np.float64(alpha))
    assert c[2] == f(0.08124285829863521110029445797874)
    assert c[3] == f(1.0 / 4.5)
