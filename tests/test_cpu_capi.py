"""CPU-only checks of the C-ABI library: it loads, exports every symbol that
include/ssim2b200.h declares, and its host-only helpers behave.  No compute
call is made (no GPU here)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            text = open(os.path.join(ROOT, "include", fn)).read()
            text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
            names |= set(re.findall(r"\b(s2_[a-z0-9_]+)\s*\(", text))
    return sorted(names)


def test_library_exports_every_declared_symbol(tmb):
    lib = ctypes.CDLL(tmb.library_path)
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing
    assert len(declared_symbols()) >= 25


def test_version_and_status_strings(tmb):
    assert "sm_100a" in tmb.version()
    assert tmb.lib.s2_status_string(2).decode() == "invalid image size"
    assert tmb.lib.s2_status_string(4).decode() == "no cached reference"


@pytest.mark.parametrize("w,h,rule,n", [
    (1920, 1080, "cpu", 6), (16, 16, "cpu", 3), (16, 16, "min8", 2), (16, 16, "all6", 6),
    (7, 100, "cpu", 0), (7, 100, "min8", 0), (8, 8, "cpu", 2), (8, 8, "min8", 1),
    (64, 64, "cpu", 5), (64, 64, "min8", 4), (2048, 64, "cpu", 5), (1, 1, "all6", 6)])
def test_num_scales_matches_oracle(tmb, oracle, w, h, rule, n):
    assert tmb.num_scales(w, h, rule) == n
    assert oracle.num_scales(w, h, rule) == n


def test_config_validation_needs_no_gpu(tmb):
    cfg = tmb.capi.make_config()
    cfg.strip_rows = 48  # not one of 16, 32, 64
    h = ctypes.c_void_p()
    assert tmb.lib.s2_create(ctypes.byref(cfg), 64, 64, ctypes.byref(h)) == 8  # S2_ERR_INVALID_ARG
    cfg = tmb.capi.make_config()
    assert tmb.lib.s2_create(ctypes.byref(cfg), 7, 64, ctypes.byref(h)) == 2  # invalid size
    cfg.struct_size = 4
    assert tmb.lib.s2_create(ctypes.byref(cfg), 64, 64, ctypes.byref(h)) == 8


def test_result_layout_and_metric_bits(tmb):
    """s2_result: score, 108 stats, 108 sums, n_scales, status, then the DSSIM
    value and its five per-scale scores."""
    R = tmb.capi.Result
    assert ctypes.sizeof(R) == 8 + 108 * 8 * 2 + 4 + 4 + 8 + 5 * 8
    assert R.dssim.offset == 8 + 108 * 8 * 2 + 8
    assert tmb.capi.metrics_mask("ssimulacra2") == 1
    assert tmb.capi.metrics_mask("dssim") == 2
    assert tmb.capi.metrics_mask(("ssimulacra2", "dssim")) == 3
    with pytest.raises(KeyError):
        tmb.capi.metrics_mask("butteraugli")


def test_dssim_entry_points_validate_without_gpu(tmb):
    """Argument and size checks come before any device call."""
    lib = tmb.lib
    d = ctypes.c_void_p()
    assert lib.s2_dssim_create(0, 7, 64, ctypes.byref(d)) == 2  # below 8x8: invalid size
    assert lib.s2_dssim_create(0, 64, 64, None) == 8
    v = ctypes.c_double()
    assert lib.s2_dssim_compute_srgb8(None, None, 0, None, 0, 0, None, ctypes.byref(v)) == 8
    assert lib.s2_dssim_compute_dis_only_srgb8(None, None, 0, 0, None, ctypes.byref(v)) == 8
    assert lib.s2_set_metrics(None, 3) == 8
    assert lib.s2_batch_set_metrics(None, 2) == 8
    assert lib.s2_get_dssim(None, None, None) == 8


def test_tile_timeout_hook_validates_without_gpu(tmb):
    lib = tmb.lib
    assert lib.s2_debug_tile_timeout(-1, -5) == 8  # negative wait bound
    assert lib.s2_debug_tile_timeout(3, 1 << 20) == 0
    assert lib.s2_debug_tile_timeout(-1, 0) == 0  # back to the defaults
    assert tmb.capi._ERRS[tmb.capi.S2_ERR_TIMEOUT] is tmb.Timeout
