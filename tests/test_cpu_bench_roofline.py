"""The roofline arithmetic of bench.py, without a GPU: the fused pass's
algorithmic bytes per launch (both frames' XYB planes read once over the six
scales), the prep pass's (NV12 read, XYB written), and the issue roofline
(warp instructions per launch over the issue peak at the sampled SM clock,
148 SMs x 4 schedulers x one instruction per cycle)."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def test_scale_sizes_and_algorithmic_bytes():
    # 1920x1080 and its five halvings (rounded up): 2,764,200 pixels in all
    assert bench.sum_pixels() == 1920 * 1080 + 960 * 540 + 480 * 270 + 240 * 135 + 120 * 68 + 60 * 34 == 2764200
    assert bench.algorithmic_bytes_fused(64) == 64 * 2 * 3 * 4 * 2764200 == 4245811200
    assert bench.algorithmic_bytes_prep(1) == 2 * 1.5 * 1920 * 1080 + 2 * 3 * 4 * 2764200


def test_issue_roofline():
    roof = {"warp_instructions_per_launch": 1982400000, "kernel_ms": {"fused": 2.85}}
    out = bench.with_issue_roofline(roof, {"sm_mhz": 1965.0}, {})
    iss = out["issue"]
    peak = 148 * 4 * 1965e6
    assert abs(iss["peak"] - peak / 1e9) < 1e-9
    assert abs(iss["achieved"] - 1982400000 / 2.85e-3 / 1e9) < 1e-6
    assert abs(iss["frac"] - 1982400000 / 2.85e-3 / peak) < 1e-12
    assert 0.59 < iss["frac"] < 0.61
    # unsampled clocks: the measured maximum of the pool's peaks file
    out = bench.with_issue_roofline({"warp_instructions_per_launch": 1e9, "kernel_ms": {"fused": 1.0}},
                                    {"sm_mhz": None}, {"sm_max_mhz": 1965.0})
    assert out["issue"]["sm_mhz"] == 1965.0
    # no instruction count: no issue roofline
    out = bench.with_issue_roofline({"warp_instructions_per_launch": None, "kernel_ms": {"fused": 1.0}},
                                    {"sm_mhz": 1965.0}, {})
    assert "issue" not in out
