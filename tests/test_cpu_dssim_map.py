"""Host-only check of the DSSIM tile pass's thread-to-item mapping
(tests/dssim_map_check.cu): for each blur stage the block's threads cover
every (plane, row segment, column pair) exactly once, and each aligned
half-warp reads 32 consecutive floats of one row.  Builds the harness with
nvcc (host code only runs)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CUDA = "/usr/local/cuda"


@pytest.mark.skipif(shutil.which("nvcc") is None and not os.path.exists(os.path.join(CUDA, "bin", "nvcc")),
                    reason="nvcc not available")
def test_dssim_stage_mapping(tmp_path):
    nvcc = os.path.join(CUDA, "bin", "nvcc") if os.path.exists(os.path.join(CUDA, "bin", "nvcc")) else "nvcc"
    exe = str(tmp_path / "dssim_map_check")
    subprocess.run([nvcc, "-std=c++17", "-O1", os.path.join(ROOT, "tests", "dssim_map_check.cu"), "-o", exe],
                   check=True, capture_output=True)
    out = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0 and out.stdout.strip().endswith("OK"), out.stdout + out.stderr
