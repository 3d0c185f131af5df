"""Host-only check of the submission planner (tests/plan_check.cu): layout
invariants of the device regions of random submissions of every format,
metric set, scale rule and storage type, including the DSSIM levels that the
clamp pass builds for small images.  Builds the harness with nvcc (host code
only runs) and links the library for the planner's host helpers."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "turbo-metrics_b200")
CUDA = "/usr/local/cuda"


@pytest.mark.skipif(shutil.which("nvcc") is None and not os.path.exists(os.path.join(CUDA, "bin", "nvcc")),
                    reason="nvcc not available")
def test_plan_layout_invariants(tmb, tmp_path):
    nvcc = os.path.join(CUDA, "bin", "nvcc") if os.path.exists(os.path.join(CUDA, "bin", "nvcc")) else "nvcc"
    exe = str(tmp_path / "plan_check")
    subprocess.run([nvcc, "-std=c++17", "-O1", "-gencode", "arch=compute_100a,code=sm_100a",
                    os.path.join(ROOT, "tests", "plan_check.cu"), "-o", exe, "-L" + PKG, "-lssim2b200",
                    "-L" + os.path.join(CUDA, "lib64"), "-lcudart", "-Xlinker", "-rpath=" + PKG],
                   check=True, capture_output=True)
    env = dict(os.environ)
    env["LD_LIBRARY_PATH"] = PKG + os.pathsep + os.path.join(CUDA, "lib64") + os.pathsep + env.get("LD_LIBRARY_PATH", "")
    out = subprocess.run([exe, "400"], capture_output=True, text=True, env=env, timeout=300)
    assert out.returncode == 0 and out.stdout.startswith("OK"), out.stdout + out.stderr
    # the random submissions exercised the clamp pass's layout too
    assert "clamped=0" not in out.stdout
