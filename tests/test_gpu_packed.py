"""The search kernels' packed FP32x2 distance against the scalar reference-order distance.

Every hit test of the tile walk and the per-query walk compares distance bits computed two
candidates at a time (rtnn_b200/csrc/packed.cuh: dist2_pair). Rows are bit-exact only if
those bits equal ((dx*dx + dy*dy) + dz*dz) with every step rounded to FP32
(src/sutil/vec_math.h:527-530 as check.cpp:36-37 uses it), which dist2_ref in common.cuh
computes one operation at a time. The probe compiles the library's own header for sm_100a
and compares the two on 2^25 pairs per value range.
"""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "rtnn_b200", "csrc")


@pytest.mark.gpu
def test_packed_distance_matches_scalar_bits(tmp_path):
    nvcc = os.environ.get("NVCC", "nvcc")
    if not shutil.which(nvcc):
        pytest.skip("nvcc not found")
    exe = tmp_path / "packed_probe"
    subprocess.run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17",
                    "-I" + CSRC, os.path.join(ROOT, "tests", "cuda", "packed_probe.cu"),
                    "-o", str(exe)], check=True, timeout=300)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    lines = r.stdout.strip().splitlines()
    assert len(lines) == 3, r.stdout + r.stderr
    for line in lines:
        assert " 0 of " in line and "(no error)" in line, line
    assert r.returncode == 0
