"""Visited placement 4's plan for moving a search's bitmap into its block's
shared memory (gmapf_b200/csrc/region_plan.cuh), checked over every case on
the host: the same source the kernel includes, built by nvcc as host code."""
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def test_region_plan_every_case(tmp_path):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(nvcc).exists():
        pytest.skip("nvcc not found")
    exe = tmp_path / "region_plan_check"
    subprocess.run([nvcc, "-std=c++17", "-O2", "-Wno-deprecated-gpu-targets", "-I", str(ROOT / "gmapf_b200" / "csrc"),
                    str(ROOT / "tests" / "cpp" / "region_plan_check.cu"), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.startswith("ok ")
