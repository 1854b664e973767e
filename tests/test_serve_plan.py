"""The serving loop's wave policy (paralanczos_b200/csrc/pl_serve_plan.cuh),
the function the device planning kernel runs, driven on the host over request
tables: every wave makes progress and ends (full on time, sets, indices or
pieces), its pieces are laid out contiguously, and every set of every request
is scheduled exactly once.  Needs nvcc (host code only), no GPU."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


def test_wave_policy_invariants(tmp_path):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc absent")
    exe = tmp_path / "plan_check"
    subprocess.run([nvcc, "-std=c++17", "-O1", "--expt-relaxed-constexpr", os.path.join(HERE, "serve_plan_check.cu"), "-o", str(exe)],
                   check=True, capture_output=True, text=True, timeout=300)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.strip().endswith("OK"), r.stdout + r.stderr
