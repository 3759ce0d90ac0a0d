"""The slab plan of snac_gpu_step_host (snac_b200/csrc/snac_slab_plan.h) is
hazard-free: compiled on the host with the checker tests/slab_plan_check.cpp,
which replays the plan's operations over every node and hex row for ragged
and full-size meshes, 1 to 64 slabs, with and without the temperature
stages (no GPU needed)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_slab_plan_reads_and_writes_in_dependency_order(tmp_path):
    exe = tmp_path / "slab_plan_check"
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "snac_b200", "csrc"),
                    os.path.join(ROOT, "tests", "slab_plan_check.cpp"), "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.startswith("ok "), r.stdout
