"""CPU check of the cluster V-cycle's plan (otm_cluster.cuh, cl_plan) at the library's cluster
size: shared-memory regions inside the plan and disjoint, slabs covering every plane, plane tables
within bounds, and every ghost copy fed (tests/cpp/cluster_plan_check.cu, host code compiled with
nvcc; no GPU needed)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _nvcc():
    return shutil.which("nvcc") or ("/usr/local/cuda/bin/nvcc" if os.path.exists("/usr/local/cuda/bin/nvcc") else None)


@pytest.mark.skipif(_nvcc() is None, reason="needs nvcc")
def test_cluster_plans_fit_and_feed_every_ghost(tmp_path):
    exe = tmp_path / "cluster_plan_check"
    subprocess.run([_nvcc(), "-std=c++17", "-O1", "-gencode", "arch=compute_100a,code=sm_100a",
                    "-I", os.path.join(ROOT, "include"), "-I", os.path.join(ROOT, "opentm_b200", "csrc"),
                    os.path.join(ROOT, "tests", "cpp", "cluster_plan_check.cu"), "-o", str(exe)], check=True,
                   timeout=300)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.strip() == "ok"
