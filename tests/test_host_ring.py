"""CPU check of the serving form's pinned-ring bookkeeping (opentm_b200/csrc/otm_host_ring.h),
compiled with the host C++ compiler."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_ring_offsets_randomised(tmp_path):
    exe = tmp_path / "ring_check"
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "opentm_b200", "csrc"),
                    os.path.join(ROOT, "tests", "cpp", "ring_check.cpp"), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.strip() == "ok"
