"""The pinned staging ring of the batch path (gzippy_b200/csrc/stage.h),
checked on the CPU: the header is plain C++, and tests/stage_check.cpp runs
its plan and its upload/download pipelines against a byte-array device whose
copies are deferred the way a CUDA stream defers them."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_stage_ring_plan_and_pipelines():
    out = os.path.join(HERE, "_build")
    os.makedirs(out, exist_ok=True)
    exe = os.path.join(out, "stage_check")
    subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-Werror", "-o", exe,
                    os.path.join(HERE, "stage_check.cpp")], check=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "0 failures" in r.stdout
