"""The enumeration's branch-free helpers equal their sequential forms (CPU;
tests/native/flat_helpers_check.cpp, built with g++ against the kernels'
own headers)."""
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_flat_helpers_equal_sequential_forms(tmp_path):
    exe = tmp_path / "flat_helpers_check"
    subprocess.check_call(["g++", "-O2", "-std=c++17", "-I", str(ROOT / "culs_b200" / "csrc"), "-I", str(ROOT / "include"),
                           "-I", "/usr/local/cuda/include", str(ROOT / "tests" / "native" / "flat_helpers_check.cpp"),
                           "-o", str(exe)])
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "bad 0" in out.stdout
