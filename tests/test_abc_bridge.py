"""The ABC-patch front end (CULS src/abc_patch/: gget, gput, grw, gst, gb,
gps) is written against a neutral view of an ABC network
(culs_b200/abc_patch/abc_bridge.hpp) so that it is tested here without ABC,
whose tree is absent: tests/native/abc_bridge_check.cpp drives it with a
mock network whose AND constructor folds and merges as Abc_AigAnd does.
The ABC adapter itself (culs_abc_patch.cpp) is compiled only against a real
ABC tree."""
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
LIB = ROOT / "culs_b200" / "libculs_b200.so"


def build(tmp_path):
    if shutil.which("g++") is None or not LIB.exists():
        pytest.skip("needs g++ and the built library")
    exe = tmp_path / "abc_bridge_check"
    subprocess.check_call(["g++", "-O2", "-std=c++17", "-I", str(ROOT / "culs_b200" / "abc_patch"),
                           "-I", str(ROOT / "include"), str(ROOT / "tests" / "native" / "abc_bridge_check.cpp"),
                           "-o", str(exe), "-L", str(LIB.parent), "-lculs_b200", f"-Wl,-rpath,{LIB.parent}"])
    return exe


def test_network_conversions_round_trip(tmp_path):
    """gput's construction then gget's numbering keeps every output's
    function, folds constants and duplicates as a strashing constructor
    does, and refuses AND nodes out of DFS order and cyclic fanins."""
    out = subprocess.run([str(build(tmp_path))], capture_output=True, text=True)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "bad 0" in out.stdout


@pytest.mark.gpu
def test_abc_commands_through_the_library(tmp_path):
    """gget; grw; gst; grw -z -d; gb; grw; grw; gst -c; gps; gput on a mock
    network keeps the outputs' functions; gb -s, gresyn2 and an unknown
    option fail as ABC commands do (return 1), as does grw before gget."""
    out = subprocess.run([str(build(tmp_path)), "--gpu"], capture_output=True, text=True)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "bad 0" in out.stdout and out.stdout.count("gpu:") == 3
