"""Host-side checks that need no GPU: the C ABI library loads and exports
every entry point of include/culs_b200.h, AIGER I/O, generators, the
embedded rewriting library."""
import ctypes
import hashlib
import os
import re
import struct
from pathlib import Path

import numpy as np
import pytest

import culs_b200 as C

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "culs_b200.h"


def header_functions():
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    return sorted(set(re.findall(r"\b(culs_\w+)\s*\(", text)))


def test_library_exports_every_header_symbol():
    lib = ctypes.CDLL(str(C.LIB_PATH))
    names = header_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_embedded_library_digest():
    blob = (ROOT / "culs_b200" / "data" / "rwlib.bin").read_bytes()
    assert blob[:8] == b"CULSRWL1"
    from culs_b200.data import make_rwlib
    assert blob[8:40].hex() == make_rwlib.EXPECTED_SHA
    assert len(blob) == 40 + 218008


def test_aiger_roundtrip(tmp_path):
    for g in [C.gen_multiplier(6), C.gen_layered(3, 20, 10, 800, 20, 4, 0.1, True)]:
        p = tmp_path / "x.aig"
        C.write_aiger(p, g)
        h = C.read_aiger(p)
        assert h.nPIs == g.nPIs and h.nPOs == g.nPOs
        assert np.array_equal(h.fanin0, g.fanin0) and np.array_equal(h.fanin1, g.fanin1)
        assert np.array_equal(h.outs, g.outs)


def test_aiger_constants_and_header(tmp_path):
    # one AND of PI1 and TRUE, POs: the AND, constant FALSE, constant TRUE
    g = C.Aig(1, np.array([-1, -1, 2], np.int32), np.array([-1, -1, 0], np.int32), np.array([4, 1, 0], np.int32))
    p = tmp_path / "c.aig"
    C.write_aiger(p, g)
    raw = p.read_bytes()
    assert raw.startswith(b"aig 2 1 0 3 1\n4\n0\n1\n")  # AIGER constants are the other way round
    h = C.read_aiger(p)
    assert np.array_equal(h.outs, g.outs)
    assert sorted([int(h.fanin0[2]), int(h.fanin1[2])]) == [0, 2]


@pytest.mark.parametrize("content", [b"", b"aag 1 1 0 1 0\n2\n", b"aig 1 1 1 1 0\n2\n", b"aig 3 1 0 1 1\n2\n",
                                     b"aig 2 1 0 1 1\n4\n\x01"])
def test_aiger_rejects_malformed(tmp_path, content):
    p = tmp_path / "bad.aig"
    p.write_bytes(content)
    with pytest.raises(C.CulsError) as e:
        C.read_aiger(p)
    assert e.value.code == -6


def test_aiger_missing_file(tmp_path):
    with pytest.raises(C.CulsError):
        C.read_aiger(tmp_path / "nope.aig")


def _check_strashed(g):
    n = g.nObjs
    keys = set()
    for v in range(g.nPIs + 1, n):
        a, b = int(g.fanin0[v]), int(g.fanin1[v])
        assert 0 <= (a >> 1) < v and 0 <= (b >> 1) < v  # topological
        assert (a >> 1) != (b >> 1) and (a >> 1) != 0 and (b >> 1) != 0
        k = (min(a, b), max(a, b))
        assert k not in keys
        keys.add(k)


def test_generators_deterministic_and_strashed():
    a = C.gen_layered(1, 64, 32, 5000, 40, 4, 0.0, True)
    b = C.gen_layered(1, 64, 32, 5000, 40, 4, 0.0, True)
    assert np.array_equal(a.fanin0, b.fanin0) and np.array_equal(a.outs, b.outs)
    assert a.nPIs == 64 and a.nPOs == 32 and 2000 < a.nAnds <= 5000
    _check_strashed(a)
    m = C.gen_multiplier(64)
    assert m.nPIs == 128 and m.nPOs == 128 and 30000 < m.nAnds < 45000
    _check_strashed(m)


def test_generator_refuses_impossible_shape():
    """176 AND nodes in a first layer over 9 PIs (only 144 distinct
    complemented fanin pairs exist there): an error code, not an abort."""
    with pytest.raises(C.CulsError) as e:
        C.gen_layered(201, 9, 11, 1408, 8, 3, 0.0, True)
    assert e.value.code == C.CULS_E_INVALID


def test_host_allocation_failure_is_an_error_code():
    """A C entry point whose host allocation fails returns CULS_E_OOM instead
    of letting std::bad_alloc end the process (run in a child process whose
    address space is capped 512 MiB above its size at start)."""
    import subprocess
    import sys
    import textwrap
    code = textwrap.dedent("""
        import resource, culs_b200 as C
        size = next(int(l.split()[1]) * 1024 for l in open("/proc/self/status") if l.startswith("VmSize"))
        resource.setrlimit(resource.RLIMIT_AS, (size + (512 << 20), size + (512 << 20)))
        try:
            C.gen_layered(1, 64, 32, 50_000_000, 7000, 4, 0.0, True)
            print("generated")
        except C.CulsError as e:
            print("error", e.code)
    """)
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=120,
                       cwd=os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    assert r.returncode == 0, r.stderr[-500:]
    assert r.stdout.split() == ["error", str(C.CULS_E_OOM)]


def test_gen_batch_matches_sequential():
    par = C.gen_batch(4, 0, 6, 1000, 5000, 16, 512, threads=4)
    seq = C.gen_batch(4, 0, 6, 1000, 5000, 16, 512, threads=1)
    for x, y in zip(par, seq):
        assert np.array_equal(x.fanin0, y.fanin0)
    sizes = [g.nAnds for g in par]
    assert all(1000 <= s <= 5000 for s in sizes)


def test_context_fails_loudly_without_gpu():
    if os.path.exists("/dev/nvidia0") or os.path.exists("/dev/nvidiactl"):
        pytest.skip("a GPU is present")
    with pytest.raises(C.CulsError) as e:
        C.Context()
    assert e.value.code == -5


def _gpuls():
    exe = ROOT / "culs_b200" / "gpuls"
    if not exe.exists():
        pytest.skip("gpuls not built (python culs_b200/build.py)")
    return exe


def test_cli_command_surface_without_graph():
    """The gpuls-compatible CLI parses the reference's script syntax and
    answers the commands that need no device the way gpuls does."""
    import subprocess
    out = subprocess.run([str(_gpuls()), "-c", "ps; time; b; foo; rw -q; write x.txt"], capture_output=True,
                         text=True, timeout=60).stdout.splitlines()
    assert out[0] == 'Running in script mode: "ps; time; b; foo; rw -q; write x.txt".'
    assert "AIG stats: i/o = 0/0 and = 0 level = 0" in out
    assert any(l.startswith("{time} prev cmd: alg 0.00 s, full 0.00 s;") for l in out)
    assert "Command foo not registered, ignored." in out
    assert "Command rw not recognized or in wrong format!" in out
    assert "write: only support .aig format!" in out
