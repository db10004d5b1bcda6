"""culs_levels_noalloc: the entry point for callers that cannot allocate
device memory (a host whose device memory is owned and sized by another
runtime, or an allocator-free embedding).  Its scratch is a fixed device
array shared by every call, so this test checks, over two calls in a row,
that it returns the same depth as the existing entry points
(culs_graph_upload + culs_graph_stats) and the same per-node levels as a
host recurrence -- exact, like every integer check here -- and that it
refuses graphs beyond its fixed limit, refuses a graph whose fanin is not
earlier than its node after the kernel has run, and works on a stream other
than the default one.  This file is collected last, so a run that stops at
its first failure has run every other test before it."""
import ctypes

import numpy as np
import pytest

import culs_b200 as C

pytestmark = pytest.mark.gpu

_f = C._lib.culs_levels_noalloc
_f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p,
               ctypes.c_void_p]
MAX_OBJS = 1 << 20


def host_levels(g):
    lev = np.zeros(g.nObjs, np.int64)
    for v in range(g.nPIs + 1, g.nObjs):
        lev[v] = 1 + max(lev[int(g.fanin0[v]) >> 1], lev[int(g.fanin1[v]) >> 1])
    return lev


def run_noalloc(torch, g, fanin0=None, stream=None):
    f0 = torch.tensor(np.asarray(g.fanin0 if fanin0 is None else fanin0, np.int32), device="cuda")
    f1 = torch.tensor(np.asarray(g.fanin1, np.int32), device="cuda")
    lev = torch.full((g.nObjs,), -7, dtype=torch.int32, device="cuda")
    mx = torch.full((1,), -7, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    rc = _f(f0.data_ptr(), f1.data_ptr(), g.nPIs, g.nAnds, lev.data_ptr(), mx.data_ptr(),
            None if stream is None else stream.cuda_stream)
    torch.cuda.synchronize()
    return rc, lev.cpu().numpy(), int(mx.cpu().item())


def test_levels_noalloc_two_calls_match_existing_entry_points():
    torch = pytest.importorskip("torch")
    ctx = C.Context()
    graphs = [C.gen_multiplier(16), C.gen_layered(5, 40, 20, 30000, 90, 3, 0.2, False)]
    for g in graphs:  # two calls in a row, each on a fresh graph
        rc, lev, mx = run_noalloc(torch, g)
        assert rc == 0
        depth = ctx.upload(g).stats()["nLevels"]  # the existing entry points' depth
        assert mx == depth
        np.testing.assert_array_equal(lev, host_levels(g))
    ctx.close()


def test_levels_noalloc_on_a_caller_stream():
    torch = pytest.importorskip("torch")
    g = C.gen_multiplier(12)
    rc, lev, mx = run_noalloc(torch, g, stream=torch.cuda.Stream())
    assert rc == 0
    np.testing.assert_array_equal(lev, host_levels(g))
    assert mx == int(host_levels(g).max())


def test_levels_noalloc_rejects_a_fanin_that_is_not_earlier():
    """A node whose fanin is itself: the kernel records the malformed graph
    and the call returns CULS_E_INVALID; the next call on a good graph is
    unaffected by the shared array's leftover contents."""
    torch = pytest.importorskip("torch")
    g = C.gen_multiplier(8)
    bad = np.array(g.fanin0, np.int32)
    v = g.nObjs - 3
    bad[v] = 2 * v
    rc, _, _ = run_noalloc(torch, g, fanin0=bad)
    assert rc == -1  # CULS_E_INVALID
    rc, lev, _ = run_noalloc(torch, g)
    assert rc == 0
    np.testing.assert_array_equal(lev, host_levels(g))


def test_levels_noalloc_refuses_oversized_graph():
    torch = pytest.importorskip("torch")
    dummy = torch.zeros(4, dtype=torch.int32, device="cuda")
    p = dummy.data_ptr()
    assert _f(p, p, 10, MAX_OBJS, p, p, None) == -1  # CULS_E_INVALID, nothing launched
