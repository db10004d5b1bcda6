"""Binary AIGER decoded and encoded on the device (culs_batch_upload_aiger,
culs_batch_download_aiger) against the host reader and writer
(culs_aiger_read / culs_aiger_write, the rules of AIGMan::readFromMemory and
AIGMan::saveFile, CULS src/aig_manager.cu:110-267): the same arrays, the
same depth, the same bytes, and CULS_E_IO for what the host reader refuses."""
import numpy as np
import pytest

import culs_b200 as C
from util import oracle_rw_st, same_graph

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = C.Context()
    yield c
    c.close()


def graphs():
    gs = [C.gen_multiplier(8), C.gen_multiplier(32), C.gen_layered(41, 64, 32, 20000, 60, 4, 0.0, True),
          C.gen_layered(42, 300, 40, 150000, 80, 3, 0.3, False)]
    gs += C.gen_batch(4, 900, 6, 1000, 40000, 16, 512, threads=8)
    # no AND nodes; no POs; POs on the constants and on PIs
    gs.append(C.Aig(3, np.array([-1] * 4, np.int32), np.array([-1] * 4, np.int32), np.array([0, 1, 2, 7], np.int32)))
    m = C.gen_multiplier(4)
    gs.append(C.Aig(m.nPIs, m.fanin0, m.fanin1, np.zeros(0, np.int32)))
    return gs


def host_bytes(g, tmp_path, name):
    p = tmp_path / f"{name}.aig"
    C.write_aiger(p, g)
    return p.read_bytes()


def host_depth(g):
    f0 = np.asarray(g.fanin0) >> 1
    f1 = np.asarray(g.fanin1) >> 1
    lev = np.zeros(len(f0), np.int64)
    for i in range(1 + g.nPIs, len(f0)):
        lev[i] = 1 + max(lev[f0[i]], lev[f1[i]])
    return int(lev.max()) if len(f0) > 1 + g.nPIs else 0


def test_device_decode_equals_host_reader(ctx, tmp_path):
    gs = graphs()
    files = [host_bytes(g, tmp_path, f"g{i}") for i, g in enumerate(gs)]
    d = ctx.upload_aiger_batch(files)
    got = d.download_all()
    for i, (g, f) in enumerate(zip(gs, files)):
        p = tmp_path / f"r{i}.aig"
        p.write_bytes(f)
        ref = C.read_aiger(p)
        assert same_graph(got[i], ref), i
        assert d.stats(i)["nLevels"] == host_depth(ref), i
    d.free()


def test_device_encode_equals_host_writer(ctx, tmp_path):
    gs = graphs()
    d = ctx.upload_batch(gs)
    out = d.download_aiger_all()
    for i, g in enumerate(gs):
        assert out[i] == host_bytes(g, tmp_path, f"w{i}"), i
    # the library-allocated form gives the same bytes
    ptrs = (C._vp * len(gs))()
    lens = (C.ctypes.c_size_t * len(gs))()
    assert C._lib.culs_batch_download_aiger(ctx.h, d.h, ptrs, lens) == 0
    for i in range(len(gs)):
        assert C.ctypes.string_at(ptrs[i], lens[i]) == out[i], i
        C._lib.culs_buffer_free(ptrs[i])
    # after rw; st, and decoded again on the device
    ctx.rw_st(d)
    res = d.download_all()
    enc = d.download_aiger_all()
    for i, g in enumerate(gs):
        assert same_graph(res[i], oracle_rw_st(g).graph()), i
        assert enc[i] == host_bytes(res[i], tmp_path, f"x{i}"), i
    d2 = ctx.upload_aiger_batch(enc)
    back = d2.download_all()
    for i in range(len(gs)):
        assert same_graph(back[i], res[i]), i
    d.free()
    d2.free()


def test_large_deltas_round_trip(ctx, tmp_path):
    """Fanins far below their node (1.1M PIs): three- and four-byte numbers."""
    rng = np.random.default_rng(43)
    nPIs, nA = 1_100_000, 5000
    f0 = np.full(1 + nPIs + nA, -1, np.int32)
    f1 = f0.copy()
    for k in range(nA):
        i = 1 + nPIs + k
        a, b = (1, i - 1) if k % 10 == 0 else rng.integers(1, i, 2)  # delta1 above 2^21: four bytes
        if a == b:
            b = i - 1 if a != i - 1 else 1
        f0[i], f1[i] = 2 * a + int(rng.integers(2)), 2 * b + int(rng.integers(2))
    g = C.Aig(nPIs, f0, f1, (2 * np.arange(1 + nPIs + nA - 8, 1 + nPIs + nA)).astype(np.int32))
    b = host_bytes(g, tmp_path, "far")
    body = b[len(b"aig ") + b[4:].index(b"\n") + 1:]
    assert any(body[k] & 0x80 and body[k + 1] & 0x80 and body[k + 2] & 0x80 for k in range(len(body) - 3))
    d = ctx.upload_aiger_batch([b])
    assert same_graph(d.download(), C.read_aiger(tmp_path / "far.aig"))
    assert d.download_aiger_all()[0] == b
    d.free()


def test_malformed_files_are_refused(ctx, tmp_path):
    ok = host_bytes(C.gen_multiplier(6), tmp_path, "ok")
    head_end = ok.index(b"\n") + 1
    body = ok.index(b"c\n", len(ok) - 2)
    bad = {
        "not aiger": b"aag 3 2 0 1 1\n2\n4\n6\n6 2 4\n",
        "latches": b"aig 3 2 1 1 0\n" + ok[head_end:],
        "truncated numbers": ok[:body - 3],
        "zero delta (fanin not below its node)": b"aig 3 2 0 1 1\n6\n" + b"\x00\x02c\n",
        "six-byte number": b"aig 3 2 0 1 1\n6\n" + b"\x80\x80\x80\x80\x80\x01\x02c\n",
    }
    for name, data in bad.items():
        with pytest.raises(C.CulsError) as e:
            ctx.upload_aiger_batch([ok, data])
        assert e.value.code == C.CULS_E_IO, name
        # the host reader refuses it too
        p = tmp_path / "bad.aig"
        p.write_bytes(data)
        with pytest.raises(C.CulsError):
            C.read_aiger(p)
    # the context stays usable
    d = ctx.upload_aiger_batch([ok])
    assert d.download_aiger_all()[0] == ok
    d.free()
