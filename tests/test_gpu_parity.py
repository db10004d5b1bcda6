"""GPU path (libculs_b200.so through the C ABI) against the oracle and
against the reference's golden fixtures.  Integer work: every comparison is
exact (tolerance 0)."""
import hashlib
import json
import os
from pathlib import Path

import numpy as np
import pytest

import aigcanon
import culs_b200 as C
from oracle.oracle import Oracle
from oracle import oracle as O
from util import oracle_rw_st, same_graph, to_oracle

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"


@pytest.fixture(scope="module")
def ctx():
    c = C.Context()
    yield c
    c.close()


def random_unstrashed(seed, nPIs, nAnds, nPOs, pconst=0.05, pdup=0.05):
    """Topological AIG with constant fanins, x&x / x&!x nodes, duplicate
    nodes, dangling nodes and PO literals on constants and PIs."""
    rng = np.random.default_rng(seed)
    n = 1 + nPIs + nAnds
    f0 = np.full(n, -1, np.int32)
    f1 = np.full(n, -1, np.int32)
    for v in range(nPIs + 1, n):
        if v > nPIs + 2 and rng.random() < pdup:
            u = int(rng.integers(nPIs + 1, v))
            f0[v], f1[v] = f0[u], f1[u]
            continue
        def lit():
            if rng.random() < pconst:
                return int(rng.integers(0, 2))
            return int(2 * rng.integers(1, v) + rng.integers(0, 2))
        a = lit()
        b = a if rng.random() < 0.03 else (a ^ 1 if rng.random() < 0.03 else lit())
        f0[v], f1[v] = min(a, b), max(a, b)
    outs = np.array([int(rng.integers(0, 2 * n)) for _ in range(nPOs)], np.int32)
    return C.Aig(nPIs, f0, f1, outs)


def edge_graphs():
    gs = {}
    gs["no_ands"] = C.Aig(3, np.full(4, -1, np.int32), np.full(4, -1, np.int32), np.array([0, 1, 2, 7], np.int32))
    gs["no_pos"] = C.Aig(4, *[np.concatenate([np.full(5, -1), x]).astype(np.int32)
                              for x in ([2, 4, 10], [4, 6, 12])], np.zeros(0, np.int32))
    gs["single_and"] = C.Aig(2, np.array([-1, -1, -1, 2], np.int32), np.array([-1, -1, -1, 5], np.int32),
                             np.array([7, 6], np.int32))
    for s in range(6):
        gs[f"unstrashed{s}"] = random_unstrashed(s, 6 + s, 200 + 150 * s, 4 + s)
    gs["mult6"] = C.gen_multiplier(6)
    gs["mult12"] = C.gen_multiplier(12)
    gs["c1"] = C.gen_layered(1, 64, 32, 5000, 40, 4, 0.0, True)
    gs["far20k"] = C.gen_layered(7, 100, 50, 20000, 60, 3, 0.2, False)
    return gs


GRAPHS = edge_graphs()


def gpu_run(ctx, g, ops):
    d = ctx.upload(g)
    for op in ops:
        op(ctx, d)
    return d.download()


def oracle_run(g, ops):
    o = Oracle()
    o.set_graph(to_oracle(g))
    for op in ops:
        op(o)
    return o.graph()


FLOWS = {
    "rw;st": ([lambda c, d: c.rw(d), lambda c, d: c.st(d)], [lambda o: o.rw(), lambda o: o.st()]),
    "rw -z;st": ([lambda c, d: c.rw(d, zeros=True), lambda c, d: c.st(d)],
                 [lambda o: o.rw(zeros=True), lambda o: o.st()]),
    "st": ([lambda c, d: c.st(d)], [lambda o: o.st()]),
    "st -c": ([lambda c, d: c.st(d, cpu=True)], [lambda o: o.st(cpu=True)]),
    "rw (cpu dedup)": ([lambda c, d: c.rw(d, gpu_dedup=False)], [lambda o: o.rw(dedup=1)]),
    "rw;rw;st": ([lambda c, d: c.rw(d), lambda c, d: c.rw(d), lambda c, d: c.st(d)],
                 [lambda o: o.rw(), lambda o: o.rw(), lambda o: o.st()]),
}


@pytest.mark.parametrize("flow", list(FLOWS))
@pytest.mark.parametrize("name", list(GRAPHS))
def test_gpu_matches_oracle(ctx, name, flow):
    g = GRAPHS[name]
    gops, oops = FLOWS[flow]
    a = gpu_run(ctx, g, gops)
    b = oracle_run(g, oops)
    assert same_graph(a, b), f"{name} {flow}: gpu {a.nAnds} ands vs oracle {b.nAnds}"
    if g.nAnds:
        assert a.nLevels == b.nLevels


@pytest.mark.parametrize("name", ["mult12", "c1", "far20k", "unstrashed3", "unstrashed5"])
def test_gpu_per_node_dumps_match_oracle(ctx, name):
    g = GRAPHS[name]
    d = ctx.upload(g)
    ctx.rw(d, dump=True)
    D = ctx.dump()
    st = ctx.rw_stats()
    o = Oracle()
    o.set_graph(to_oracle(g))
    o.rw()
    f0, f1, outs = o.dump_reorder(g.nPOs)
    np.testing.assert_array_equal(D["reorder_f0"], f0)
    np.testing.assert_array_equal(D["reorder_f1"], f1)
    np.testing.assert_array_equal(D["reorder_out"], outs)
    np.testing.assert_array_equal(D["cuts"].reshape(-1, 8, 9), o.dump_cuts())
    np.testing.assert_array_equal(D["selected"].reshape(-1, 10), o.dump_selected())
    rep, nf0, nf1 = o.dump_replace()
    np.testing.assert_array_equal(D["replace"], rep)
    np.testing.assert_array_equal(D["new_f0"], nf0)
    np.testing.assert_array_equal(D["new_f1"], nf1)
    np.testing.assert_array_equal(D["choice"], o.dump_choice())
    ost = o.dump_stats()
    for k in ["replaced", "replaced_pos", "replaced_zero", "reverted", "compromised", "expected"]:
        assert st[k] == ost[k], k


def test_batch_equals_single(ctx):
    names = ["no_ands", "mult6", "unstrashed2", "no_pos", "c1", "single_and", "unstrashed4"]
    gs = [GRAPHS[n] for n in names]
    db = ctx.upload_batch(gs)
    ctx.rw_st(db)
    assert len(db) == len(gs)
    for i, g in enumerate(gs):
        single = gpu_run(ctx, g, FLOWS["rw;st"][0])
        got = db.download(i)
        assert same_graph(got, single), names[i]
        assert got.nLevels == single.nLevels


@pytest.mark.parametrize("name", sorted(p.stem for p in GOLDEN.glob("*.npz") if p.stem not in ("chains", "balance")))
def test_gpu_matches_reference_fixture(ctx, name):
    f = dict(np.load(GOLDEN / f"{name}.npz"))
    g = C.Aig(int(f["nPIs"]), f["in_f0"], f["in_f1"], f["in_outs"])
    d = ctx.upload(g)
    ctx.rw(d, dump=True)
    D = ctx.dump()
    assert aigcanon.digest(D["cuts"]) == str(f["cuts_sha"])
    assert aigcanon.digest(D["selected"]) == str(f["selected_sha"])
    stats = ctx.rw_stats()
    assert [stats[k] for k in ["replaced", "replaced_pos", "replaced_zero", "reverted", "compromised"]] == \
        [int(x) for x in f["z0_stats"][:5]]
    ctx.st(d)
    out = d.download()
    assert (out.nAnds, out.nLevels) == tuple(int(x) for x in f["z0_st"])
    ands, pos = aigcanon.signature(out.nPIs, out.fanin0, out.fanin1, out.outs)
    assert hashlib.sha256(json.dumps([ands, pos]).encode()).hexdigest() == str(f["z0_sig"])


def test_large_single_graph_matches_oracle(ctx):
    g = C.gen_layered(3, 4096, 4096, 1_000_000, 200, 3, 0.2, False)
    a = gpu_run(ctx, g, FLOWS["rw;st"][0])
    b = oracle_rw_st(g).graph()
    assert same_graph(a, b)
    assert a.nLevels == b.nLevels


def _digest(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(np.asarray(a, np.int32)).tobytes())
    return h.hexdigest()


def test_full_size_single_graph_matches_oracle_digest(ctx):
    """The 10M-AND single-graph workload (seeded layered AIG, 4,096 PIs and
    POs, 2,000 layers, 80% window-3 / 20% far fanins): the CUDA path's `rw;
    st` result equals the oracle's exactly, checked through the SHA-256 of
    its fanin and output arrays recorded by tests/golden/make_c3_digest.py
    (the oracle takes about a minute of CPU per pass at this size)."""
    rec = json.loads((GOLDEN / "c3_layered10M.json").read_text())
    g = C.gen_layered(*rec["args"])
    assert _digest(g.fanin0, g.fanin1, g.outs) == rec["input"]["sha256"]
    d = ctx.upload(g)
    ctx.rw_st(d)
    out = d.download()
    d.free()
    want = rec["rw_st"]
    assert (out.nAnds, out.nLevels, out.nPOs) == (want["nAnds"], want["nLevels"], want["nPOs"])
    assert _digest(out.fanin0, out.fanin1, out.outs) == want["sha256"]


def test_wide_c4_family_batch_equals_plain_path_and_oracle(ctx):
    """256 graphs of the batched workload's family (AND counts log-uniform
    1k-200k) plus two 200k-AND members, in one batch: every graph's result
    equals the plain single-graph path on the same graph, node for node, and
    the largest graphs and a spread sample equal the oracle."""
    from concurrent.futures import ThreadPoolExecutor
    gs = C.gen_batch(4, 0, 256, 1000, 200_000, 16, 512, threads=8)
    gs += C.gen_batch(4, 9000, 2, 200_000, 200_000, 16, 512, threads=8)
    assert max(g.nAnds for g in gs) > 150_000
    db = ctx.upload_batch(gs)
    ctx.rw_st(db)
    outs = db.download_all()
    for i, g in enumerate(gs):
        d = ctx.upload(g)
        ctx.rw_st(d)
        assert same_graph(outs[i], d.download()), i
        d.free()
    db.free()
    by_size = sorted(range(len(gs)), key=lambda i: -gs[i].nAnds)
    sample = by_size[:6] + by_size[6::16]
    with ThreadPoolExecutor(max_workers=min(16, os.cpu_count() or 4)) as ex:
        refs = list(ex.map(lambda i: oracle_rw_st(gs[i]).graph(), sample))
    for i, r in zip(sample, refs):
        assert same_graph(outs[i], r), i


def test_batch_of_generated_graphs_matches_oracle(ctx):
    gs = C.gen_batch(4, 0, 24, 1000, 20000, 16, 512, threads=8)
    db = ctx.upload_batch(gs)
    ctx.rw_st(db)
    for i, g in enumerate(gs):
        assert same_graph(db.download(i), oracle_rw_st(g).graph()), i


def _host_depth(g):
    lev = np.zeros(g.nObjs, np.int64)
    for v in range(g.nPIs + 1, g.nObjs):
        lev[v] = 1 + max(lev[int(g.fanin0[v]) >> 1], lev[int(g.fanin1[v]) >> 1])
    return int(lev.max()) if g.nObjs else 0


def test_batch_transfers_agree(ctx):
    """Upload computes every graph's depth on several host threads; the batch
    sizes equal the per-graph ones; the three download paths (per graph, into
    caller arrays, library-allocated) return the same arrays."""
    gs = C.gen_batch(4, 100, 40, 1000, 60000, 16, 512, threads=8)
    db = ctx.upload_batch(gs)
    for i, g in enumerate(gs):
        assert db.stats(i)["nLevels"] == _host_depth(g), i
    ctx.rw_st(db)
    allst = db.stats_all()  # culs_batch_stats equals culs_graph_stats per graph
    for i in range(len(db)):
        assert {k: int(v[i]) for k, v in allst.items()} == db.stats(i), i
    whole = db.download_all()
    arr = (C._HostGraph * len(db))()
    assert C._lib.culs_batch_download(ctx.h, db.h, arr) == 0
    for i in range(len(db)):
        one = db.download(i)
        lib = C._take(arr[i])
        for got in (whole[i], lib):
            np.testing.assert_array_equal(got.fanin0, one.fanin0)
            np.testing.assert_array_equal(got.fanin1, one.fanin1)
            np.testing.assert_array_equal(got.outs, one.outs)
        assert whole[i].nLevels == one.nLevels


def test_cli_script_matches_library(ctx, tmp_path):
    """gpuls -c "read; rw; st; ps; write" gives the oracle's rw;st result."""
    import subprocess
    exe = Path(__file__).resolve().parents[1] / "culs_b200" / "gpuls"
    g = C.gen_layered(11, 48, 24, 6000, 40, 4, 0.0, True)
    src, dst = tmp_path / "in.aig", tmp_path / "out.aig"
    C.write_aiger(src, g)
    r = subprocess.run([str(exe), "-c", f"read {src}; rw; st; ps; write {dst}"], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    out = C.read_aiger(dst)
    ref = oracle_rw_st(g).graph()
    assert same_graph(out, ref)
    assert f"AIG stats: i/o = {g.nPIs}/{len(g.outs)} and = {ref.nAnds} level = {ref.nLevels}" in r.stdout


def test_rewrite_preserves_function(ctx):
    for g in [GRAPHS["mult12"], GRAPHS["c1"], GRAPHS["unstrashed5"], C.gen_multiplier(32)]:
        out = gpu_run(ctx, g, FLOWS["rw;st"][0])
        assert O.equivalent_sim(to_oracle(g), to_oracle(out), words=8)
        assert out.nAnds <= g.nAnds or g.nAnds == 0


def test_budget_refusal(ctx):
    small = C.Context(hbm_budget=1 << 20)
    d = small.upload(C.gen_multiplier(64))
    with pytest.raises(C.CulsError) as e:
        small.rw(d)
    assert e.value.code == -3
    small.close()


def test_strash_probe_cap_reports_and_leaves_graph(ctx, monkeypatch):
    """A strash table too small for the graph: the bounded probes run out, the
    call reports CULS_E_PROBE, the graph stays as it was and the context keeps
    working (the status word is cleared)."""
    g = C.gen_multiplier(32)
    d = ctx.upload(g)
    monkeypatch.setenv("CULS_STRASH_TABLE_CAP", "1024")
    with pytest.raises(C.CulsError) as e:
        ctx.st(d)
    assert e.value.code == C.CULS_E_PROBE
    monkeypatch.delenv("CULS_STRASH_TABLE_CAP")
    assert same_graph(d.download(), g)
    ctx.rw(d)
    ctx.st(d)
    assert same_graph(d.download(), oracle_rw_st(g).graph())
    d.free()


def test_expired_waits_report_probe_quickly_and_leave_graph(ctx, monkeypatch):
    """CULS_SPIN_LIMIT=1: a dependency wait that is not satisfied at its first
    look runs out.  On a deep layered graph the rewrite's dataflow kernels
    wait, so the call reports CULS_E_PROBE; once one wait has failed the
    others give up at once instead of spinning out their own bound, so the
    error comes back quickly.  The graph stays as it was and, with the bound
    restored, the context runs rw; st and equals the oracle."""
    import time
    g = C.gen_layered(11, 64, 32, 200_000, 2000, 3, 0.2, False)
    d = ctx.upload(g)
    monkeypatch.setenv("CULS_SPIN_LIMIT", "1")
    t0 = time.perf_counter()
    with pytest.raises(C.CulsError) as e:
        ctx.rw(d)
    dt = time.perf_counter() - t0
    assert e.value.code == C.CULS_E_PROBE
    assert dt < 5.0
    with pytest.raises(C.CulsError) as e:
        ctx.st(d)
    assert e.value.code == C.CULS_E_PROBE
    monkeypatch.delenv("CULS_SPIN_LIMIT")
    assert same_graph(d.download(), g)
    ctx.rw(d)
    ctx.st(d)
    assert same_graph(d.download(), oracle_rw_st(g).graph())
    d.free()


def test_batch_beyond_30_bit_positions_is_refused(ctx):
    """Node positions are 30-bit: a batch of 3 x 200M AND nodes is refused
    with CULS_E_INVALID from its sizes alone, before any array is read (each
    graph here passes 4-element arrays)."""
    one = np.zeros(4, np.int32)
    hg = (C._HostGraph * 3)()
    for h in hg:
        h.nPIs, h.nPOs, h.nAnds = 1, 0, 200_000_000
        h.fanin0 = h.fanin1 = h.outs = one.ctypes.data_as(C._ip)
    out = C._vp()
    assert C._lib.culs_batch_upload(ctx.h, 3, hg, C.ctypes.byref(out)) == C.CULS_E_INVALID
    assert out.value is None


def test_invalid_graph_rejected(ctx):
    bad = C.Aig(2, np.array([-1, -1, -1, 8], np.int32), np.array([-1, -1, -1, 2], np.int32), np.array([6], np.int32))
    with pytest.raises(C.CulsError) as e:
        ctx.upload(bad)
    assert e.value.code == -1


def test_graph_deeper_than_16_bit_levels_matches_oracle():
    """A graph over 65,535 levels deep, alone and inside a batch of shallow
    ones: evaluation keeps library-node levels in 32 bits there (16 bits
    otherwise), with the same results."""
    deep = C.gen_layered(31, 8, 4, 200000, 100000, 2, 0.0, True)  # 96k ANDs, depth 70,687
    shallow = C.gen_batch(4, 500, 3, 1000, 20000, 16, 256, threads=8)
    c = C.Context()
    try:
        d = c.upload(deep)
        c.rw_st(d)
        ref = oracle_rw_st(deep).graph()
        out = d.download()
        assert same_graph(out, ref)
        assert out.nLevels == ref.nLevels
        db = c.upload_batch(shallow + [deep])
        c.rw_st(db)
        for i, g in enumerate(shallow + [deep]):
            assert same_graph(db.download(i), oracle_rw_st(g).graph()), i
    finally:
        c.close()


@pytest.mark.parametrize("wide_min", [1, 1 << 30])
def test_both_enumeration_schedules_match_oracle(wide_min):
    """Every level on one thread per node (1), or every level on one warp per
    node (2^30): the enumeration schedule changes speed, never results."""
    c = C.Context()
    try:
        c.set_param("enum_wide_min", wide_min)
        for name in ["mult12", "c1", "unstrashed3", "far20k"]:
            g = GRAPHS[name]
            d = c.upload(g)
            c.rw(d, dump=True)
            D = c.dump()
            # pairs replayed by the warp-per-node schedule: none when every
            # level runs one node per thread
            assert (c.rw_stats()["enum_warp_pairs"] > 0) == (wide_min > 1), name
            o = Oracle()
            o.set_graph(to_oracle(g))
            o.rw()
            np.testing.assert_array_equal(D["cuts"].reshape(-1, 8, 9), o.dump_cuts())
            c.st(d)
            assert same_graph(d.download(), oracle_rw_st(g).graph()), name
        gs = C.gen_batch(4, 300, 12, 1000, 30000, 16, 512, threads=8)
        db = c.upload_batch(gs)
        c.rw_st(db)
        for i, g in enumerate(gs):
            assert same_graph(db.download(i), oracle_rw_st(g).graph()), i
    finally:
        c.close()


def test_autotune_keeps_results():
    c = C.Context()
    try:
        gs = C.gen_batch(4, 400, 16, 1000, 30000, 16, 512, threads=8)
        sample = c.upload_batch(gs)
        chosen = c.autotune(sample)
        assert chosen["enum_wide_min"] in (2048, 4096, 8192, 16384, 32768, 65536, 1 << 30)
        assert chosen["enum_blocks_per_sm"] in (4, 6, 8, 12, 16)
        assert chosen["eval_group_mslots"] in (4, 8, 16, 32, 64)
        c.rw_st(sample)  # the sample itself is left unchanged by the tuner
        for i, g in enumerate(gs):
            assert same_graph(sample.download(i), oracle_rw_st(g).graph()), i
    finally:
        c.close()


def test_evaluation_groups_do_not_change_results():
    """The evaluation builds and probes the existence tables of a group of
    graphs at a time (a speed parameter): groups of at most 1M table slots
    split this 36-graph batch (3.3M slots) into four, with the oracle's
    graphs as the result."""
    c = C.Context()
    try:
        c.set_param("eval_group_mslots", 1)
        assert c.get_param("eval_group_mslots") == 1
        gs = C.gen_batch(4, 500, 36, 5000, 60000, 16, 512, threads=8)
        db = c.upload_batch(gs)
        c.rw_st(db)
        for i, g in enumerate(gs):
            assert same_graph(db.download(i), oracle_rw_st(g).graph()), i
    finally:
        c.close()
