"""Levels of the rewrite's deduplication (the strash that ends
AIGMan::rewrite, src/aig_manager.cu:454-546).  The default computes them in
in-order passes over a nearly topological order of the rewritten batch; the
level-synchronous worklist, its fallback, runs alone when
CULS_DEDUP_WORKLIST is set.  Both must give the same graphs, equal to the
oracle, for GPU- and CPU-deduplicating rewrites and for a second rewrite
that starts from the kept manager graph.  The same holds for the two ways
the hashing runs (CULS_DEDUP_MODE: fixed-point rounds or the level
dataflow)."""
import pytest

import culs_b200 as C
from oracle.oracle import Oracle
from util import same_graph, to_oracle

pytestmark = pytest.mark.gpu


def graphs():
    gs = [C.gen_multiplier(16), C.gen_multiplier(48), C.gen_layered(7, 64, 32, 30000, 60, 4, 0.0, True)]
    gs += C.gen_batch(5, 0, 48, 1000, 20000, 16, 128, threads=8)
    return gs


def run(ctx, gs, gpu_dedup, twice):
    d = ctx.upload_batch(gs)
    ctx.rw(d, gpu_dedup=gpu_dedup)
    if twice:
        ctx.rw(d, gpu_dedup=gpu_dedup)
    ctx.st(d)
    out = d.download_all()
    d.free()
    return out


def oracle(g, gpu_dedup, twice):
    o = Oracle()
    o.set_graph(to_oracle(g))
    for _ in range(2 if twice else 1):
        o.rw(dedup=2 if gpu_dedup else 1)
    o.st()
    return o.graph()


@pytest.mark.parametrize("gpu_dedup,twice", [(True, False), (False, False), (False, True)])
def test_level_paths_agree(gpu_dedup, twice, monkeypatch):
    gs = graphs()
    ctx = C.Context()
    try:
        a = run(ctx, gs, gpu_dedup, twice)
        monkeypatch.setenv("CULS_DEDUP_WORKLIST", "1")
        b = run(ctx, gs, gpu_dedup, twice)
    finally:
        ctx.close()
    for i, g in enumerate(gs):
        assert same_graph(a[i], b[i]), i
        assert same_graph(a[i], oracle(g, gpu_dedup, twice)), i


@pytest.mark.parametrize("gpu_dedup", [True, False])
def test_hashing_rounds_equal_level_dataflow(gpu_dedup, monkeypatch):
    """The hashing's fixed-point rounds (the default on batches whose table
    fits in L2) and its level-by-level dataflow (the default on larger ones)
    give the same graphs, equal to the oracle, on both the rewrite's
    deduplication and `st`; a chain of `rw; rw; st` makes the second rewrite
    start from a graph with merges left to cascade."""
    gs = graphs()
    ctx = C.Context()
    try:
        got, rounds = {}, {}
        for mode in ["rounds", "levels"]:
            monkeypatch.setenv("CULS_DEDUP_MODE", mode)
            d = ctx.upload_batch(gs)
            rounds[mode] = []
            for _ in range(2):
                ctx.rw(d, gpu_dedup=gpu_dedup)
                rounds[mode].append(ctx.rw_stats()["hash_rounds"])
            ctx.st(d)
            got[mode] = d.download_all()
            d.free()
    finally:
        ctx.close()
    # the rounds settled by themselves (the level dataflow did not step in)
    assert all(1 <= r <= 8 for r in rounds["rounds"]), rounds
    assert rounds["levels"] == [0, 0], rounds
    for i, g in enumerate(gs):
        assert same_graph(got["rounds"][i], got["levels"][i]), i
        assert same_graph(got["rounds"][i], oracle(g, gpu_dedup, True)), i
