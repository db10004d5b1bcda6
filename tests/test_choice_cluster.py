"""The choice loop of a single graph (CULS src/algorithms/rewrite.cu:830-921)
runs on a thread-block cluster with the graph's fanins, deletion flags and
reference counts in distributed shared memory when the graph has at most
65,536 objects (rewritten nodes included), and one thread per graph over
HBM otherwise (CULS_CHOICE_GLOBAL forces the latter).  Both must give the
oracle's graph, with the same choice statistics."""
import pytest

import culs_b200 as C
from oracle.oracle import Oracle
from util import same_graph, to_oracle

pytestmark = pytest.mark.gpu


def graphs():
    return [
        C.gen_multiplier(4),                                  # one block of 256 objects
        C.gen_multiplier(16),
        C.gen_multiplier(64),                                 # config 2: six blocks
        C.gen_layered(11, 64, 32, 60000, 120, 4, 0.0, True),  # near the bound
        C.gen_layered(13, 128, 64, 130000, 160, 4, 0.0, True),  # above it: one thread over HBM
    ]


def oracle(g, zeros):
    o = Oracle()
    o.set_graph(to_oracle(g))
    o.rw(zeros=zeros)
    o.st()
    return o.graph(), o.dump_stats()


@pytest.mark.parametrize("zeros", [False, True])
def test_cluster_choice_matches_oracle_and_global_walk(zeros, monkeypatch):
    ctx = C.Context()
    try:
        for i, g in enumerate(graphs()):
            got = {}
            for mode in ["cluster", "global"]:
                if mode == "global":
                    monkeypatch.setenv("CULS_CHOICE_GLOBAL", "1")
                else:
                    monkeypatch.delenv("CULS_CHOICE_GLOBAL", raising=False)
                d = ctx.upload(g)
                ctx.rw(d, zeros=zeros)
                st = ctx.rw_stats()
                ctx.st(d)
                got[mode] = (d.download(), st)
                d.free()
            ref, rs = oracle(g, zeros)
            assert same_graph(got["cluster"][0], ref), i
            assert same_graph(got["global"][0], ref), i
            for k in ["replaced", "replaced_pos", "replaced_zero", "reverted", "compromised"]:
                assert got["cluster"][1][k] == got["global"][1][k] == rs[k], (i, k)
    finally:
        ctx.close()
