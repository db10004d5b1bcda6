"""Properties of the oracle's `rw; st` that hold whatever the graph: on
seeded random layered AIGs and multipliers, with and without -z and with
GPU- and CPU-style deduplication, the result computes the same functions as
the input, is strashed (no duplicate fanin pair, no trivial AND), has no
dangling AND, and a second `st` leaves it unchanged.  Graphs with at most 14
inputs are compared on every input pattern (exact); larger ones on 4,096
random patterns, which on deep random AND graphs misses part of the
single-literal errors (many nodes there are almost always 0).  These check
the CPU restatement itself, beside its golden fixtures from the reference."""
import numpy as np
import pytest

import culs_b200 as C
from oracle import oracle as O
from oracle.oracle import Oracle
from util import to_oracle


def cases():
    out = []
    for seed in range(8):  # exhaustively simulated
        rng = np.random.default_rng(50 + seed)
        nPIs, nAnds = int(rng.integers(8, 15)), int(rng.integers(100, 1200))
        nLayers = max(4, nAnds // (4 * nPIs))  # layers no wider than 4 nodes per PI
        out.append((f"small{seed}", C.gen_layered(200 + seed, nPIs, int(rng.integers(2, 12)), nAnds, nLayers,
                                                  int(rng.integers(2, 6)), float(rng.choice([0.0, 0.3])),
                                                  bool(seed % 2))))
    for seed in range(6):
        rng = np.random.default_rng(seed)
        n = int(rng.integers(300, 4000))
        out.append((f"layered{seed}", C.gen_layered(100 + seed, int(rng.integers(8, 64)), int(rng.integers(4, 32)), n,
                                                    int(rng.integers(5, 40)), int(rng.integers(2, 6)),
                                                    float(rng.choice([0.0, 0.2])), bool(seed % 2))))
    out += [("mult6", C.gen_multiplier(6)), ("mult10", C.gen_multiplier(10))]
    return out


def outputs(g):
    """PO truth tables over every input pattern (nPIs <= 14), 64 patterns a
    word; literal 0 is constant TRUE (the AIGMan convention)."""
    f0, f1 = np.asarray(g.fanin0), np.asarray(g.fanin1)
    k = g.nPIs
    W = max(1, (1 << k) // 64)
    pat = np.arange(W * 64, dtype=np.uint64).reshape(W, 64)
    sh = np.arange(64, dtype=np.uint64)
    val = np.zeros((len(f0), W), np.uint64)
    val[0] = ~np.uint64(0)
    for i in range(k):
        val[1 + i] = np.bitwise_or.reduce(((pat >> np.uint64(i)) & np.uint64(1)) << sh, axis=1)

    def lit(l):
        v = val[l >> 1]
        return ~v if l & 1 else v

    for i in range(1 + k, len(f0)):
        val[i] = lit(f0[i]) & lit(f1[i])
    return np.array([lit(o) for o in np.asarray(g.outs)])


def equivalent(a, b):
    if a.nPIs <= 14:
        return a.nPIs == b.nPIs and np.array_equal(outputs(a), outputs(b))
    return O.equivalent_sim(a, b, words=64, seed=7)


def run(g, zeros, dedup):
    o = Oracle()
    o.set_graph(to_oracle(g))
    o.rw(zeros=zeros, dedup=dedup)
    o.st()
    return o.graph()


def strashed(g):
    f0, f1 = np.asarray(g.fanin0), np.asarray(g.fanin1)
    ands = np.arange(1 + g.nPIs, len(f0))
    a, b = f0[ands], f1[ands]
    lo, hi = np.minimum(a, b), np.maximum(a, b)
    pairs = set(zip(lo.tolist(), hi.tolist()))
    trivial = (lo >> 1 == hi >> 1) | (lo >> 1 == 0)  # x&x, x&!x, or a constant fanin
    return len(pairs) == len(ands) and not trivial.any()


def no_dangling(g):
    f0, f1 = np.asarray(g.fanin0), np.asarray(g.fanin1)
    used = np.zeros(len(f0), bool)
    used[np.asarray(g.outs) >> 1] = True
    for i in range(len(f0) - 1, g.nPIs, -1):
        if used[i]:
            used[f0[i] >> 1] = used[f1[i] >> 1] = True
    return bool(used[1 + g.nPIs:].all())


@pytest.mark.parametrize("zeros,dedup", [(False, 2), (True, 2), (False, 1)])
def test_oracle_rw_st_properties(zeros, dedup):
    for name, g in cases():
        r = run(g, zeros, dedup)
        assert equivalent(to_oracle(g), r), name
        assert strashed(r), name
        assert no_dangling(r), name
        o = Oracle()
        o.set_graph(r)
        o.st()
        again = o.graph()
        assert np.array_equal(np.asarray(again.fanin0), np.asarray(r.fanin0)), name
        assert np.array_equal(np.asarray(again.fanin1), np.asarray(r.fanin1)), name
        assert np.array_equal(np.asarray(again.outs), np.asarray(r.outs)), name
