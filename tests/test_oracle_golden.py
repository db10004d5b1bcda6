"""Pins the CPU oracle to the reference: every fixture in tests/golden was
produced by the reference CULS code (oracle/_ref/rw_harness built from the
reference sources, run on a B200 by tests/golden/make_golden.py).

Exact (bit-for-bit) comparisons: the reordered fanins, all 8 cut slots per
node, the selected cut and root per node, the choice-loop counters.  Up to
renumbering (the reference numbers new nodes by atomicAdd and picks strash
winners by thread timing): replace[] targets and the final AIG, plus exact
AND count and level."""
import hashlib
import json
from pathlib import Path

import numpy as np
import pytest

import aigcanon
from oracle.oracle import Graph, Oracle

GOLDEN = Path(__file__).resolve().parent / "golden"
CASES = sorted(p.stem for p in GOLDEN.glob("*.npz") if p.stem not in ("chains", "balance"))


def load(name):
    return dict(np.load(GOLDEN / f"{name}.npz", allow_pickle=False))


def oracle_for(f):
    o = Oracle()
    o.set_graph(Graph(int(f["nPIs"]), f["in_f0"], f["in_f1"], f["in_outs"]))
    return o


def test_fixtures_present():
    assert {"c1_layered5k", "c2_mult64", "mult8"} <= set(CASES)


@pytest.mark.parametrize("name", CASES)
def test_oracle_per_node_results_match_reference(name):
    f = load(name)
    o = oracle_for(f)
    o.rw(zeros=False, dedup=2)
    n0, n1 = o.dump_sizes()
    assert n0 == int(f["n"])
    f0, f1, outs = o.dump_reorder(len(f["in_outs"]))
    nPIs = int(f["nPIs"])
    f0[:nPIs + 1] = 0
    f1[:nPIs + 1] = 0
    assert aigcanon.digest(f0) == str(f["ref_f0_sha"])
    assert aigcanon.digest(f1) == str(f["ref_f1_sha"])
    assert aigcanon.digest(outs) == str(f["ref_outs_sha"])
    cuts = o.dump_cuts().reshape(-1)
    sel = o.dump_selected().reshape(-1)
    if "cuts" in f:
        bad = np.nonzero((cuts.reshape(-1, 9) != f["cuts"].reshape(-1, 9)).any(1))[0]
        assert len(bad) == 0, f"cut slots differ at {bad[:5]}"
        np.testing.assert_array_equal(sel, f["selected"])
    assert aigcanon.digest(cuts) == str(f["cuts_sha"])
    assert aigcanon.digest(sel) == str(f["selected_sha"])
    rep, nf0, nf1 = o.dump_replace()
    ref_f0, ref_f1, _ = o.dump_reorder(len(f["in_outs"]))
    ref_f0[:nPIs + 1] = 0
    ref_f1[:nPIs + 1] = 0
    tgt = aigcanon.replace_targets(n0, rep, np.concatenate([ref_f0, nf0]), np.concatenate([ref_f1, nf1]), nPIs)
    want = [tuple(t) if t is not None else None for t in json.loads(str(f["replace_targets"]))]
    assert [tuple(t) if t is not None else None for t in tgt] == want


@pytest.mark.parametrize("zeros", [0, 1])
@pytest.mark.parametrize("name", CASES)
def test_oracle_rw_st_matches_reference(name, zeros):
    f = load(name)
    o = oracle_for(f)
    o.rw(zeros=bool(zeros), dedup=2)
    st = o.dump_stats()
    g_rw = o.graph()
    o.st()
    g = o.graph()
    ref_stats = [int(x) for x in f[f"z{zeros}_stats"]]
    mine = [st[k] for k in ["replaced", "replaced_pos", "replaced_zero", "reverted", "compromised", "pre_eval",
                            "small_cut", "new_idx"]]
    assert mine == ref_stats
    assert (g_rw.nAnds, g_rw.nLevels) == tuple(int(x) for x in f[f"z{zeros}_rw"])
    assert (g.nAnds, g.nLevels) == tuple(int(x) for x in f[f"z{zeros}_st"])
    ands, pos = aigcanon.signature(g.nPIs, g.fanin0, g.fanin1, g.outs)
    assert hashlib.sha256(json.dumps([ands, pos]).encode()).hexdigest() == str(f[f"z{zeros}_sig"])
