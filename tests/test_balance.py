"""Balance `b` (tests/golden/balance.npz, from the reference CULS code:
tests/golden/make_balance.py).

The reference balance with sortDecId 1 (the `b` default) is deterministic:
every chain gave the same file on every run.  The oracle must equal it
exactly -- AND count and level after every command, the
renumbering-invariant signature of the final AIG and, for the small cases,
the final arrays -- and stay equivalent to the input by simulation.  The GPU
path (culs_b, `-m gpu`) must equal the oracle exactly.
"""
import hashlib
import importlib.util
import json
from pathlib import Path

import numpy as np
import pytest

import aigcanon
import culs_b200 as C
from oracle import oracle as O
from oracle.oracle import Oracle
from util import same_graph, to_oracle

GOLDEN = Path(__file__).resolve().parent / "golden"
_spec = importlib.util.spec_from_file_location("make_balance", GOLDEN / "make_balance.py")
MB = importlib.util.module_from_spec(_spec)
_spec.loader.exec_module(MB)
FIX = np.load(GOLDEN / "balance.npz")
SMALL = ["mult8", "mult16", "layered3k_w4", "c1_layered5k", "layered20k_far"]


def oracle_chain(g, chain):
    o = Oracle()
    o.set_graph(to_oracle(g))
    after = []
    for tok in chain.split(","):
        if tok == "st":
            o.st()
        elif tok == "b":
            o.b(update_level=True)
        elif tok == "bn":
            o.b(update_level=False)
        else:
            o.rw()
        r = o.graph()
        after.append((r.nAnds, r.nLevels))
    return o.graph(), after


def sig_digest(g):
    ands, pos = aigcanon.signature(g.nPIs, g.fanin0, g.fanin1, g.outs)
    return hashlib.sha256(json.dumps([ands, pos]).encode()).hexdigest()


def test_reference_balance_is_deterministic():
    for case in MB.CASES:
        for chain in MB.CHAINS:
            assert bool(FIX[f"{case}/{chain}/same_file"][0]), (case, chain)


@pytest.mark.parametrize("case", SMALL)
def test_oracle_balance_matches_reference(case):
    g = MB.CASES[case]()
    for chain in MB.CHAINS:
        key = f"{case}/{chain}"
        out, after = oracle_chain(g, chain)
        assert after == [tuple(int(v) for v in x) for x in FIX[key + "/afters"][0]], key
        assert sig_digest(out) == str(FIX[key + "/sig"][0]), key
        if key + "/f0" in FIX:
            assert np.array_equal(out.fanin0, FIX[key + "/f0"]), key
            assert np.array_equal(out.fanin1, FIX[key + "/f1"]), key
            assert np.array_equal(out.outs, FIX[key + "/outs"]), key
        assert O.equivalent_sim(out, to_oracle(g)), key


@pytest.mark.parametrize("case", ["c2_mult64", "c4_graph200k"])
def test_oracle_balance_matches_reference_large(case):
    """The 64x64 multiplier and a 200k-AND member of the batched family, on
    the `b` command alone and `b; rw; st`."""
    g = MB.CASES[case]()
    for chain in ["b", "b,rw,st"]:
        key = f"{case}/{chain}"
        out, after = oracle_chain(g, chain)
        assert after == [tuple(int(v) for v in x) for x in FIX[key + "/afters"][0]], key
        assert sig_digest(out) == str(FIX[key + "/sig"][0]), key


def test_balance_without_and_driven_outputs():
    """No PO on an AND node: the balance keeps no AND node."""
    g = C.Aig(2, np.array([-1, -1, -1, 2], np.int32), np.array([-1, -1, -1, 5], np.int32),
              np.array([2, 5, 0], np.int32))
    o = Oracle()
    o.set_graph(to_oracle(g))
    o.b()
    r = o.graph()
    assert r.nAnds == 0 and list(r.outs) == [2, 5, 0]
