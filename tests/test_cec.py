"""The z3 SAT-sweeping CEC (oracle/cec.py), the substitute for ABC `cec`:
it proves `rw; st` and `b` results equivalent to their inputs, finds a
planted difference, and the recorded proofs of the single-graph
configurations (tests/golden/cec.json, tests/golden/run_cec.py) all hold."""
import json
from pathlib import Path

import numpy as np
import pytest

import culs_b200 as C
from oracle.cec import cec
from oracle.oracle import Oracle
from util import oracle_rw_st, to_oracle

GOLDEN = Path(__file__).resolve().parent / "golden"
pytest.importorskip("z3")


def test_rw_st_and_balance_are_proved_equivalent():
    for g in [C.gen_multiplier(8), C.gen_layered(11, 16, 8, 600, 20, 4, 0.0, True)]:
        r = oracle_rw_st(g).graph()
        assert cec(to_oracle(g), r)["equivalent"]
        o = Oracle()
        o.set_graph(to_oracle(g))
        o.b()
        assert cec(to_oracle(g), o.graph())["equivalent"]


def test_planted_difference_is_found():
    g = C.gen_multiplier(8)
    r = oracle_rw_st(g).graph()
    f0 = np.array(r.fanin0)
    f0[len(f0) - 7] ^= 1  # complement one fanin edge of the rewritten graph
    r.fanin0 = f0
    res = cec(to_oracle(g), r)
    assert not res["equivalent"] and res["pos_proved"] < res["pos"]


def test_recorded_proofs_of_the_single_graph_configurations():
    rec = json.loads((GOLDEN / "cec.json").read_text())
    assert {"c1_layered5k rw;st", "c2_mult64x64 rw;st"} <= set(rec)
    for name, r in rec.items():
        assert r["equivalent"] and r["pos_proved"] == r["pos"], name
