"""Proves `rw; st` and `b` equivalence-preserving on the single-graph
configurations with the z3 SAT-sweeping CEC (oracle/cec.py, the substitute
for ABC `cec`, which cannot be built here), and records the outcome in
tests/golden/cec.json.  Runs on the CPU, one process per check (about an
hour, set by the 64x64 multiplier):

    python tests/golden/run_cec.py

The graphs checked are the oracle's results, which the GPU tests show equal
to the CUDA path's node for node (tests/test_gpu_parity.py,
tests/test_balance.py), so the proof covers both.
"""
import json
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))
import culs_b200 as C  # noqa: E402  (generators only)
from oracle.cec import cec  # noqa: E402
from oracle.oracle import Oracle  # noqa: E402
from util import to_oracle  # noqa: E402

CASES = {
    "c1_layered5k": lambda: C.gen_layered(1, 64, 32, 5000, 40, 4, 0.0, True),
    "c2_mult64x64": lambda: C.gen_multiplier(64),
}


def run(g, ops):
    o = Oracle()
    o.set_graph(to_oracle(g))
    for op in ops:
        op(o)
    return o.graph()


FLOWS = {"rw;st": [lambda o: o.rw(), lambda o: o.st()], "b": [lambda o: o.b()]}


def check(job):
    name, flow = job
    g = CASES[name]()
    r = run(g, FLOWS[flow])
    res = cec(to_oracle(g), r, words=32)
    res.update({"and_in": g.nAnds, "and_out": r.nAnds, "level_out": r.nLevels})
    print(name, flow, res, flush=True)
    return f"{name} {flow}", res


def main():
    import multiprocessing as mp
    jobs = [(name, flow) for name in CASES for flow in FLOWS]
    # one z3 process per check (the multiplier's take the better part of an hour)
    with mp.get_context("spawn").Pool(len(jobs)) as pool:
        out = dict(pool.map(check, jobs))
    out = {f"{n} {f}": out[f"{n} {f}"] for n, f in jobs}
    (Path(__file__).resolve().parent / "cec.json").write_text(json.dumps(out, indent=1) + "\n")


if __name__ == "__main__":
    main()
