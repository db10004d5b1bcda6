"""Generates tests/golden/balance.npz by running balance chains through the
reference CULS code (oracle/_ref/rw_harness chain, built from the reference
sources by oracle/build_ref.sh).  Needs a GPU; run it once on a GPU box:

    python tests/golden/make_balance.py [--out tests/golden]

Commands: b is the `b` command (AIGMan::balance with sortDecId 1, then a GPU
strash), bn the balance alone as resyn2 calls it (no strash), rw a rewrite
with GPU deduplication, st a strash.  Every chain runs RUNS times; per
(case, chain) the fixture holds, per run, the AND count and level printed
after each command and the renumbering-invariant signature of the final
AIG, whether all runs wrote the same file, and for small cases the final
arrays of the first run.
"""
import argparse
import hashlib
import json
import re
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))
import culs_b200 as C  # noqa: E402  (generators and AIGER I/O only)
import aigcanon  # noqa: E402

HARNESS = ROOT / "oracle" / "_ref" / "rw_harness"
FULL_LIMIT = 30000
RUNS = 3

CASES = {
    "mult8": lambda: C.gen_multiplier(8),
    "mult16": lambda: C.gen_multiplier(16),
    "layered3k_w4": lambda: C.gen_layered(11, 16, 8, 3000, 50, 4, 0.0, True),
    "c1_layered5k": lambda: C.gen_layered(1, 64, 32, 5000, 40, 4, 0.0, True),
    "layered20k_far": lambda: C.gen_layered(7, 100, 50, 20000, 60, 3, 0.2, False),
    "c2_mult64": lambda: C.gen_multiplier(64),
    "c4_graph200k": lambda: C.gen_batch(4, 9000, 1, 200000, 200000, 16, 512, threads=8)[0],
}
CHAINS = ["b", "bn,st", "bn,rw,st", "b,rw,st", "rw,st,b", "b,b"]

AFTER_RE = re.compile(r"HARNESS after (\w+): and = (\d+) level = (-?\d+)")


def sig_digest(g):
    ands, pos = aigcanon.signature(g.nPIs, g.fanin0, g.fanin1, g.outs)
    return hashlib.sha256(json.dumps([ands, pos]).encode()).hexdigest()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=str(Path(__file__).resolve().parent))
    a = ap.parse_args()
    if not HARNESS.exists():
        sys.exit(f"{HARNESS} missing: run oracle/build_ref.sh first")
    rec = {}
    with tempfile.TemporaryDirectory() as td:
        tmp = Path(td)
        for name, make in CASES.items():
            g = make()
            inp = tmp / f"{name}.aig"
            C.write_aiger(inp, g)
            for ci, chain in enumerate(CHAINS):
                afters, sigs, blobs = [], [], set()
                first = None
                for run in range(RUNS):
                    out = tmp / f"{name}_{ci}_{run}.aig"
                    r = subprocess.run([str(HARNESS), "chain", str(inp), str(out), chain], check=True,
                                       capture_output=True, text=True)
                    afters.append([(int(n), int(lv)) for _, n, lv in AFTER_RE.findall(r.stdout)])
                    res = C.read_aiger(out)
                    sigs.append(sig_digest(res))
                    blobs.add(out.read_bytes())
                    if first is None:
                        first = res
                key = f"{name}/{chain}"
                rec[key + "/afters"] = np.array(afters, np.int64)
                rec[key + "/sig"] = np.array(sigs)
                rec[key + "/same_file"] = np.array([len(blobs) == 1])
                if first.nObjs <= FULL_LIMIT:
                    rec[key + "/f0"], rec[key + "/f1"], rec[key + "/outs"] = first.fanin0, first.fanin1, first.outs
                print(name, chain, afters[0], "runs identical" if len(blobs) == 1 else "runs differ", flush=True)
    np.savez_compressed(Path(a.out) / "balance.npz", **rec)


if __name__ == "__main__":
    main()
