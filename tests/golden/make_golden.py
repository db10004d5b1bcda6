"""Generates the golden fixtures in tests/golden/ by running the reference
CULS code (oracle/_ref/rw_harness, built from the reference sources by
oracle/build_ref.sh) on seeded synthetic AIGs.  Needs a GPU (the reference's
rewrite runs on the device); run it once on a GPU box:

    python tests/golden/make_golden.py [--out tests/golden]

Each fixture <case>.npz holds the input AIG (AIGMan layout), the reference's
per-node results of rw (reordered fanins, all cut slots, selected cuts with
root index, replace[] after the rebuild with the rebuilt nodes' fanins) --
in full for small cases, as SHA-256 digests for large ones -- and the final
AIG after `rw; st` and `rw -z; st` (full arrays for small cases, a
renumbering-invariant signature for all) with the reference's printed
counters.
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
FULL_LIMIT = 6000  # objects: store full per-node arrays up to this size

CASES = {
    # the 5,000-AND layered graph: 64 PIs, 32 POs, 5,000 ANDs in 40 layers, window 4 + PIs
    "c1_layered5k": lambda: C.gen_layered(1, 64, 32, 5000, 40, 4, 0.0, True),
    # the 64x64 array multiplier
    "c2_mult64": lambda: C.gen_multiplier(64),
    "mult8": lambda: C.gen_multiplier(8),
    "mult16": lambda: C.gen_multiplier(16),
    "layered3k_w4": lambda: C.gen_layered(11, 16, 8, 3000, 50, 4, 0.0, True),
    "layered20k_far": lambda: C.gen_layered(7, 100, 50, 20000, 60, 3, 0.2, False),
}

STAT_RE = re.compile(r"successfully replaced (\d+) cones \(pos (\d+), zero (\d+)\), reverted (\d+) cones, "
                     r"compromised (\d+) cones, pre-eval rejected (\d+) cones, small cut reject (\d+) cones, "
                     r"new idx reject (\d+) cones")
AFTER_RE = re.compile(r"HARNESS after (rw|st): and = (\d+) level = (-?\d+)")


def read_dump(path):
    raw = np.fromfile(path, dtype=np.int32)
    out, k = [], 0
    while k < len(raw):
        n = int(raw[k])
        out.append(raw[k + 1:k + 1 + n].copy())
        k += 1 + n
    return out


def sig_digest(g):
    ands, pos = aigcanon.signature(g.nPIs, g.fanin0, g.fanin1, g.outs)
    return hashlib.sha256(json.dumps([ands, pos]).encode()).hexdigest()


def run_case(name, g, tmp: Path):
    inp = tmp / f"{name}.aig"
    C.write_aiger(inp, g)
    rec = {"nPIs": g.nPIs, "in_f0": g.fanin0, "in_f1": g.fanin1, "in_outs": g.outs}
    small = g.nObjs <= FULL_LIMIT
    subprocess.run([str(HARNESS), "dump", str(inp), str(tmp / name)], check=True, capture_output=True)
    hdr, f0, f1, outs, cuts, sel, rep, nf0, nf1 = read_dump(tmp / f"{name}.bin")
    n, n1 = int(hdr[0]), int(hdr[1])
    rec["n"], rec["n1"] = n, n1
    tgt = aigcanon.replace_targets(n, rep, np.concatenate([f0, nf0]), np.concatenate([f1, nf1]), g.nPIs)
    rec["replace_targets"] = json.dumps(tgt)
    if small:
        rec.update(ref_f0=f0, ref_f1=f1, ref_outs=outs, cuts=cuts, selected=sel)
    rec.update(ref_f0_sha=aigcanon.digest(f0), ref_f1_sha=aigcanon.digest(f1), ref_outs_sha=aigcanon.digest(outs),
               cuts_sha=aigcanon.digest(cuts), selected_sha=aigcanon.digest(sel))
    for zeros in (0, 1):
        out = tmp / f"{name}_z{zeros}.aig"
        r = subprocess.run([str(HARNESS), "full", str(inp), str(out), str(zeros)], check=True, capture_output=True,
                           text=True)
        m = STAT_RE.search(r.stdout)
        stats = [int(x) for x in m.groups()] if m else []
        after = {k: (int(a), int(lv)) for k, a, lv in AFTER_RE.findall(r.stdout)}
        res = C.read_aiger(out)
        rec[f"z{zeros}_stats"] = np.array(stats, dtype=np.int64)
        rec[f"z{zeros}_rw"] = np.array(after["rw"], dtype=np.int64)
        rec[f"z{zeros}_st"] = np.array(after["st"], dtype=np.int64)
        rec[f"z{zeros}_sig"] = sig_digest(res)
        if small:
            rec[f"z{zeros}_f0"], rec[f"z{zeros}_f1"], rec[f"z{zeros}_outs"] = res.fanin0, res.fanin1, res.outs
    return rec


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=str(Path(__file__).resolve().parent))
    ap.add_argument("--cases", nargs="*", default=list(CASES))
    a = ap.parse_args()
    if not HARNESS.exists():
        sys.exit(f"{HARNESS} missing: run oracle/build_ref.sh first")
    with tempfile.TemporaryDirectory() as td:
        for name in a.cases:
            rec = run_case(name, CASES[name](), Path(td))
            np.savez_compressed(Path(a.out) / f"{name}.npz", **rec)
            print(name, "ok", rec["n"], rec.get("z0_st"))


if __name__ == "__main__":
    main()
