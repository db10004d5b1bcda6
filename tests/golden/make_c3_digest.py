"""Records the oracle's `rw; st` result on the 10M-AND single-graph workload
(seeded layered AIG: 4,096 PIs and POs, 2,000 layers, fanins 80% from the
previous 3 layers and 20% from all earlier nodes, complemented with p=0.5,
seed 3) as SHA-256 digests, so that a GPU test can check the CUDA path on the
full-size graph without running the oracle there (about a minute of CPU work
per pass on one core).  Runs on the CPU:

    python tests/golden/make_c3_digest.py [--out tests/golden/c3_layered10M.json]

The oracle is pinned to the reference's own outputs by the other fixtures in
this folder; this file extends that check to the full-size graph.
"""
import argparse
import hashlib
import json
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))
import culs_b200 as C  # noqa: E402  (generator only)
from util import oracle_rw_st  # noqa: E402

# (seed, PIs, POs, ANDs, layers, window, far fraction, window includes PIs)
C3 = (3, 4096, 4096, 10_000_000, 2000, 3, 0.2, False)


def digest(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(np.asarray(a, np.int32)).tobytes())
    return h.hexdigest()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=str(Path(__file__).resolve().parent / "c3_layered10M.json"))
    a = ap.parse_args()
    t0 = time.time()
    g = C.gen_layered(*C3)
    t1 = time.time()
    o = oracle_rw_st(g)
    r = o.graph()
    t2 = time.time()
    rec = {"generator": "gen_layered", "args": list(C3),
           "input": {"nPIs": g.nPIs, "nAnds": g.nAnds, "nPOs": g.nPOs,
                     "sha256": digest(g.fanin0, g.fanin1, g.outs)},
           "rw_st": {"nAnds": r.nAnds, "nLevels": r.nLevels, "nPOs": r.nPOs,
                     "sha256": digest(r.fanin0, r.fanin1, r.outs)},
           "rw_stats": {k: int(v) for k, v in o.dump_stats().items()},
           "oracle_seconds": round(t2 - t1, 1), "generate_seconds": round(t1 - t0, 1)}
    Path(a.out).write_text(json.dumps(rec, indent=1) + "\n")
    print(json.dumps(rec))


if __name__ == "__main__":
    main()
