"""Combinational equivalence check of two AIGs by SAT sweeping with z3.

TEST INFRASTRUCTURE.  ABC's `cec`, the check the reference's users run,
cannot be built here: the reference's ABC submodule is empty.  This is a
substitute, reported under its own name ("z3 SAT-sweeping CEC"), not as
ABC:

1. both AIGs (AIGMan convention: literal 0 = TRUE) share their PIs and are
   simulated on random 64-bit patterns, every node of both;
2. every node of the second AIG whose simulation signature equals that of a
   node of the first (or its complement) is a candidate pair;
3. one incremental z3 solver holds the Tseitin encoding of both AIGs; the
   candidate pairs are proved in topological order of the second AIG, each
   proved pair added as an equality (so later proofs see both cones merged,
   which keeps each query local), a refuted pair left out and its
   counterexample kept: every 64 counterexamples become one more simulation
   word, which splits the candidate classes they refute;
4. the outputs are equivalent when, for every PO pair, z3 finds no input
   assignment that tells them apart (UNSAT).

Returns a dict: equivalent (True only when every PO pair is proved), the
counts of candidate pairs proved and refuted, the PO pairs proved, and the
time taken.
"""
import time

import numpy as np


def _simulate_all(g, words, seed):
    """Values of every object of g (AIGMan literals) under `words` x 64
    random patterns: uint64 array [nObjs, words] (object 0 = TRUE)."""
    n = len(g.fanin0)
    rng = np.random.default_rng(seed)
    val = np.zeros((n, words), np.uint64)
    val[0] = np.uint64(0xFFFFFFFFFFFFFFFF)
    val[1:g.nPIs + 1] = rng.integers(0, 2 ** 64, (g.nPIs, words), dtype=np.uint64)
    f0 = np.asarray(g.fanin0)
    f1 = np.asarray(g.fanin1)
    full = np.uint64(0xFFFFFFFFFFFFFFFF)
    for v in range(g.nPIs + 1, n):
        a, b = int(f0[v]), int(f1[v])
        x = val[a >> 1] ^ (full if a & 1 else np.uint64(0))
        y = val[b >> 1] ^ (full if b & 1 else np.uint64(0))
        val[v] = x & y
    return val


def _simulate_word(g, pi_word):
    """One 64-bit word per object of g for the given PI word array."""
    n = len(g.fanin0)
    val = np.zeros(n, np.uint64)
    val[0] = np.uint64(0xFFFFFFFFFFFFFFFF)
    val[1:g.nPIs + 1] = pi_word
    f0 = np.asarray(g.fanin0)
    f1 = np.asarray(g.fanin1)
    full = np.uint64(0xFFFFFFFFFFFFFFFF)
    for v in range(g.nPIs + 1, n):
        a, b = int(f0[v]), int(f1[v])
        x = val[a >> 1] ^ (full if a & 1 else np.uint64(0))
        y = val[b >> 1] ^ (full if b & 1 else np.uint64(0))
        val[v] = x & y
    return val


def cec(a, b, words=8, seed=1, max_pairs=None, query_ms=20000, verbose=False):
    """query_ms bounds each z3 query; a candidate whose query runs out is
    left unmerged, a PO pair whose query runs out is left unproved.  Every
    refuted candidate's counterexample is kept; each 64 of them become one
    more simulation word, which splits the candidate classes they refute."""
    import z3
    t0 = time.time()
    if a.nPIs != b.nPIs or len(a.outs) != len(b.outs):
        return {"equivalent": False, "reason": "interfaces differ", "seconds": time.time() - t0}
    va = _simulate_all(a, words, seed)
    vb = _simulate_all(b, words, seed)
    full = np.uint64(0xFFFFFFFFFFFFFFFF)
    s = z3.Solver()
    s.set("timeout", query_ms)
    pis = [z3.BoolVal(True)] + [z3.Bool(f"i{k}") for k in range(1, a.nPIs + 1)]

    def encode(g, tag):
        xs = list(pis) + [None] * (len(g.fanin0) - g.nPIs - 1)
        for v in range(g.nPIs + 1, len(g.fanin0)):
            x = z3.Bool(f"{tag}{v}")
            l0, l1 = int(g.fanin0[v]), int(g.fanin1[v])
            p = xs[l0 >> 1] if not l0 & 1 else z3.Not(xs[l0 >> 1])
            q = xs[l1 >> 1] if not l1 & 1 else z3.Not(xs[l1 >> 1])
            s.add(x == z3.And(p, q))
            xs[v] = x
        return xs

    xa = encode(a, "a")
    xb = encode(b, "b")

    def lit(xs, l):
        return xs[l >> 1] if not l & 1 else z3.Not(xs[l >> 1])

    # candidate pairs: signature of a node of b equal to a node of a (or its complement)
    def build_sig():
        sig = {}
        for v in range(len(a.fanin0)):
            sig.setdefault(va[v].tobytes(), (v, 0))
        for v in range(len(a.fanin0)):
            sig.setdefault((va[v] ^ full).tobytes(), (v, 1))
        return sig

    sig = build_sig()
    cex = []  # counterexample input vectors, bit k of PI k
    proved = refuted = unknown = 0
    for v in range(b.nPIs + 1, len(b.fanin0)):
        c = sig.get(vb[v].tobytes())
        if c is None:
            continue
        if max_pairs is not None and proved + refuted >= max_pairs:
            break
        u, comp = c
        ea = xa[u] if not comp else z3.Not(xa[u])
        s.push()
        s.add(ea != xb[v])
        r = s.check()
        if r == z3.sat:
            m = s.model()
            cex.append([z3.is_true(m.eval(pis[k], model_completion=True)) for k in range(1, a.nPIs + 1)])
        s.pop()
        if r == z3.unsat:
            s.add(ea == xb[v])
            proved += 1
        elif r == z3.sat:
            refuted += 1
            if len(cex) == 64:  # one more simulation word from the counterexamples
                bits = np.array(cex, bool)  # [64, nPIs]
                w = np.zeros(a.nPIs, np.uint64)
                for k in range(64):
                    w |= bits[k].astype(np.uint64) << np.uint64(k)
                va = np.concatenate([va, _simulate_word(a, w)[:, None]], axis=1)
                vb = np.concatenate([vb, _simulate_word(b, w)[:, None]], axis=1)
                sig = build_sig()
                cex = []
        else:
            unknown += 1
        if verbose and (proved + refuted + unknown) % 2000 == 0:
            print(f"  cec {v}/{len(b.fanin0)}: proved {proved} refuted {refuted} unknown {unknown} "
                  f"{time.time() - t0:.0f} s", flush=True)
    po_proved = 0
    for oa, ob in zip(a.outs, b.outs):
        s.push()
        s.add(lit(xa, int(oa)) != lit(xb, int(ob)))
        r = s.check()
        s.pop()
        if r == z3.unsat:
            po_proved += 1
    return {"equivalent": po_proved == len(a.outs), "pos": len(a.outs), "pos_proved": po_proved,
            "pairs_proved": proved, "pairs_refuted": refuted, "pairs_unknown": unknown,
            "seconds": round(time.time() - t0, 2),
            "method": "z3 SAT-sweeping CEC (simulation candidates, incremental proofs)"}
