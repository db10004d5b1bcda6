"""Renumbering-invariant views of AIGs, for comparing results whose node
order the reference leaves to thread timing (GPU strash winners, atomicAdd
ids of new nodes)."""
import hashlib

import numpy as np

_M = (1 << 64) - 1


def _mix(x):
    x = (x + 0x9E3779B97F4A7C15) & _M
    x = ((x ^ (x >> 30)) * 0xBF58476D1CE4E5B9) & _M
    x = ((x ^ (x >> 27)) * 0x94D049BB133111EB) & _M
    return x ^ (x >> 31)


def node_hashes(nPIs, f0, f1, const_true_lit=0):
    """Structural hash of every object: PIs hash their index, the constant a
    fixed value, AND nodes the unordered pair of their fanins' hashes (a
    complemented edge flips the hash).  f0/f1 are literal arrays over ids in
    topological order (entries of the constant and PIs ignored)."""
    n = len(f0)
    h = [0] * n
    h[0] = _mix(0xC0517)
    for i in range(1, nPIs + 1):
        h[i] = _mix(i)
    for v in range(nPIs + 1, n):
        a, b = int(f0[v]), int(f1[v])
        ha = h[a >> 1] ^ (0x5A5A5A5A5A5A5A5A if a & 1 else 0)
        hb = h[b >> 1] ^ (0x5A5A5A5A5A5A5A5A if b & 1 else 0)
        lo, hi = (ha, hb) if ha <= hb else (hb, ha)
        h[v] = _mix(lo * 1000003 ^ _mix(hi))
    return h


def lit_hash(h, lit):
    return h[lit >> 1] ^ (0x5A5A5A5A5A5A5A5A if lit & 1 else 0)


def signature(nPIs, f0, f1, outs):
    """(sorted AND-node hashes, PO hashes in order) -- equal for two AIGs
    that differ only in the numbering of their AND nodes."""
    h = node_hashes(nPIs, f0, f1)
    ands = sorted(h[nPIs + 1:])
    pos = [lit_hash(h, int(o)) for o in outs]
    return ands, pos


def digest(arr):
    return hashlib.sha256(np.ascontiguousarray(arr, dtype=np.int32).tobytes()).hexdigest()


def replace_targets(nn, replace, fanin0_all, fanin1_all, nPIs):
    """Per node id 0..nn: None, ('id', target, compl) for an existing node, or
    ('new', hash, compl) for a node created by the rewrite (ids > nn).
    fanin arrays cover ids 0..n1 in AIGER constant convention."""
    h = node_hashes(nPIs, fanin0_all, fanin1_all)
    out = []
    for i in range(nn + 1):
        r = int(replace[i])
        if r < 0:
            out.append(None)
        elif (r >> 1) <= nn:
            out.append(("id", r >> 1, r & 1))
        else:
            out.append(("new", h[r >> 1], r & 1))
    return out
