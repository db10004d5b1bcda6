"""Bit-parallel simulation of AIGs (AIGMan layout, literal 0 = TRUE) used to
check that rewriting preserves every PO function."""
import numpy as np

ALL = np.uint64(0xFFFFFFFFFFFFFFFF)


def simulate(nPIs, f0, f1, outs, pi_words):
    """pi_words: array (nPIs, W) of uint64 patterns; returns (nPOs, W)."""
    n = len(f0)
    W = pi_words.shape[1]
    val = np.zeros((n, W), dtype=np.uint64)
    val[0] = ALL  # constant TRUE
    val[1:nPIs + 1] = pi_words
    for v in range(nPIs + 1, n):
        a, b = int(f0[v]), int(f1[v])
        x = val[a >> 1] ^ (ALL if a & 1 else np.uint64(0))
        y = val[b >> 1] ^ (ALL if b & 1 else np.uint64(0))
        val[v] = x & y
    res = np.zeros((len(outs), W), dtype=np.uint64)
    for k, o in enumerate(outs):
        o = int(o)
        res[k] = val[o >> 1] ^ (ALL if o & 1 else np.uint64(0))
    return res


def patterns(nPIs, words=16, seed=1):
    """Exhaustive patterns for up to 12 PIs, otherwise seeded random words."""
    if nPIs <= 12:
        m = 1 << nPIs
        W = max(1, (m + 63) // 64)
        ks = np.arange(W * 64, dtype=np.uint64) % np.uint64(m)
        sh = np.arange(64, dtype=np.uint64)
        out = np.zeros((nPIs, W), dtype=np.uint64)
        for i in range(nPIs):
            b = ((ks >> np.uint64(i)) & np.uint64(1)).reshape(W, 64)
            out[i] = (b << sh).sum(axis=1, dtype=np.uint64)
        return out
    rng = np.random.default_rng(seed)
    return rng.integers(0, np.iinfo(np.uint64).max, size=(nPIs, words), dtype=np.uint64, endpoint=True)


def equivalent(a, b, words=16, seed=1):
    """True if AIGs a and b (same PI/PO counts) agree on the patterns."""
    if a.nPIs != b.nPIs or len(a.outs) != len(b.outs):
        return False
    p = patterns(a.nPIs, words, seed)
    return np.array_equal(simulate(a.nPIs, a.fanin0, a.fanin1, a.outs, p),
                          simulate(b.nPIs, b.fanin0, b.fanin1, b.outs, p))
