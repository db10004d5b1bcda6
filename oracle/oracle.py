"""ctypes wrapper of the CPU oracle (oracle/culs_oracle.cpp).

ORACLE -- test infrastructure only.  Only tests/, __graft_entry__.smoke()
and bench.py's CPU-baseline leg import this module, as the checker or as the
timed CPU baseline; the product (culs_b200) never does.
"""
import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liboracle.so"
RWLIB = HERE.parent / "culs_b200" / "data" / "rwlib.bin"

CUT_INTS = 9  # used, nLeaves, leaves[4], tt, sign, value
SEL_INTS = 10  # cut record + chosen root index

CHOICE_NAMES = ["not_visited", "no_cut", "small_cut", "no_replace", "self_ref", "compromised", "committed",
                "reverted"]
STAT_NAMES = ["replaced", "replaced_pos", "replaced_zero", "reverted", "compromised", "pre_eval", "small_cut",
              "new_idx", "expected", "new_nodes"]


def build(force=False):
    """Compile liboracle.so with g++ (used by __graft_entry__.build)."""
    src = HERE / "culs_oracle.cpp"
    if force or not LIB_PATH.exists() or LIB_PATH.stat().st_mtime < src.stat().st_mtime:
        subprocess.check_call(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-o", str(LIB_PATH), str(src)])
    return LIB_PATH


_lib = None


def _load():
    global _lib
    if _lib is None:
        build()
        lib = ctypes.CDLL(str(LIB_PATH))
        vp, ip = ctypes.c_void_p, ctypes.POINTER(ctypes.c_int)
        lib.orc_create.restype = vp
        lib.orc_create.argtypes = [ctypes.c_char_p]
        lib.orc_destroy.argtypes = [vp]
        lib.orc_set_graph.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ip, ip, ip]
        lib.orc_rw.argtypes = [vp, ctypes.c_int, ctypes.c_int]
        lib.orc_st.argtypes = [vp, ctypes.c_int]
        lib.orc_b.argtypes = [vp, ctypes.c_int]
        lib.orc_get_sizes.argtypes = [vp, ip, ip, ip, ip]
        lib.orc_get_graph.argtypes = [vp, ip, ip, ip]
        lib.orc_dump_sizes.argtypes = [vp, ip, ip]
        lib.orc_dump_reorder.argtypes = [vp, ip, ip, ip]
        lib.orc_dump_cuts.argtypes = [vp, ip]
        lib.orc_dump_selected.argtypes = [vp, ip]
        lib.orc_dump_replace.argtypes = [vp, ip, ip, ip]
        lib.orc_dump_choice.argtypes = [vp, ip]
        lib.orc_dump_stats.argtypes = [vp, ctypes.POINTER(ctypes.c_longlong)]
        lib.orc_prededup_sizes.argtypes = [vp, ip, ip]
        lib.orc_prededup_graph.argtypes = [vp, ip, ip, ip]
        lib.orc_simulate.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ip, ip, ip, ctypes.c_int,
                                     ctypes.c_ulonglong, ctypes.POINTER(ctypes.c_ulonglong)]
        _lib = lib
    return _lib


def _ip(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


class Graph:
    """AIG in the AIGMan layout (literal 0 = TRUE); arrays are int32 numpy."""

    def __init__(self, nPIs, fanin0, fanin1, outs, nLevels=None):
        self.nPIs = int(nPIs)
        self.fanin0 = np.ascontiguousarray(fanin0, dtype=np.int32)
        self.fanin1 = np.ascontiguousarray(fanin1, dtype=np.int32)
        self.outs = np.ascontiguousarray(outs, dtype=np.int32)
        self.nLevels = nLevels

    @property
    def nObjs(self):
        return len(self.fanin0)

    @property
    def nAnds(self):
        return self.nObjs - 1 - self.nPIs

    @property
    def nPOs(self):
        return len(self.outs)


class Oracle:
    def __init__(self):
        self.lib = _load()
        self.h = self.lib.orc_create(str(RWLIB).encode())
        if not self.h:
            raise RuntimeError(f"oracle: cannot load rewriting library {RWLIB}")

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.orc_destroy(self.h)
            self.h = None

    def set_graph(self, g: Graph):
        f0 = g.fanin0.copy()
        f1 = g.fanin1.copy()
        outs = g.outs.copy() if g.nPOs else np.zeros(1, np.int32)
        rc = self.lib.orc_set_graph(self.h, g.nPIs, g.nPOs, g.nAnds, _ip(f0), _ip(f1), _ip(outs))
        if rc != 0:
            raise ValueError("oracle: malformed AIG")

    def rw(self, zeros=False, dedup=2):
        self.lib.orc_rw(self.h, int(zeros), int(dedup))

    def st(self, cpu=False):
        self.lib.orc_st(self.h, int(cpu))

    def b(self, update_level=True):
        """`b` (balance, sortDecId 1), followed by a GPU-style strash when
        update_level (the command's behaviour)."""
        if self.lib.orc_b(self.h, int(update_level)) != 0:
            raise RuntimeError("oracle balance: inconsistent state")

    def graph(self) -> Graph:
        a = [ctypes.c_int() for _ in range(4)]
        self.lib.orc_get_sizes(self.h, *[ctypes.byref(x) for x in a])
        nPIs, nPOs, nAnds, nLevels = [x.value for x in a]
        n = 1 + nPIs + nAnds
        f0 = np.empty(n, np.int32)
        f1 = np.empty(n, np.int32)
        outs = np.empty(max(nPOs, 1), np.int32)
        self.lib.orc_get_graph(self.h, _ip(f0), _ip(f1), _ip(outs))
        return Graph(nPIs, f0, f1, outs[:nPOs], nLevels)

    # ---------------------------------------------------------- dumps
    def dump_sizes(self):
        a, b = ctypes.c_int(), ctypes.c_int()
        self.lib.orc_dump_sizes(self.h, ctypes.byref(a), ctypes.byref(b))
        return a.value, b.value

    def dump_reorder(self, nPOs):
        n0, _ = self.dump_sizes()
        f0 = np.empty(n0 + 1, np.int32)
        f1 = np.empty(n0 + 1, np.int32)
        outs = np.empty(max(nPOs, 1), np.int32)
        self.lib.orc_dump_reorder(self.h, _ip(f0), _ip(f1), _ip(outs))
        return f0, f1, outs[:nPOs]

    def dump_cuts(self):
        n0, _ = self.dump_sizes()
        out = np.empty((n0 + 1) * 8 * CUT_INTS, np.int32)
        self.lib.orc_dump_cuts(self.h, _ip(out))
        return out.reshape(n0 + 1, 8, CUT_INTS)

    def dump_selected(self):
        n0, _ = self.dump_sizes()
        out = np.empty((n0 + 1) * SEL_INTS, np.int32)
        self.lib.orc_dump_selected(self.h, _ip(out))
        return out.reshape(n0 + 1, SEL_INTS)

    def dump_replace(self):
        n0, n1 = self.dump_sizes()
        rep = np.empty(n0 + 1, np.int32)
        nf0 = np.empty(max(n1 - n0, 1), np.int32)
        nf1 = np.empty(max(n1 - n0, 1), np.int32)
        self.lib.orc_dump_replace(self.h, _ip(rep), _ip(nf0), _ip(nf1))
        return rep, nf0[:n1 - n0], nf1[:n1 - n0]

    def dump_choice(self):
        n0, _ = self.dump_sizes()
        out = np.empty(n0 + 1, np.int32)
        self.lib.orc_dump_choice(self.h, _ip(out))
        return out

    def dump_stats(self):
        out = (ctypes.c_longlong * 10)()
        self.lib.orc_dump_stats(self.h, out)
        return dict(zip(STAT_NAMES, list(out)))

    def prededup(self, nPIs, nPOs):
        a, b = ctypes.c_int(), ctypes.c_int()
        self.lib.orc_prededup_sizes(self.h, ctypes.byref(a), ctypes.byref(b))
        n = a.value
        f0 = np.empty(n, np.int32)
        f1 = np.empty(n, np.int32)
        outs = np.empty(max(nPOs, 1), np.int32)
        self.lib.orc_prededup_graph(self.h, _ip(f0), _ip(f1), _ip(outs))
        return Graph(nPIs, f0, f1, outs[:nPOs], b.value)


def rw_st(g: Graph, zeros=False, st=True):
    """Run `rw` (GPU dedup) then optionally `st` on the oracle; returns the graph."""
    o = Oracle()
    o.set_graph(g)
    o.rw(zeros=zeros, dedup=2)
    if st:
        o.st()
    return o.graph()


def simulate(g, words=4, seed=1):
    """PO words of g under seeded random PI patterns (C simulator)."""
    lib = _load()
    f0 = np.ascontiguousarray(g.fanin0, dtype=np.int32)
    f1 = np.ascontiguousarray(g.fanin1, dtype=np.int32)
    outs = np.ascontiguousarray(g.outs, dtype=np.int32) if len(g.outs) else np.zeros(1, np.int32)
    res = np.zeros(max(len(g.outs), 1) * words, dtype=np.uint64)
    rc = lib.orc_simulate(g.nPIs, len(g.outs), len(f0) - 1 - g.nPIs, _ip(f0), _ip(f1), _ip(outs), words, seed,
                          res.ctypes.data_as(ctypes.POINTER(ctypes.c_ulonglong)))
    if rc != 0:
        raise ValueError("simulate: not topological")
    return res[:len(g.outs) * words].reshape(len(g.outs), words)


def equivalent_sim(a, b, words=4, seed=1):
    return a.nPIs == b.nPIs and len(a.outs) == len(b.outs) and np.array_equal(simulate(a, words, seed),
                                                                                simulate(b, words, seed))
