"""Conversions between the product's Aig, the oracle's Graph and fixtures."""
import numpy as np

from oracle.oracle import Graph, Oracle


def to_oracle(a):
    return Graph(a.nPIs, a.fanin0, a.fanin1, a.outs)


def oracle_rw_st(a, zeros=False, st=True, dedup=2):
    o = Oracle()
    o.set_graph(to_oracle(a))
    o.rw(zeros=zeros, dedup=dedup)
    if st:
        o.st()
    return o


def same_graph(x, y):
    return (x.nPIs == y.nPIs and np.array_equal(np.asarray(x.fanin0), np.asarray(y.fanin0))
            and np.array_equal(np.asarray(x.fanin1), np.asarray(y.fanin1))
            and np.array_equal(np.asarray(x.outs), np.asarray(y.outs)))
