"""Seeded workload generators and binary AIGER writing for the reference
arm of bench.py, without the product library.

TEST INFRASTRUCTURE.  oracle/libworkload.so is compiled from the host-only
generator and AIGER sources of the package (culs_b200/csrc/host_gen.cpp and
host_aiger.cpp, plain C++ with no device code), so that the timed CPU port
of the reference and the reference's own GPU harness get exactly the graphs
the product's bench generates, while the reference arm's process loads no
part of the product's CUDA library.
"""
import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

from oracle.oracle import Graph

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
LIB_PATH = HERE / "libworkload.so"
SOURCES = [ROOT / "culs_b200" / "csrc" / "host_gen.cpp", ROOT / "culs_b200" / "csrc" / "host_aiger.cpp"]


def build(force=False):
    deps = SOURCES + [ROOT / "include" / "culs_b200.h", ROOT / "culs_b200" / "csrc" / "guard.hpp"]
    if force or not LIB_PATH.exists() or any(LIB_PATH.stat().st_mtime < d.stat().st_mtime for d in deps):
        subprocess.check_call(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-pthread", "-I", str(ROOT / "include"),
                               "-I", str(ROOT / "culs_b200" / "csrc"), "-o", str(LIB_PATH)] + [str(s) for s in SOURCES])
    return LIB_PATH


class _HostGraph(ctypes.Structure):
    _fields_ = [("nPIs", ctypes.c_int32), ("nPOs", ctypes.c_int32), ("nAnds", ctypes.c_int32),
                ("fanin0", ctypes.POINTER(ctypes.c_int32)), ("fanin1", ctypes.POINTER(ctypes.c_int32)),
                ("outs", ctypes.POINTER(ctypes.c_int32))]


_lib = None


def _load():
    global _lib
    if _lib is None:
        build()
        lib = ctypes.CDLL(str(LIB_PATH))
        hp = ctypes.POINTER(_HostGraph)
        lib.culs_gen_layered.argtypes = [ctypes.c_uint64, ctypes.c_int, ctypes.c_int, ctypes.c_int64, ctypes.c_int,
                                         ctypes.c_int, ctypes.c_double, ctypes.c_int, hp]
        lib.culs_gen_multiplier.argtypes = [ctypes.c_int, hp]
        lib.culs_gen_batch.argtypes = [ctypes.c_uint64, ctypes.c_int, ctypes.c_int, ctypes.c_int64, ctypes.c_int64,
                                       ctypes.c_int, ctypes.c_int, ctypes.c_int, hp]
        lib.culs_host_graph_free.argtypes = [hp]
        lib.culs_aiger_write.argtypes = [ctypes.c_char_p, hp]
        _lib = lib
    return _lib


def _take(h):
    n = 1 + h.nPIs + h.nAnds
    f0 = np.ctypeslib.as_array(h.fanin0, (n,)).copy()
    f1 = np.ctypeslib.as_array(h.fanin1, (n,)).copy()
    outs = np.ctypeslib.as_array(h.outs, (max(h.nPOs, 1),))[:h.nPOs].copy()
    _lib.culs_host_graph_free(ctypes.byref(h))
    return Graph(h.nPIs, f0, f1, outs)


def gen_layered(seed, nPIs, nPOs, nAnds, nLayers, window, pFar=0.0, withPIs=True):
    lib = _load()
    h = _HostGraph()
    if lib.culs_gen_layered(seed, nPIs, nPOs, nAnds, nLayers, window, pFar, int(withPIs), ctypes.byref(h)) != 0:
        raise RuntimeError("gen_layered failed")
    return _take(h)


def gen_multiplier(n):
    lib = _load()
    h = _HostGraph()
    if lib.culs_gen_multiplier(n, ctypes.byref(h)) != 0:
        raise RuntimeError("gen_multiplier failed")
    return _take(h)


def gen_batch(tag, first, count, minAnds, maxAnds, minPIs, maxPIs, threads=None):
    lib = _load()
    arr = (_HostGraph * count)()
    if lib.culs_gen_batch(tag, first, count, minAnds, maxAnds, minPIs, maxPIs, threads or os.cpu_count() or 8,
                          arr) != 0:
        raise RuntimeError("gen_batch failed")
    return [_take(arr[i]) for i in range(count)]


def write_aiger(path, g):
    lib = _load()
    f0 = np.ascontiguousarray(g.fanin0, np.int32)
    f1 = np.ascontiguousarray(g.fanin1, np.int32)
    outs = np.ascontiguousarray(g.outs, np.int32) if len(g.outs) else np.zeros(1, np.int32)
    ip = ctypes.POINTER(ctypes.c_int32)
    h = _HostGraph(g.nPIs, len(g.outs), len(f0) - 1 - g.nPIs, f0.ctypes.data_as(ip), f1.ctypes.data_as(ip),
                   outs.ctypes.data_as(ip))
    if lib.culs_aiger_write(str(path).encode(), ctypes.byref(h)) != 0:
        raise RuntimeError(f"write {path} failed")
