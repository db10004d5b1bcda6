"""culs_b200 -- B200 implementation of CULS's `rw` (AIG rewriting) and `st`
(structural hashing with dangling-node removal).

Python mirror of the reference's AIG manager surface (CULS
src/aig_manager.h:13-26: readFile / saveFile / rewrite / strash /
printStats) over the C ABI in include/culs_b200.h.  The compute path is the
in-tree libculs_b200.so; importing this package fails if it is missing.
"""
import ctypes
from dataclasses import dataclass
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
LIB_PATH = _HERE / "libculs_b200.so"

if not LIB_PATH.exists():
    raise ImportError(f"{LIB_PATH} is missing: build it with `python -m culs_b200.build`")

_lib = ctypes.CDLL(str(LIB_PATH))

CULS_OK = 0
CULS_E_INVALID = -1
CULS_E_OOM = -2
CULS_E_BUDGET = -3
CULS_E_PROBE = -4
CULS_E_DEVICE = -5
CULS_E_IO = -6
CULS_E_BUSY = -7
CULS_E_NOTFOUND = -8
CULS_E_CANCELLED = -9
ERRORS = {-1: "CULS_E_INVALID", -2: "CULS_E_OOM", -3: "CULS_E_BUDGET", -4: "CULS_E_PROBE", -5: "CULS_E_DEVICE",
          -6: "CULS_E_IO", -7: "CULS_E_BUSY", -8: "CULS_E_NOTFOUND", -9: "CULS_E_CANCELLED"}
RW_ZEROS, RW_GPU_DEDUP, RW_DUMP = 1, 2, 4
SERVE_BYTES_PER_OBJ = 720  # device bytes the served mode's admission charges per object
ST_CPU = 1
B_NO_STRASH = 1
STAT_NAMES = ["replaced", "replaced_pos", "replaced_zero", "reverted", "compromised", "pre_eval", "small_cut",
              "new_idx", "expected", "new_nodes", "candidates", "enum_warp_pairs", "hash_rounds"]
DUMPS = ["reorder_f0", "reorder_f1", "reorder_out", "cuts", "selected", "replace", "new_f0", "new_f1", "choice"]


class CulsError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class _HostGraph(ctypes.Structure):
    _fields_ = [("nPIs", ctypes.c_int32), ("nPOs", ctypes.c_int32), ("nAnds", ctypes.c_int32),
                ("fanin0", ctypes.POINTER(ctypes.c_int32)), ("fanin1", ctypes.POINTER(ctypes.c_int32)),
                ("outs", ctypes.POINTER(ctypes.c_int32))]


_vp = ctypes.c_void_p
_ip = ctypes.POINTER(ctypes.c_int32)
_lib.culs_create.restype = _vp
_lib.culs_create.argtypes = [ctypes.c_size_t]
_lib.culs_destroy.argtypes = [_vp]
_lib.culs_set_device.argtypes = [ctypes.c_int]
_lib.culs_last_error.restype = ctypes.c_char_p
_lib.culs_last_error.argtypes = [_vp]
_lib.culs_sync.argtypes = [_vp]
_lib.culs_graph_upload.argtypes = [_vp, _ip, _ip, _ip, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                   ctypes.POINTER(_vp)]
_lib.culs_batch_upload.argtypes = [_vp, ctypes.c_int, ctypes.POINTER(_HostGraph), ctypes.POINTER(_vp)]
_lib.culs_batch_upload_aiger.argtypes = [_vp, ctypes.c_int, _vp, ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(_vp)]
_lib.culs_batch_download_aiger_into.argtypes = [_vp, _vp, _vp, ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)]
_lib.culs_batch_download_aiger.argtypes = [_vp, _vp, ctypes.POINTER(_vp), ctypes.POINTER(ctypes.c_size_t)]
_lib.culs_buffer_free.argtypes = [_vp]
_lib.culs_buffer_free.restype = None
_lib.culs_graph_free.argtypes = [_vp]
_lib.culs_graph_count.argtypes = [_vp]
_lib.culs_graph_stats.argtypes = [_vp, ctypes.c_int, _ip, _ip, _ip, _ip]
_lib.culs_batch_stats.argtypes = [_vp, _ip, _ip, _ip, _ip]
_lib.culs_batch_download.argtypes = [_vp, _vp, ctypes.POINTER(_HostGraph)]
_lib.culs_batch_download_into.argtypes = [_vp, _vp, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
_lib.culs_set_param.argtypes = [_vp, ctypes.c_int, ctypes.c_int64]
_lib.culs_get_param.argtypes = [_vp, ctypes.c_int, ctypes.POINTER(ctypes.c_int64)]
_lib.culs_autotune.argtypes = [_vp, _vp, ctypes.c_int]
_lib.culs_rw_st_batch.argtypes = [_vp, ctypes.c_void_p, ctypes.c_int, ctypes.c_uint32, ctypes.c_uint32]
_lib.culs_serve_start.argtypes = [_vp, ctypes.c_size_t, ctypes.c_int, ctypes.c_int]
_lib.culs_serve_stop.argtypes = [_vp]
_lib.culs_submit.argtypes = [_vp, _ip, _ip, _ip, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_uint32,
                             ctypes.c_uint32, ctypes.POINTER(ctypes.c_int64)]
_lib.culs_poll.argtypes = [_vp, ctypes.c_int64, _ip, _ip, _ip, _ip]
_lib.culs_wait.argtypes = [_vp, ctypes.c_int64, ctypes.c_int]
_lib.culs_cancel.argtypes = [_vp, ctypes.c_int64]
_lib.culs_fetch.argtypes = [_vp, ctypes.c_int64, _ip, _ip, _ip, ctypes.POINTER(ctypes.c_double)]
_lib.culs_submit_aiger.argtypes = [_vp, _vp, ctypes.c_size_t, ctypes.c_uint32, ctypes.c_uint32,
                                   ctypes.POINTER(ctypes.c_int64)]
_lib.culs_fetch_aiger.argtypes = [_vp, ctypes.c_int64, _vp, ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t),
                                  ctypes.POINTER(ctypes.c_double)]
_lib.culs_graph_download.argtypes = [_vp, _vp, ctypes.c_int, _ip, _ip, _ip]
_lib.culs_rw.argtypes = [_vp, _vp, ctypes.c_uint32]
_lib.culs_st.argtypes = [_vp, _vp, ctypes.c_uint32]
_lib.culs_b.argtypes = [_vp, _vp, ctypes.c_uint32]
_lib.culs_rw_st.argtypes = [_vp, _vp, ctypes.c_uint32, ctypes.c_uint32]
_lib.culs_rw_stats.argtypes = [_vp, ctypes.POINTER(ctypes.c_int64), ctypes.c_int]
_lib.culs_dump_size.restype = ctypes.c_int64
_lib.culs_dump_size.argtypes = [_vp, ctypes.c_int]
_lib.culs_dump_copy.argtypes = [_vp, ctypes.c_int, _ip]
_lib.culs_kernel_launches.restype = ctypes.c_int64
_lib.culs_kernel_launches.argtypes = [_vp]
_lib.culs_graph_clone.argtypes = [_vp, _vp, ctypes.POINTER(_vp)]
_lib.culs_profile.argtypes = [_vp, ctypes.c_int]
_lib.culs_mark.argtypes = [_vp, ctypes.c_int]
_lib.culs_profile_read.argtypes = [_vp, ctypes.POINTER(ctypes.c_float), ctypes.c_int]
_lib.culs_aiger_read.argtypes = [ctypes.c_char_p, ctypes.POINTER(_HostGraph)]
_lib.culs_aiger_write.argtypes = [ctypes.c_char_p, ctypes.POINTER(_HostGraph)]
_lib.culs_gen_layered.argtypes = [ctypes.c_uint64, ctypes.c_int, ctypes.c_int, ctypes.c_int64, ctypes.c_int,
                                  ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.POINTER(_HostGraph)]
_lib.culs_gen_multiplier.argtypes = [ctypes.c_int, ctypes.POINTER(_HostGraph)]
_lib.culs_gen_batch.argtypes = [ctypes.c_uint64, ctypes.c_int, ctypes.c_int, ctypes.c_int64, ctypes.c_int64,
                                ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(_HostGraph)]
_lib.culs_host_graph_free.argtypes = [ctypes.POINTER(_HostGraph)]


def _p(a):
    return a.ctypes.data_as(_ip)


@dataclass
class Aig:
    """AIG in the AIGMan layout: fanin arrays over objects 0..nObjs-1
    (entries 0..nPIs are -1), literal 0 = constant TRUE."""
    nPIs: int
    fanin0: np.ndarray
    fanin1: np.ndarray
    outs: np.ndarray
    nLevels: int = -1

    @property
    def nObjs(self):
        return len(self.fanin0)

    @property
    def nAnds(self):
        return self.nObjs - 1 - self.nPIs

    @property
    def nPOs(self):
        return len(self.outs)

    def host(self):
        """A culs_host_graph view (keeps references to the arrays); built
        once and reused while the three arrays stay the same objects."""
        c = self.__dict__.get("_hostc")
        if c is not None and c[0] is self.fanin0 and c[1] is self.fanin1 and c[2] is self.outs and c[3] == self.nPIs:
            return c[4]
        self.fanin0 = np.ascontiguousarray(self.fanin0, dtype=np.int32)
        self.fanin1 = np.ascontiguousarray(self.fanin1, dtype=np.int32)
        self.outs = np.ascontiguousarray(self.outs, dtype=np.int32)
        h = _HostGraph(self.nPIs, self.nPOs, self.nAnds, _p(self.fanin0), _p(self.fanin1), _p(self.outs))
        self.__dict__["_hostc"] = (self.fanin0, self.fanin1, self.outs, self.nPIs, h)
        return h


def _take(h: _HostGraph) -> Aig:
    n = 1 + h.nPIs + h.nAnds
    f0 = np.ctypeslib.as_array(h.fanin0, (n,)).copy()
    f1 = np.ctypeslib.as_array(h.fanin1, (n,)).copy()
    outs = np.ctypeslib.as_array(h.outs, (max(h.nPOs, 1),))[:h.nPOs].copy()
    _lib.culs_host_graph_free(ctypes.byref(h))
    return Aig(h.nPIs, f0, f1, outs)


def _check(rc, what=""):
    if rc != CULS_OK:
        raise CulsError(rc, what)


def read_aiger(path) -> Aig:
    h = _HostGraph()
    _check(_lib.culs_aiger_read(str(path).encode(), ctypes.byref(h)), f"read {path}")
    return _take(h)


def write_aiger(path, g: Aig):
    hg = g.host()
    _check(_lib.culs_aiger_write(str(path).encode(), ctypes.byref(hg)), f"write {path}")


def gen_layered(seed, nPIs, nPOs, nAnds, nLayers, window, pFar=0.0, withPIs=True) -> Aig:
    h = _HostGraph()
    _check(_lib.culs_gen_layered(seed, nPIs, nPOs, nAnds, nLayers, window, pFar, int(withPIs), ctypes.byref(h)),
           "gen_layered")
    return _take(h)


def gen_multiplier(n) -> Aig:
    h = _HostGraph()
    _check(_lib.culs_gen_multiplier(n, ctypes.byref(h)), "gen_multiplier")
    return _take(h)


def gen_batch(tag, first, count, minAnds, maxAnds, minPIs, maxPIs, threads=8):
    arr = (_HostGraph * count)()
    _check(_lib.culs_gen_batch(tag, first, count, minAnds, maxAnds, minPIs, maxPIs, threads, arr), "gen_batch")
    return [_take(arr[i]) for i in range(count)]


class Context:
    """One GPU context (stream, rewriting library, scratch arena)."""

    def __init__(self, hbm_budget=0, device=None):
        if device is not None:
            _check(_lib.culs_set_device(int(device)), "set device")
        self.h = _lib.culs_create(hbm_budget)
        if not self.h:
            raise CulsError(-5, _lib.culs_last_error(None).decode())

    def close(self):
        if getattr(self, "h", None):
            _lib.culs_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def _err(self, rc, what):
        if rc != CULS_OK:
            raise CulsError(rc, f"{what}: {_lib.culs_last_error(self.h).decode()}")

    def upload(self, g: Aig) -> "DeviceGraphs":
        out = _vp()
        hg = g.host()
        self._err(_lib.culs_graph_upload(self.h, hg.fanin0, hg.fanin1, hg.outs, g.nPIs, g.nPOs, g.nAnds,
                                         ctypes.byref(out)), "upload")
        return DeviceGraphs(self, out)

    def upload_aiger_batch(self, files) -> "DeviceGraphs":
        """Binary AIGER files' contents (bytes or any contiguous byte
        buffer), decoded on the device; nothing is copied on the way in."""
        n = len(files)
        keep, addr = [], np.empty(max(n, 1), np.uint64)
        for i, f in enumerate(files):
            if isinstance(f, bytes):
                c = ctypes.c_char_p(f)
                keep.append(c)
                addr[i] = ctypes.cast(c, ctypes.c_void_p).value or 0
            else:
                a = np.frombuffer(f, np.uint8)
                keep.append(a)
                addr[i] = a.ctypes.data
        lens = (ctypes.c_size_t * max(n, 1))(*[len(f) for f in files])
        out = _vp()
        self._err(_lib.culs_batch_upload_aiger(self.h, n, addr.ctypes.data, lens, ctypes.byref(out)), "AIGER upload")
        return DeviceGraphs(self, out)

    def upload_batch(self, graphs) -> "DeviceGraphs":
        arr = (_HostGraph * len(graphs))(*[g.host() for g in graphs])
        out = _vp()
        self._err(_lib.culs_batch_upload(self.h, len(graphs), arr, ctypes.byref(out)), "batch upload")
        return DeviceGraphs(self, out)

    def rw(self, d, zeros=False, gpu_dedup=True, dump=False):
        f = (RW_ZEROS if zeros else 0) | (RW_GPU_DEDUP if gpu_dedup else 0) | (RW_DUMP if dump else 0)
        self._err(_lib.culs_rw(self.h, d.h, f), "rw")

    def st(self, d, cpu=False):
        self._err(_lib.culs_st(self.h, d.h, ST_CPU if cpu else 0), "st")

    def b(self, d, update_level=True):
        """`b`: balance (sortDecId 1) every graph of d, then strash unless
        update_level is False (the balance as resyn2 calls it)."""
        self._err(_lib.culs_b(self.h, d.h, 0 if update_level else B_NO_STRASH), "b")

    def rw_st(self, d, zeros=False, gpu_dedup=True, cpu_st=False):
        f = (RW_ZEROS if zeros else 0) | (RW_GPU_DEDUP if gpu_dedup else 0)
        self._err(_lib.culs_rw_st(self.h, d.h, f, ST_CPU if cpu_st else 0), "rw;st")

    def rw_st_batch(self, handles, zeros=False, gpu_dedup=True, cpu_st=False):
        """`rw; st` over several device handles in one pass."""
        f = (RW_ZEROS if zeros else 0) | (RW_GPU_DEDUP if gpu_dedup else 0)
        arr = (_vp * len(handles))(*[d.h for d in handles])
        self._err(_lib.culs_rw_st_batch(self.h, ctypes.cast(arr, ctypes.c_void_p), len(handles), f,
                                        ST_CPU if cpu_st else 0), "rw;st batch")

    # ---- tuning (speed only; results never change)
    PARAMS = {"enum_wide_min": 1, "enum_blocks_per_sm": 2, "sm_share": 4, "high_priority": 5, "eval_group_mslots": 6}

    def set_param(self, name, value):
        self._err(_lib.culs_set_param(self.h, self.PARAMS[name], value), f"set_param {name}")

    def get_param(self, name):
        v = ctypes.c_int64()
        self._err(_lib.culs_get_param(self.h, self.PARAMS[name], ctypes.byref(v)), f"get_param {name}")
        return v.value

    def autotune(self, sample, rounds=1):
        """Chooses the enumeration schedule by timing it on clones of the
        device handle `sample`; returns the chosen parameters."""
        self._err(_lib.culs_autotune(self.h, sample.h, rounds), "autotune")
        return {k: self.get_param(k) for k in self.PARAMS}

    # ---- served mode
    def serve_start(self, admit_bytes=0, max_batch=0, workers=0):
        self._err(_lib.culs_serve_start(self.h, admit_bytes, max_batch, workers), "serve start")

    def serve_stop(self):
        self._err(_lib.culs_serve_stop(self.h), "serve stop")

    def submit(self, g: Aig, zeros=False, gpu_dedup=True, cpu_st=False) -> int:
        f = (RW_ZEROS if zeros else 0) | (RW_GPU_DEDUP if gpu_dedup else 0)
        h = g.host()
        job = ctypes.c_int64()
        self._err(_lib.culs_submit(self.h, h.fanin0, h.fanin1, h.outs, h.nPIs, h.nPOs, h.nAnds, f,
                                   ST_CPU if cpu_st else 0, ctypes.byref(job)), "submit")
        return job.value

    def poll(self, job):
        """None while the job runs, else its result sizes."""
        v = [ctypes.c_int32() for _ in range(4)]
        rc = _lib.culs_poll(self.h, job, *[ctypes.byref(x) for x in v])
        if rc == CULS_E_BUSY:
            return None
        self._err(rc, "poll")
        return dict(zip(["nPIs", "nPOs", "nAnds", "nLevels"], [x.value for x in v]))

    def wait(self, job, timeout_ms=-1):
        rc = _lib.culs_wait(self.h, job, timeout_ms)
        if rc == CULS_E_BUSY:
            return False
        self._err(rc, "wait")
        return True

    def cancel(self, job):
        """Takes a queued job out of the queue (it ends with CULS_E_CANCELLED);
        raises CulsError(CULS_E_BUSY) once its batch runs."""
        self._err(_lib.culs_cancel(self.h, job), "cancel")

    def fetch(self, job):
        """The finished job's result and its submit-to-done latency in ms.  A
        job that failed or was cancelled raises its code and is forgotten."""
        v = [ctypes.c_int32() for _ in range(4)]
        rc = _lib.culs_poll(self.h, job, *[ctypes.byref(x) for x in v])
        if rc == CULS_E_BUSY:
            raise CulsError(CULS_E_BUSY, "fetch: job still running")
        if rc not in (0, CULS_E_NOTFOUND):
            _lib.culs_fetch(self.h, job, None, None, None, None)  # forgets the failed job
        self._err(rc, "fetch")
        st = dict(zip(["nPIs", "nPOs", "nAnds", "nLevels"], [x.value for x in v]))
        n = 1 + st["nPIs"] + st["nAnds"]
        f0, f1 = np.empty(n, np.int32), np.empty(n, np.int32)
        outs = np.empty(max(st["nPOs"], 1), np.int32)
        lat = ctypes.c_double()
        self._err(_lib.culs_fetch(self.h, job, _p(f0), _p(f1), _p(outs), ctypes.byref(lat)), "fetch")
        return Aig(st["nPIs"], f0, f1, outs[:st["nPOs"]], st["nLevels"]), lat.value

    def submit_aiger(self, data, zeros=False, gpu_dedup=True, cpu_st=False) -> int:
        """A served job given as a binary AIGER file's bytes."""
        f = (RW_ZEROS if zeros else 0) | (RW_GPU_DEDUP if gpu_dedup else 0)
        a = np.frombuffer(data, np.uint8)
        job = ctypes.c_int64()
        self._err(_lib.culs_submit_aiger(self.h, a.ctypes.data if len(a) else None, len(a), f,
                                         ST_CPU if cpu_st else 0, ctypes.byref(job)), "submit")
        return job.value

    def fetch_aiger(self, job):
        """The finished AIGER job's result (bytes) and its latency in ms."""
        n = ctypes.c_size_t()
        self._err(_lib.culs_fetch_aiger(self.h, job, None, 0, ctypes.byref(n), None), "fetch")
        buf = ctypes.create_string_buffer(max(n.value, 1))
        lat = ctypes.c_double()
        self._err(_lib.culs_fetch_aiger(self.h, job, buf, n.value, ctypes.byref(n), ctypes.byref(lat)), "fetch")
        return buf.raw[:n.value], lat.value

    def rw_stats(self):
        out = (ctypes.c_int64 * len(STAT_NAMES))()
        _lib.culs_rw_stats(self.h, out, len(STAT_NAMES))
        return dict(zip(STAT_NAMES, list(out)))

    def dump(self):
        res = {}
        for i, name in enumerate(DUMPS):
            n = _lib.culs_dump_size(self.h, i)
            a = np.empty(max(n, 1), np.int32)
            _lib.culs_dump_copy(self.h, i, _p(a))
            res[name] = a[:n]
        return res

    PROFILE_NAMES = ["front", "enumerate", "evaluate", "replace", "choice", "redundancy", "dedup", "st",
                     "k_enumerate", "k_evaluate", "k_dedup", "user", "k_level"]

    def clone(self, d, into=None):
        if into is not None:
            self._err(_lib.culs_graph_clone(self.h, d.h, ctypes.byref(into.h)), "clone")
            return into
        out = _vp()
        self._err(_lib.culs_graph_clone(self.h, d.h, ctypes.byref(out)), "clone")
        return DeviceGraphs(self, out)

    def profile(self, on=True):
        _lib.culs_profile(self.h, int(on))

    def mark(self, slot):
        _lib.culs_mark(self.h, slot)

    def profile_read(self):
        n = len(self.PROFILE_NAMES)
        out = (ctypes.c_float * n)()
        _lib.culs_profile_read(self.h, out, n)
        return dict(zip(self.PROFILE_NAMES, [float(x) for x in out]))

    def kernel_launches(self):
        return _lib.culs_kernel_launches(self.h)

    def sync(self):
        self._err(_lib.culs_sync(self.h), "sync")


class DeviceGraphs:
    """Handle of one or more AIGs resident in device memory."""

    def __init__(self, ctx: Context, h):
        self.ctx = ctx
        self.h = h

    def free(self):
        if getattr(self, "h", None):
            _lib.culs_graph_free(self.h)
            self.h = None

    def __del__(self):
        self.free()

    def __len__(self):
        return _lib.culs_graph_count(self.h)

    def stats(self, i=0):
        v = [ctypes.c_int32() for _ in range(4)]
        _check(_lib.culs_graph_stats(self.h, i, *[ctypes.byref(x) for x in v]), "stats")
        return dict(zip(["nPIs", "nPOs", "nAnds", "nLevels"], [x.value for x in v]))

    def download_aiger_all(self):
        """Every graph of the handle as binary AIGER file contents, encoded
        on the device: memoryviews into one buffer holding the files back to
        back (bytes(view) copies one out)."""
        n = len(self)
        off = (ctypes.c_size_t * (n + 1))()
        self.ctx._err(_lib.culs_batch_download_aiger_into(self.ctx.h, self.h, None, 0, off), "AIGER download")
        buf = np.empty(max(off[n], 1), np.uint8)
        self.ctx._err(_lib.culs_batch_download_aiger_into(self.ctx.h, self.h, buf.ctypes.data, off[n], off),
                      "AIGER download")
        mv = memoryview(buf)
        o = list(off)
        return [mv[o[i]:o[i + 1]] for i in range(n)]

    def stats_all(self):
        """nPIs, nPOs, nAnds, nLevels of every graph, as int32 arrays."""
        n = len(self)
        v = [np.empty(max(n, 1), np.int32) for _ in range(4)]
        _check(_lib.culs_batch_stats(self.h, *[_p(x) for x in v]), "stats")
        return dict(zip(["nPIs", "nPOs", "nAnds", "nLevels"], [x[:n] for x in v]))

    def download_all(self):
        """Every graph of the handle as an Aig, in one transfer (the graphs'
        arrays are views of three buffers)."""
        n = len(self)
        st = self.stats_all()
        nobj = 1 + st["nPIs"].astype(np.int64) + st["nAnds"]
        npo = st["nPOs"].astype(np.int64)
        o0 = np.zeros(n + 1, np.int64)
        np.cumsum(nobj, out=o0[1:])
        p0 = np.zeros(n + 1, np.int64)
        np.cumsum(npo, out=p0[1:])
        F0 = np.empty(max(int(o0[-1]), 1), np.int32)
        F1 = np.empty(max(int(o0[-1]), 1), np.int32)
        PO = np.empty(max(int(p0[-1]), 1), np.int32)
        ptrs = [np.ascontiguousarray(B.ctypes.data + 4 * off[:n], dtype=np.uint64) for B, off in ((F0, o0), (F1, o0), (PO, p0))]
        self.ctx._err(_lib.culs_batch_download_into(self.ctx.h, self.h, *[x.ctypes.data_as(ctypes.c_void_p) for x in ptrs]),
                      "batch download")
        nP, nL = st["nPIs"].tolist(), st["nLevels"].tolist()
        a, b = o0.tolist(), p0.tolist()
        return [Aig(nP[i], F0[a[i]:a[i + 1]], F1[a[i]:a[i + 1]], PO[b[i]:b[i + 1]], nL[i]) for i in range(n)]

    def download(self, i=0) -> Aig:
        s = self.stats(i)
        n = 1 + s["nPIs"] + s["nAnds"]
        f0 = np.empty(n, np.int32)
        f1 = np.empty(n, np.int32)
        outs = np.empty(max(s["nPOs"], 1), np.int32)
        self.ctx._err(_lib.culs_graph_download(self.ctx.h, self.h, i, _p(f0), _p(f1), _p(outs)), "download")
        return Aig(s["nPIs"], f0, f1, outs[:s["nPOs"]], s["nLevels"])


class AIGMan:
    """Mirror of CULS's AIGMan command surface for one graph
    (src/aig_manager.h:13-26)."""

    def __init__(self, ctx: Context = None):
        self.ctx = ctx or Context()
        self.dev = None

    def readFile(self, path):
        self.dev = self.ctx.upload(read_aiger(path))
        return 1

    def load(self, g: Aig):
        self.dev = self.ctx.upload(g)

    def saveFile(self, path):
        write_aiger(path, self.dev.download())

    def rewrite(self, fUseZeros=False, fGPUDeduplicate=True):
        self.ctx.rw(self.dev, zeros=fUseZeros, gpu_dedup=fGPUDeduplicate)

    def strash(self, fCPU=False):
        self.ctx.st(self.dev, cpu=fCPU)

    def balance(self, sortDecId=1, updateLevel=True):
        if sortDecId != 1:
            raise CulsError(CULS_E_INVALID, "balance: only sortDecId 1 (the `b` default) is provided")
        self.ctx.b(self.dev, update_level=updateLevel)

    def printStats(self):
        s = self.dev.stats()
        return f"AIG stats: i/o = {s['nPIs']}/{s['nPOs']} and = {s['nAnds']} level = {s['nLevels']}"
