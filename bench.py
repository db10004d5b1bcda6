"""Benchmark of `rw; st` (CULS AIG rewriting + strash) on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload c4|c4m|c3|c3m|c2|c1] [--impl ours|reference]

Metric: input AND nodes processed by one `rw; st` per second (whole job).
A step is one `rw; st` over the workload's graphs:
  c4  4,096 seeded layered AIGs, AND counts log-uniform 1k-200k, PIs 16-512,
      depth ~ sqrt(size), window-4 fanins, every sink a PO (batched mode, the
      headline workload; inputs ~1.2 GB, larger than the 126 MB L2)
  c3  one 10M-AND layered AIG, 4,096 PIs/POs, 2,000 layers, 80% window-3 /
      20% far fanins
  c2  64x64 array multiplier; c1  5,000-AND 40-layer AIG (parity cases)
  c5  served mode: Poisson arrivals (0.25, 0.5, 0.75 and --load x measured
      batch capacity; --jobs jobs per run, --repeats runs per load) of jobs
      drawn from 512 c4-family graphs of 500-2M ANDs and 512 n x n
      multipliers (n 8-128), submitted one by one through culs_submit under
      a 150 GB admission budget; reports throughput and p50/p99
      submit-to-done latency (the default c4 line carries a short run)
`value` times device-resident steps (a device clone of the input, rw, st);
`e2e` times the public C-ABI path from host arrays: upload, rw, st,
download; `e2e_aiger` the same from binary AIGER files' bytes to files'
bytes, decoded and encoded on the device.  With --gpus N (under torchrun) every rank rewrites its own
4,096 graphs (weak scaling, no data-path collective).
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

import numpy as np  # noqa: E402


def _load_dist():
    """culs_b200/dist.py loaded by path: importing it as culs_b200.dist would
    load the package and its CUDA library, which the reference arm must not."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("culs_b200_dist", ROOT / "culs_b200" / "dist.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


Group = _load_dist().Group

METRIC = "rw+st AND-nodes/sec"
UNIT = "AND-nodes/s"
# Kernels timed live (CUDA-event marks around their launches) with the
# algorithmic bytes each moves per input AND node; the roofline reports the
# one that takes longest.
KERNELS = {
    "k_enumerate": ("cut enumeration", 584),  # 2 fanin cut sets read + own set written
    # table build and evaluation alternate per group of graphs inside one
    # marked region: own cuts, fanins, refs, levels, table probes (328) plus
    # the build's byGraph, fanins, graph, level reads and slot write (36)
    "k_evaluate": ("existence-table build + MFFC + NPN match + gain", 364),
    "k_dedup": ("strash hashing dataflow", 52),  # fanins, level, map, table slot, key out
}


def make_workload(name, rank, gen=None):
    """The workload's graphs.  `gen` supplies the seeded generators: the
    product package by default; the reference arm passes oracle.workload,
    the same generator sources built without the product's CUDA library."""
    if gen is None:
        import culs_b200 as gen
    threads = os.cpu_count() or 8
    if name == "c4":
        return gen.gen_batch(4, rank * 4096, 4096, 1000, 200000, 16, 512, threads=threads)
    if name == "c5":  # the served workload's job pool
        return served_pool(gen=gen)
    if name == "c4m":  # profiling case: the first 256 graphs of the c4 family
        return gen.gen_batch(4, rank * 4096, 256, 1000, 200000, 16, 512, threads=threads)
    if name == "c3":
        return [gen.gen_layered(3 + rank, 4096, 4096, 10_000_000, 2000, 3, 0.2, False)]
    if name == "c3m":  # profiling case: a 1M-AND member of the c3 family
        return [gen.gen_layered(3 + rank, 4096, 4096, 1_000_000, 200, 3, 0.2, False)]
    if name == "c2":
        return [gen.gen_multiplier(64)]
    if name == "c1":
        return [gen.gen_layered(1 + rank, 64, 32, 5000, 40, 4, 0.0, True)]
    raise SystemExit(f"unknown workload {name}")


WORKLOAD_DESC = {"c5": "c5_served_poisson_500-2M_and_multipliers_8-128", "c4": "c4_batched_4096_layered_1k-200k", "c4m": "c4_family_batched_256_layered_1k-200k", "c3": "c3_single_10M_layered_2000",
                 "c3m": "c3_family_1M_layered_200", "c2": "c2_mult64x64", "c1": "c1_layered5k_40"}


class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""

    def __init__(self, device):
        self.device = device
        self.samples = []
        self.stop = threading.Event()
        self.th = None

    def _run(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        while not self.stop.is_set():
            try:
                r = subprocess.run(["nvidia-smi", "-i", str(self.device), f"--query-gpu={q}",
                                    "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                f = [x.strip() for x in r.stdout.strip().split(",")]
                if len(f) == 7:
                    self.samples.append(f)
            except Exception:
                pass
            self.stop.wait(0.2)

    def __enter__(self):
        self.th = threading.Thread(target=self._run, daemon=True)
        self.th.start()
        return self

    def __exit__(self, *a):
        self.stop.set()
        self.th.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if s[3 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": float(self.samples[0][1]), "reasons": reasons,
                "samples": len(sm)}


def measured_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def traffic_per_node(kernel, workload):
    """DRAM bytes per input AND node of `kernel` from its committed ncu
    summary (profiles/<kernel>_traffic.json), when that capture is of the
    same workload family (a smaller member, scaled by the AND nodes
    processed); (None, None) otherwise."""
    p = ROOT / "profiles" / f"{kernel}_traffic.json"
    if p.exists():
        d = json.loads(p.read_text())
        if workload in d.get("families", []):
            return float(d["dram_bytes_per_and_node"]), d.get("source", "")
    return None, None


def cpu_model():
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def cpu_baseline(name, graphs, budget_s=12.0, threads=None):
    """Times the CPU restatement of the reference rw;st (oracle/, kind
    "port") on a bounded sample of the workload, on `threads` host threads
    (ctypes releases the GIL, one graph per call)."""
    from oracle.oracle import Graph, Oracle
    from oracle import workload as W
    threads = threads or (os.cpu_count() or 1)
    if name in ("c3", "c3m"):  # the 10M graph takes minutes on one core: a 1M-AND member of the same family
        sample = [W.gen_layered(3, 4096, 4096, 1_000_000, 200, 3, 0.2, False)]
        desc = "c3 family (80% window-3 / 20% far fanins), one 1M-AND graph, 1 thread"
        threads = 1
    else:
        sample = list(graphs)
        desc = f"first graphs of the workload until {budget_s:.0f} s elapse, one graph per thread"

    def one(g):
        o = Oracle()
        o.set_graph(Graph(g.nPIs, g.fanin0, g.fanin1, g.outs))
        o.rw()
        o.st()
        return g.nAnds

    done = 0
    t0 = time.perf_counter()
    with ThreadPoolExecutor(max_workers=threads) as ex:
        futs = []
        it = iter(sample)
        for g in it:
            futs.append(ex.submit(one, g))
            if len(futs) >= threads:
                done += futs.pop(0).result()
                if time.perf_counter() - t0 > budget_s:
                    break
        for f in futs:
            done += f.result()
    dt = time.perf_counter() - t0
    return {"value": done / dt, "unit": UNIT, "cores": threads, "cpu_model": cpu_model(), "kind": "port",
            "sample": f"{desc}: {done} AND nodes in {dt:.1f} s"}


def reference_gpu_path(graphs, max_nodes=4_000_000, timeout_s=600):
    """The reference's own rw;st on the GPU, one graph at a time: its rewrite
    and strash compiled from the CULS sources (oracle/_ref/rw_harness, built
    by oracle/build_ref.sh), timed per graph with device synchronisation,
    best of 2 runs after a warm-up.  None when the harness or a GPU is
    missing."""
    import tempfile
    from oracle import workload as W
    exe = ROOT / "oracle" / "_ref" / "rw_harness"
    if not exe.exists():
        return None
    try:
        import torch
        if not torch.cuda.is_available():
            return None
    except Exception:
        return None
    with tempfile.TemporaryDirectory() as d:
        files, nodes = [], 0
        for i, g in enumerate(graphs):
            if nodes >= max_nodes:
                break
            f = Path(d) / f"g{i}.aig"
            W.write_aiger(f, g)
            files.append(str(f))
            nodes += g.nAnds
        r = subprocess.run([str(exe), "time", "2"] + files, capture_output=True, text=True, timeout=timeout_s)
        line = [l for l in r.stdout.splitlines() if l.startswith("HARNESS time")]
        if r.returncode != 0 or not line:
            return {"unavailable": f"reference harness exited {r.returncode}"}
        kv = dict(x.split("=") for x in line[0].split()[2:])
        ms = float(kv["ms"])
        return {"value": int(kv["and_nodes"]) / (ms / 1e3), "unit": UNIT, "kind": "reference GPU rw;st",
                "sample": f"{kv['files']} graphs one at a time, {kv['and_nodes']} AND nodes, "
                          "AIGMan::rewrite + strash per graph, best of 2"}


def reference_arm(args, group):
    """`--impl reference`: the reference's rw;st restated on the CPU (oracle
    port; the reference's own rw needs a GPU for cut enumeration, so it has no
    CPU implementation to run), all host threads, a bounded sample per step."""
    if group.rank != 0:
        return 0
    from oracle import workload as W
    graphs = make_workload(args.workload, 0, gen=W)
    budget = 6.0
    for _ in range(args.warmup):
        cpu_baseline(args.workload, graphs, budget_s=1.0)
    vals = [cpu_baseline(args.workload, graphs, budget_s=budget) for _ in range(args.steps)]
    v = statistics.median(x["value"] for x in vals)
    cb = dict(vals[0])
    cb["value"] = v
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int32", "data": "synthetic (seeded generators)",
            "config": {"workload": WORKLOAD_DESC[args.workload]}, "cpu_baseline": cb,
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if args.workload in ("c1", "c2", "c3m", "c4", "c4m"):
        line["reference_gpu_path"] = reference_gpu_path(graphs)
    print(json.dumps(line), flush=True)
    return 0


def plain_path(ctx, graphs, budget_s=8.0, e2e=False):
    """The plain single-graph path: the workload's graphs one at a time, each
    its own handle (device-resident clone + rw;st, or with e2e the whole
    upload + rw;st + download), for about budget_s seconds of graphs in
    workload order.  Returns AND nodes per second and the sample."""
    nodes, t_total, k = 0, 0.0, 0
    t_end = time.perf_counter() + budget_s
    while k < len(graphs) and time.perf_counter() < t_end:
        g = graphs[k]
        if e2e:
            t0 = time.perf_counter()
            d = ctx.upload(g)
            ctx.rw_st(d)
            d.download()
            t_total += time.perf_counter() - t0
        else:
            d0 = ctx.upload(g)
            d = ctx.clone(d0)
            ctx.sync()
            ctx.mark(0)
            ctx.rw_st(d)
            ctx.mark(1)
            ctx.sync()
            t_total += ctx.profile_read()["user"] / 1e3
            d0.free()
        d.free()
        nodes += g.nAnds
        k += 1
    return {"value": nodes / t_total if t_total > 0 else None, "unit": UNIT,
            "sample": f"first {k} graphs one at a time ({nodes} AND nodes)" +
                      (", upload + rw;st + download, wall clock" if e2e else ", device-resident, CUDA events")}


def served_pool(seed=5, count=1024, gen=None):
    """Job pool of the served workload: half seeded c4-family graphs with AND
    counts log-uniform in 500-2M, half n x n array multipliers, n uniform in
    8-128.  Jobs are drawn from the pool with repetition."""
    if gen is None:
        import culs_b200 as gen
    rng = np.random.default_rng(seed)
    pool = gen.gen_batch(seed, 0, count // 2, 500, 2_000_000, 16, 512, threads=os.cpu_count() or 8)
    pool += [gen.gen_multiplier(int(n)) for n in rng.integers(8, 129, count - count // 2)]
    return pool


SERVE_BUDGET = 150 * 10**9  # the served workload's HBM admission budget, bytes


def served_capacity(device, pool, runs=3):
    """Jobs per second when the whole pool runs as one batch from host arrays
    (upload, rw;st, download), median of `runs` after one untimed pass, on a
    context of its own that is closed afterwards (its arena would otherwise
    stay beside the served workers' engines).  (A burst through the served
    path is not a stable yardstick: how many jobs a free worker finds queued
    depends on thread timing.)"""
    import culs_b200 as C
    ctx = C.Context(device=device)
    caps = []
    for r in range(runs + 1):
        t0 = time.perf_counter()
        d = ctx.upload_batch(pool)
        ctx.rw_st(d)
        d.download_all()
        d.free()
        if r:
            caps.append(len(pool) / (time.perf_counter() - t0))
    ctx.close()
    return float(np.median(caps)), caps


def served_load(ctx, pool, rate, njobs, seed):
    """Poisson arrivals at `rate` jobs/s of `njobs` jobs drawn from the pool,
    each submitted through the C ABI (culs_submit) on this thread, waited for
    and fetched on another.  Returns (AND nodes/s from the first submission
    to the last fetch, sorted submit-to-done latencies in ms, picks)."""
    import threading
    rng = np.random.default_rng(seed)
    picks = rng.integers(0, len(pool), njobs)
    gaps = rng.exponential(1.0 / rate, njobs)
    lat, nodes, done_t, errors = [], [0], [0.0], []
    q = []
    cv = threading.Condition()

    def collector():
        for k in range(njobs):
            with cv:
                while len(q) <= k:
                    cv.wait()
                j = q[k]
            try:
                ctx.wait(j)
                out, ms = ctx.fetch(j)
            except Exception as e:  # a failed job is counted, not fatal
                errors.append(str(e))
                continue
            lat.append(ms)
            nodes[0] += pool[picks[k]].nAnds
        done_t[0] = time.perf_counter()

    th = threading.Thread(target=collector)
    th.start()
    t0 = time.perf_counter()
    due = t0
    for k in range(njobs):
        due += gaps[k]
        d = due - time.perf_counter()
        if d > 0:
            time.sleep(d)
        j = ctx.submit(pool[picks[k]])
        with cv:
            q.append(j)
            cv.notify()
    th.join()
    if errors:
        raise RuntimeError(f"{len(errors)} served jobs failed, first: {errors[0]}")
    return nodes[0] / (done_t[0] - t0), np.sort(np.array(lat)), picks


def served_session(device, pool, loads, njobs, repeats, workers, budget=SERVE_BUDGET, seed=5, max_batch=0):
    """Served mode at each offered load (a fraction of the batch capacity),
    `repeats` runs of `njobs` jobs each, on a fresh context: the median and
    the range of p50, p99 and throughput per load."""
    import culs_b200 as C
    cap, caps = served_capacity(device, pool)
    ctx = C.Context(device=device)
    ctx.serve_start(admit_bytes=budget, workers=workers, max_batch=max_batch)
    sweep = []
    try:
        for i, load in enumerate(loads):
            runs = []
            for r in range(repeats):
                v, lt, _ = served_load(ctx, pool, load * cap, njobs, seed + 100 * i + r)
                runs.append({"value": v, "p50_ms": float(np.percentile(lt, 50)),
                             "p99_ms": float(np.percentile(lt, 99)), "mean_ms": float(lt.mean()),
                             "max_ms": float(lt[-1])})
            med = {k: float(np.median([x[k] for x in runs])) for k in ("value", "p50_ms", "p99_ms")}
            sweep.append({"load_vs_capacity": load, "offered_jobs_per_s": load * cap, "jobs": njobs,
                          "repeats": repeats, **med,
                          "p50_range_ms": [min(x["p50_ms"] for x in runs), max(x["p50_ms"] for x in runs)],
                          "p99_range_ms": [min(x["p99_ms"] for x in runs), max(x["p99_ms"] for x in runs)],
                          "runs": runs})
    finally:
        ctx.serve_stop()
        ctx.close()
    return {"capacity_jobs_per_s": cap, "capacity_runs": caps, "budget_bytes": budget, "workers": workers,
            "max_batch": max_batch,
            "pool_graphs": len(pool), "pool_and_nodes": int(sum(g.nAnds for g in pool)), "sweep": sweep,
            "timing": "wall clock, submit to done"}


def served_arm(args, group):
    """Served mode (`--workload c5`): jobs drawn from the 1,024-graph pool
    arrive as a Poisson process at 0.25, 0.5 and 0.75 of the measured batch
    capacity (and --load), `--jobs` jobs per run, `--repeats` runs per load,
    under the 150 GB admission budget; reports throughput and p50/p99
    submit-to-done latency per load, and the plain one-at-a-time path on the
    same jobs."""
    import culs_b200 as C
    pool = served_pool()
    loads = sorted(set([0.25, 0.5, 0.75, args.load]))
    srv = served_session(group.local, pool, loads, args.jobs, args.repeats, args.workers, max_batch=args.max_batch)
    ctx = C.Context(device=group.local)
    at = [x for x in srv["sweep"] if x["load_vs_capacity"] == args.load][0]
    rng = np.random.default_rng(5)
    plain = plain_path(ctx, [pool[i] for i in rng.integers(0, len(pool), 400)], budget_s=8.0, e2e=True)
    line = {"metric": METRIC, "value": at["value"], "unit": UNIT, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int32",
            "data": "synthetic (seeded generators; CULS ships no benchmark inputs)",
            "config": {"workload": WORKLOAD_DESC["c5"], "jobs_per_run": args.jobs, "pool_graphs": len(pool),
                       "load_vs_capacity": args.load, "budget_bytes": SERVE_BUDGET,
                       "parallelism": f"single GPU, {args.workers} workers, continuous admission"},
            "latency_ms": {"p50": at["p50_ms"], "p99": at["p99_ms"]},
            "served": srv, "plain_single_graph_path": plain,
            "served_vs_plain": at["value"] / plain["value"] if plain["value"] else None,
            "e2e": {"value": at["value"], "unit": UNIT, "h2d_bytes_per_step": None, "d2h_bytes_per_step": None},
            "gpu_launches": ctx.kernel_launches()}
    print(json.dumps(line), flush=True)
    ctx.close()
    return 0


def parity_sample(ctx, graphs, dw, count=64, largest=8):
    """Checks the timed batch's outputs outside the timed region: a fixed
    sample of its graphs (the `largest` largest and the rest spread evenly
    over the batch) is downloaded from the batch result `dw` and compared
    node for node with the plain single-graph path run on the same input
    graph.  Returns the summary that goes into the JSON line."""
    import culs_b200 as C
    n = len(graphs)
    by_size = sorted(range(n), key=lambda i: -graphs[i].nAnds)
    pick = list(by_size[:largest])
    rest = [i for i in range(n) if i not in set(pick)]
    step = max(1, len(rest) // max(1, count - len(pick)))
    pick += rest[::step][:count - len(pick)]
    bad = []
    nodes = 0
    for i in sorted(pick):
        got = dw.download(i)
        d = ctx.upload(graphs[i])
        ctx.rw_st(d)
        ref = d.download()
        d.free()
        same = (np.array_equal(got.fanin0, ref.fanin0) and np.array_equal(got.fanin1, ref.fanin1)
                and np.array_equal(got.outs, ref.outs))
        if not same:
            bad.append(i)
        nodes += graphs[i].nAnds
    return {"checked": len(pick), "mismatches": len(bad), "mismatched_graphs": bad[:16],
            "and_nodes_checked": nodes, "largest_checked": graphs[by_size[0]].nAnds if n else 0,
            "against": "plain single-graph path on the same input graph, node for node"}


def parity_digest(dw, workload):
    """The single-graph workloads with a committed oracle digest
    (tests/golden/c3_layered10M.json: SHA-256 of the oracle's rw;st result on
    the same seeded graph) are checked against it."""
    import hashlib
    p = ROOT / "tests" / "golden" / "c3_layered10M.json"
    if workload != "c3" or not p.exists():
        return None
    want = json.loads(p.read_text())["rw_st"]
    got = dw.download(0)
    h = hashlib.sha256()
    for a in (got.fanin0, got.fanin1, got.outs):
        h.update(np.ascontiguousarray(np.asarray(a, np.int32)).tobytes())
    ok = h.hexdigest() == want["sha256"]
    return {"checked": 1, "mismatches": 0 if ok else 1, "and_nodes_checked": got.nAnds,
            "against": "oracle rw;st digest (tests/golden/c3_layered10M.json)"}


def single_graph_c2(ctx, reps=5):
    """Config 2 on the plain single-graph path: the 64x64 array multiplier,
    device-resident (clone + rw;st, CUDA events), median of `reps` runs after
    two warm-ups."""
    import culs_b200 as C
    g = C.gen_multiplier(64)
    d0 = ctx.upload(g)
    times = []
    for r in range(reps + 2):
        d = ctx.clone(d0)
        ctx.sync()
        ctx.mark(0)
        ctx.rw_st(d)
        ctx.mark(1)
        ctx.sync()
        if r >= 2:
            times.append(ctx.profile_read()["user"])
        d.free()
    d0.free()
    ms = statistics.median(times)
    return {"workload": WORKLOAD_DESC["c2"], "and_nodes": g.nAnds, "ms": ms, "value": g.nAnds / (ms / 1e3),
            "unit": UNIT, "runs_ms": [round(t, 3) for t in times]}


def our_arm(args, group):
    import culs_b200 as C
    ctx = C.Context(device=group.local)
    graphs = make_workload(args.workload, group.rank)
    n_and = sum(g.nAnds for g in graphs)
    in_bytes = sum(4 * (2 * g.nObjs + g.nPOs) for g in graphs)
    d0 = ctx.upload_batch(graphs)
    # the enumeration schedule, chosen by the autotuner on the workload
    # itself (clones; outside the timed region)
    tuned = ctx.autotune(d0, rounds=2)
    dw = ctx.clone(d0)
    ctx.profile(True)
    for _ in range(args.warmup):
        ctx.clone(d0, into=dw)
        ctx.rw_st(dw)
    ctx.sync()
    # device-resident steps
    group.barrier()
    ctx.sync()
    l0 = ctx.kernel_launches()
    with ClockSampler(group.local) as clk:
        ctx.mark(0)
        for _ in range(args.steps):
            ctx.clone(d0, into=dw)
            ctx.rw_st(dw)
        ctx.mark(1)
        ctx.sync()
    launches = ctx.kernel_launches() - l0
    prof = ctx.profile_read()
    t_ms = group.max(prof["user"])
    group.barrier()
    total_and = group.sum(n_and)
    value = total_and * args.steps / (t_ms / 1e3)
    out_and = sum(dw.stats(i)["nAnds"] for i in range(len(dw)))
    # end to end through the C ABI from host arrays
    e2e_steps = max(1, min(args.steps, 3))
    group.barrier()
    ctx.sync()
    ctx.mark(0)
    out_bytes = 0
    for _ in range(e2e_steps):
        d = ctx.upload_batch(graphs)
        ctx.rw_st(d)
        res = d.download_all()
        out_bytes = sum(4 * (2 * r.nObjs + r.nPOs) for r in res)
        d.free()
    ctx.mark(1)
    ctx.sync()
    e2e_ms = group.max(ctx.profile_read()["user"])
    e2e_value = total_and * e2e_steps / (e2e_ms / 1e3)
    # the same through binary AIGER files' bytes (the reference's read; rw;
    # st; write): decoded and encoded on the device
    files = d0.download_aiger_all()
    aig_in = sum(len(f) for f in files)
    group.barrier()
    ctx.sync()
    ctx.mark(0)
    aig_out = 0
    for _ in range(e2e_steps):
        d = ctx.upload_aiger_batch(files)
        ctx.rw_st(d)
        res = d.download_aiger_all()
        aig_out = sum(len(f) for f in res)
        d.free()
    ctx.mark(1)
    ctx.sync()
    aig_ms = group.max(ctx.profile_read()["user"])
    e2e_aiger = {"value": total_and * e2e_steps / (aig_ms / 1e3), "unit": UNIT, "h2d_bytes_per_step": aig_in,
                 "d2h_bytes_per_step": aig_out, "steps": e2e_steps,
                 "path": "binary AIGER bytes in and out (culs_batch_upload_aiger, culs_batch_download_aiger)"}
    # roofline of the dominant kernel
    peak, peak_kind = measured_peak()
    kname = max(KERNELS, key=lambda k: prof.get(k, 0.0))
    kdesc, alg = KERNELS[kname]
    k_ms = prof[kname]
    achieved = alg * n_and / (k_ms / 1e3) / 1e9 if k_ms > 0 else None
    tpn, tsrc = traffic_per_node(kname, args.workload)
    roof = {"kernel": f"{kname} ({kdesc})", "bound": "hbm", "achieved": achieved, "peak": peak,
            "peak_kind": f"{peak_kind} hbm_gbs", "unit": "GB/s", "frac": achieved / peak if achieved else None,
            "traffic": tpn * n_and if tpn else None, "traffic_source": tsrc,
            "algorithmic_bytes_per_and": alg, "launch_ms": k_ms,
            "kernel_ms": {k: prof.get(k) for k in KERNELS}}
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": group.world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int32",
            "data": "synthetic (seeded generators; CULS ships no benchmark inputs)",
            "config": {"workload": WORKLOAD_DESC[args.workload], "graphs_per_gpu": len(graphs),
                       "and_nodes_per_gpu": n_and, "and_nodes_out_per_gpu": out_and,
                       "input_bytes_per_gpu": in_bytes, "l2": "inputs and working set larger than L2",
                       "tuned": tuned,
                       "parallelism": f"graph-sharded x{group.world}" if group.world > 1 else "single GPU"},
            "roofline": roof,
            # the whole step against the same roof: 1,036 algorithmic bytes
            # per input AND node over every stage (enumerate 584, evaluate
            # 328, levels 20, two strash passes 2 x 52)
            "roofline_step": {"algorithmic_bytes_per_and": B_ALG_STEP, "achieved": value * B_ALG_STEP / 1e9,
                              "peak": peak, "unit": "GB/s", "frac": value * B_ALG_STEP / 1e9 / peak},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": in_bytes,
                    "d2h_bytes_per_step": out_bytes, "steps": e2e_steps},
            "e2e_aiger": e2e_aiger,
            "clocks": clk.summary(), "gpu_launches": launches,
            "stages_ms_last_step": {k: round(v, 3) for k, v in prof.items() if k not in ("user",)}}
    # parity of the timed result (outside the timed region): a sample of the
    # batch against the plain path, or the single graph against its digest
    if len(graphs) > 1:
        par = parity_sample(ctx, graphs, dw)
    else:
        par = parity_digest(dw, args.workload)
    line["parity"] = par
    bad = group.sum(par["mismatches"] if par else 0)
    dw.free()
    d0.free()
    if group.rank == 0:
        if group.world == 1 and len(graphs) > 1:
            plain = plain_path(ctx, graphs)
            line["plain_single_graph_path"] = plain
            line["batched_vs_plain"] = value / plain["value"] if plain["value"] else None
            line["single_graph_c2"] = single_graph_c2(ctx)
        line["cpu_baseline"] = cpu_baseline(args.workload, graphs) if group.world == 1 else None
    ctx.close()  # its arena makes room for the served run's engines
    if group.rank == 0:
        if group.world == 1 and len(graphs) > 1:
            if not args.no_served and args.workload == "c4":
                # a short served-mode run (the c5 workload's job mix, 256
                # pool graphs, 2,000 jobs at half the batch capacity, one
                # run) so the default line carries p50/p99 latency
                pool = served_pool(count=256)
                srv = served_session(group.local, pool, [0.5], 2000, 1, args.workers)
                x = srv["sweep"][0]
                line["served"] = {"workload": WORKLOAD_DESC["c5"], "pool_graphs": len(pool), "jobs": x["jobs"],
                                  "load_vs_capacity": 0.5, "offered_jobs_per_s": x["offered_jobs_per_s"],
                                  "value": x["value"], "unit": UNIT, "p50_ms": x["p50_ms"], "p99_ms": x["p99_ms"],
                                  "budget_bytes": srv["budget_bytes"], "workers": srv["workers"],
                                  "capacity_jobs_per_s": srv["capacity_jobs_per_s"],
                                  "timing": srv["timing"]}
                del pool
        print(json.dumps(line), flush=True)
    return 1 if bad else 0


B_ALG_STEP = 1036  # algorithmic bytes per input AND node of one rw; st step


def once(args):
    """One `rw; st` of the workload on a device-resident clone, nothing timed
    or printed but a one-line summary: the command the committed ncu
    summaries (profiles/) were captured from."""
    import culs_b200 as C
    ctx = C.Context()
    graphs = make_workload(args.workload, 0)
    d0 = ctx.upload_batch(graphs)
    d = ctx.clone(d0)
    ctx.rw_st(d)
    ctx.sync()
    print(json.dumps({"once": WORKLOAD_DESC.get(args.workload, args.workload), "graphs": len(graphs),
                      "and_nodes": sum(g.nAnds for g in graphs),
                      "and_nodes_out": sum(d.stats(i)["nAnds"] for i in range(len(d)))}), flush=True)
    ctx.close()
    return 0


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", default="c4", choices=["c4", "c4m", "c3", "c3m", "c2", "c1", "c5"])
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--load", type=float, default=0.75, help="c5: offered load as a fraction of measured capacity")
    ap.add_argument("--workers", type=int, default=2, help="c5: batches the served mode runs at once")
    ap.add_argument("--jobs", type=int, default=20000, help="c5: jobs per run")
    ap.add_argument("--repeats", type=int, default=3, help="c5: runs per offered load")
    ap.add_argument("--max-batch", type=int, default=0, help="c5: jobs per served batch at most (0: no cap)")
    ap.add_argument("--no-served", action="store_true",
                    help="c4: leave out the short served-mode run of the default line")
    ap.add_argument("--once", action="store_true",
                    help="one device-resident rw;st of the workload and exit (for profiler captures)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.once:
        return once(args)
    group = Group()
    try:
        if args.impl == "reference":
            rc = reference_arm(args, group)
        elif args.workload == "c5":
            rc = served_arm(args, group) if group.rank == 0 else 0
        else:
            rc = our_arm(args, group)
    finally:
        group.close()
    return rc


if __name__ == "__main__":
    sys.exit(main())
