"""Graph-sharded multi-process plumbing (culs_b200/dist.py) on CPU with the
gloo backend: under torchrun every rank rewrites its own graphs, and the
ranks only meet for the timing barrier and the max / sum reductions of
bench.py.  Two ranks reduce as bench.py expects, the shards cover every
graph once, and a rank whose peer never joins ends with an error instead of
waiting."""
import multiprocessing as mp
import os
import socket

from culs_b200.dist import shard


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def rank_main(rank, world, port, q, timeout_s):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port), CULS_PG_TIMEOUT_S=str(timeout_s))
    try:
        from culs_b200.dist import Group
        g = Group(backend="gloo")
        g.barrier()
        mx = g.max(10.0 * (rank + 1))
        sm = g.sum(rank + 1)
        lo, hi = shard(10, g.rank, g.world)
        g.close()
        q.put((rank, mx, sm, lo, hi))
    except Exception as e:  # reported to the test process
        q.put((rank, "error", type(e).__name__))


def test_shards_cover_every_graph_once():
    for count in (0, 1, 7, 4096):
        for world in (1, 2, 3, 8):
            seen = []
            for r in range(world):
                lo, hi = shard(count, r, world)
                assert hi - lo in (count // world, count // world + 1)
                seen += list(range(lo, hi))
            assert seen == list(range(count))


def test_two_ranks_reduce_over_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    ps = [ctx.Process(target=rank_main, args=(r, 2, port, q, 60)) for r in range(2)]
    for p in ps:
        p.start()
    res = sorted(q.get(timeout=180) for _ in ps)
    for p in ps:
        p.join(timeout=60)
    assert res == [(0, 20.0, 3.0, 0, 5), (1, 20.0, 3.0, 5, 10)]


def test_rank_whose_peer_never_joins_fails():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    p = ctx.Process(target=rank_main, args=(0, 2, free_port(), q, 5))  # rank 1 never starts
    p.start()
    r = q.get(timeout=180)
    p.join(timeout=60)
    assert r[0] == 0 and r[1] == "error"
