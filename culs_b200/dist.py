"""Multi-GPU plumbing for batched `rw;st`: one process per GPU, graphs
sharded by graph with no data-path collective (independent AIGs need no
exchange); torch.distributed only carries the timing barrier and the
max-over-ranks reduction."""
import os


def rank_world():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), \
        int(os.environ.get("LOCAL_RANK", "0"))


def shard(count, rank, world):
    """Contiguous graph range [lo, hi) of `count` graphs owned by `rank`."""
    base, extra = divmod(count, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


class Group:
    """Barrier and max/sum reductions; a no-op for a single process.  Ranks
    that wait for one another longer than CULS_PG_TIMEOUT_S seconds (default
    600: the autotuner and warm-up steps run between collectives) end with an
    error, as does a rank whose peers never join."""

    def __init__(self, backend=None):
        self.rank, self.world, self.local = rank_world()
        self.dist = None
        if self.world > 1:
            import datetime

            import torch
            import torch.distributed as dist
            if backend is None:
                backend = "nccl" if torch.cuda.is_available() else "gloo"
            if backend == "nccl":
                torch.cuda.set_device(self.local)
            timeout = float(os.environ.get("CULS_PG_TIMEOUT_S", "600"))
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout))
            self.dist = dist
            self.torch = torch
            self.backend = backend

    def _t(self, v):
        t = self.torch.tensor([float(v)], dtype=self.torch.float64)
        return t.cuda() if self.backend == "nccl" else t

    def barrier(self):
        if self.dist:
            self.dist.all_reduce(self._t(0.0))

    def max(self, v):
        if not self.dist:
            return v
        t = self._t(v)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def sum(self, v):
        if not self.dist:
            return v
        t = self._t(v)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM)
        return float(t.item())

    def close(self):
        if self.dist:
            self.dist.destroy_process_group()
            self.dist = None
