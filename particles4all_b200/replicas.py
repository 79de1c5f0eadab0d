"""Replicas: one process per GPU, each stepping its own scenes.

Independent scenes are the unit that shards: nothing crosses GPUs on the data
path, so the only collectives are the ones timing needs (a barrier on both sides
of the timed region, and the maximum of the per-rank device times). Ranks read
RANK / LOCAL_RANK / WORLD_SIZE / MASTER_ADDR / MASTER_PORT from the environment
as torchrun sets them; with WORLD_SIZE = 1 no process group is created.
"""
import datetime
import os


def env():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)),
            int(os.environ.get("WORLD_SIZE", 1)))


class Replicas:
    def __init__(self, backend="nccl", timeout_s=120):
        self.rank, self.local_rank, self.world = env()
        self.backend = backend
        self._dist = None
        if self.world > 1:
            import torch
            import torch.distributed as dist
            kw = {}
            if backend == "nccl":
                kw["device_id"] = torch.device("cuda", self.local_rank)
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s), **kw)
            self._dist = dist

    def _tensor(self, x):
        import torch
        dev = "cuda" if self.backend == "nccl" else "cpu"
        return torch.tensor([float(x)], dtype=torch.float64, device=dev)

    def barrier(self):
        if self._dist:
            self._dist.barrier()

    def max(self, x):
        """Maximum of x over the ranks (every rank gets it)."""
        if not self._dist:
            return float(x)
        t = self._tensor(x)
        self._dist.all_reduce(t, op=self._dist.ReduceOp.MAX)
        return float(t.item())

    def sum(self, x):
        if not self._dist:
            return float(x)
        t = self._tensor(x)
        self._dist.all_reduce(t, op=self._dist.ReduceOp.SUM)
        return float(t.item())

    def close(self):
        if self._dist:
            self._dist.barrier()
            self._dist.destroy_process_group()
            self._dist = None
