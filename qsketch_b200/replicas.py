"""Multi-GPU plumbing for the insert/query path: one independent sketch per rank.

The path has no data exchange (every rank owns a sketch and its own key stream), so N GPUs
run N replicas with no collective on the data path; the only collectives are the barrier
around the timed region and the max-over-ranks of the measured times.  One process per GPU,
launched by torchrun (RANK / LOCAL_RANK / WORLD_SIZE / MASTER_* from the environment), NCCL
on GPUs and gloo on CPU (the multi-process tests).
"""
import datetime
import os

import torch
import torch.distributed as dist


class Ranks:
    def __init__(self, backend=None, timeout_s=120):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.backend = backend or ("nccl" if torch.cuda.is_available() else "gloo")
        self.device = torch.device("cuda", self.local) if self.backend == "nccl" else torch.device("cpu")
        if self.backend == "nccl":
            torch.cuda.set_device(self.local)
        self._own = False
        if self.world > 1 and not dist.is_initialized():
            os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
            kw = {"device_id": self.device} if self.backend == "nccl" else {}
            dist.init_process_group(self.backend, timeout=datetime.timedelta(seconds=timeout_s), **kw)
            self._own = True

    def barrier(self):
        if self.world > 1:
            dist.barrier()

    def _reduce(self, x, op):
        if self.world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=self.device)
        dist.all_reduce(t, op=op)
        return float(t.item())

    def max(self, x):
        """The largest value over ranks (times: the job takes as long as its slowest rank)."""
        return self._reduce(x, dist.ReduceOp.MAX)

    def sum(self, x):
        return self._reduce(x, dist.ReduceOp.SUM)

    def gather(self, x):
        """All ranks' values of a float, in rank order."""
        if self.world == 1:
            return [float(x)]
        t = torch.tensor([x], dtype=torch.float64, device=self.device)
        out = [torch.zeros_like(t) for _ in range(self.world)]
        dist.all_gather(out, t)
        return [float(o.item()) for o in out]

    def stream_seed(self, base):
        """Each rank's key stream has its own seed: replicas insert different data."""
        return base + self.rank

    def close(self):
        if self._own and dist.is_initialized():
            dist.destroy_process_group()
            self._own = False


def aggregate_rate(units_per_rank, world, max_ms):
    """Whole-job throughput in G units/s: every rank processed units_per_rank units and the
    job took the slowest rank's time (weak scaling)."""
    return world * units_per_rank / (max_ms * 1e6)
