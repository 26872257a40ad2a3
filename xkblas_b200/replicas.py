"""Multi-GPU plumbing of the benchmark: one process per GPU (launched by
torchrun), each running an independent problem -- the level-3 tile path has
no exchange step on one node's replicas, so there is no data collective.
The only communication is timing: a barrier before and after the timed
region and the maximum of the per-rank times (the job finishes when the
slowest rank does).  `value` = all ranks' units / that maximum.

Backends: "nccl" on GPUs (the benchmark), "gloo" on CPU (tests).  Every rank
takes the same collective steps in the same order, in the timed path and
the error path alike."""
import datetime
import os


class Replicas:
    def __init__(self, backend="nccl", timeout_s=300):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.backend = backend
        self.dist = None
        if self.world > 1:
            import torch.distributed as dist
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
            self.dist = dist

    @property
    def leader(self):
        return self.rank == 0

    def _device(self):
        return "cuda:%d" % self.local if self.backend == "nccl" else "cpu"

    def barrier(self, sync=None):
        """Device sync (if given), then a barrier over all ranks."""
        if sync is not None:
            sync()
        if self.dist is not None:
            self.dist.barrier()

    def max(self, v):
        """The maximum of v over all ranks (v itself with one rank)."""
        if self.dist is None:
            return float(v)
        import torch
        t = torch.tensor([float(v)], dtype=torch.float64, device=self._device())
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def aggregate(self, units_per_rank, seconds_per_rank):
        """Whole-job throughput: every rank's units over the slowest rank's
        time (collective: call on every rank)."""
        slowest = self.max(seconds_per_rank)
        return self.world * units_per_rank / slowest, slowest

    def close(self):
        if self.dist is not None:
            self.dist.barrier()
            self.dist.destroy_process_group()
            self.dist = None
