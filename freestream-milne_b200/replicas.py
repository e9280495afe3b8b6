"""Replica coordination for runs on several GPUs of one node.

Events are independent, so each rank (one process per GPU, launched by
torch.distributed.run) works on its own events with no data exchange; the
only collectives are the timing reductions: a barrier around the timed
region, the maximum of the ranks' times and sums of counts.  The backend is
NCCL on GPUs; the tests use gloo on the CPU.
"""
import datetime
import os


class Replicas:
    def __init__(self, backend="nccl", timeout_s=120):
        self.rank = int(os.environ.get("RANK", "0"))
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.backend = backend
        self.dist = None
        if self.world > 1:
            import torch
            import torch.distributed as dist
            kw = {}
            if backend == "nccl":
                kw["device_id"] = torch.device("cuda", self.local)
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s), **kw)
            self.dist = dist

    def seed(self, base):
        """A distinct event set per replica (weak scaling)."""
        return base + 1000 * self.rank

    def barrier(self):
        if self.dist is not None:
            self.dist.barrier()

    def _reduce(self, x, op):
        if self.dist is None:
            return float(x)
        import torch
        dev = "cuda" if self.backend == "nccl" else "cpu"
        t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
        self.dist.all_reduce(t, op=op)
        return float(t.item())

    def max(self, x):
        return self._reduce(x, None if self.dist is None else self.dist.ReduceOp.MAX)

    def sum(self, x):
        return self._reduce(x, None if self.dist is None else self.dist.ReduceOp.SUM)

    def rate(self, units_local, seconds_local):
        """Whole-job throughput: all ranks' units over the slowest rank's time."""
        return self.sum(units_local) / self.max(seconds_local)

    def close(self):
        if self.dist is not None:
            self.dist.barrier()
            self.dist.destroy_process_group()
            self.dist = None
