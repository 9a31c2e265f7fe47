"""One process per GPU, each an independent replica of the product pipeline.

The multiply does not shard: a product is one transform on one device, and
the independent products of a batch or a tree level are already spread over
the SMs of that device.  So N GPUs run N replicas of the same workload with
no collective on the data path.  The only cross-rank steps are the ones the
measurement needs: a barrier around the timed region and the maximum of the
per-rank times (whole-job throughput = units of all ranks / slowest rank).

Ranks come from the launcher's environment (RANK, WORLD_SIZE, LOCAL_RANK,
MASTER_ADDR, MASTER_PORT, as torch.distributed.run sets them).  With one
rank nothing is initialised.  The process group uses NCCL when CUDA is
available and gloo otherwise (the CPU tests run two gloo ranks), always with
a short timeout so a rank that never arrives ends the others with an error.
"""
import os
from datetime import timedelta


class Replicas:
    """rank / world / local of this process and the measurement collectives."""

    def __init__(self, backend=None, timeout_s=120):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.dist = None
        self.device = "cpu"
        if self.world > 1:
            import torch
            import torch.distributed as dist
            if backend is None:
                backend = "nccl" if torch.cuda.is_available() else "gloo"
            if backend == "nccl":
                torch.cuda.set_device(self.local)
                self.device = "cuda"
            dist.init_process_group(backend, timeout=timedelta(seconds=timeout_s))
            self.dist = dist

    def barrier(self):
        if self.dist:
            self.dist.barrier()
        if self.device == "cuda":
            import torch
            torch.cuda.synchronize()

    def max(self, x):
        """The largest x over all ranks (every rank gets it)."""
        if not self.dist:
            return float(x)
        import torch
        t = torch.tensor([float(x)], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.dist:
            self.dist.barrier()
            self.dist.destroy_process_group()
            self.dist = None


def job_throughput(units_per_rank, ms_slowest, world):
    """Whole-job rate: every rank processed units_per_rank in at most
    ms_slowest milliseconds (weak scaling: per-rank work fixed)."""
    return units_per_rank * world / (ms_slowest * 1e-3)
