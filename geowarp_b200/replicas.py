"""Multi-GPU execution: independent replicas, one process per GPU.

A load step does not shard at these sizes (a domain split would need nodal
halos, a distributed Krylov solve and a global Newton norm), so N GPUs run N
independent problem instances: the batched workload deals its blocks to the
ranks, the single footing runs one copy per rank.  There is no collective on
the data path; the only collectives are the barriers that bracket a timed
region and one max-reduction of the per-rank timings, so the reported time is
that of the slowest rank.  The same code runs on NCCL (GPUs) and gloo (CPU
tests).
"""
import datetime
import os

import torch
import torch.distributed as dist


class Replicas:
    """Rank / world bookkeeping from the torchrun environment."""

    def __init__(self, backend="nccl", timeout_s=600):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.backend = backend
        self.active = self.world > 1
        if self.active:
            if backend == "nccl":
                torch.cuda.set_device(self.local)
            dist.init_process_group(backend, init_method="env://", timeout=datetime.timedelta(seconds=timeout_s))

    def barrier(self):
        if self.active:
            dist.barrier()

    def max_over_ranks(self, values, device=None):
        """Element-wise maximum of per-rank float values (every rank gets it)."""
        t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
        if self.active:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return t.tolist()

    def share(self, items):
        """This rank's items of a list dealt round-robin over the ranks."""
        return items[self.rank::self.world]

    def close(self):
        if self.active:
            dist.barrier()
            dist.destroy_process_group()
            self.active = False


def aggregate_rate(units_per_rank, ms_max):
    """Whole-job throughput: all ranks' units over the slowest rank's time."""
    return sum(units_per_rank) / (ms_max / 1e3)
