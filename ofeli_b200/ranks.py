"""One process per GPU: the rank plumbing of bench.py's workloads.

Each process reads RANK / WORLD_SIZE / LOCAL_RANK from the environment (as
torchrun sets them); with more than one rank it joins a process group
(NCCL on the GPUs, gloo on the CPU for tests) with a short timeout, so that
ranks waiting for one another end with an error instead of hanging.  Times
are combined as the maximum over ranks.  The workloads shard no data path:
each rank either runs a replica or its own share of independent problems
(`problems.partition_by_cost`).
"""
import datetime
import os


def env():
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


class Ranks:
    def __init__(self, backend, device, timeout_s=300):
        self.world, self.rank, self.local = env()
        self.device = device
        self.dist = None
        if self.world > 1:
            import torch.distributed as dist
            kwargs = {"device_id": device} if backend == "nccl" else {}
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s),
                                    **kwargs)
            self.dist = dist

    def barrier(self):
        if self.dist:
            self.dist.barrier()

    def max(self, v):
        """The maximum of a float over ranks (every rank gets it)."""
        if not self.dist:
            return float(v)
        import torch
        t = torch.tensor([float(v)], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def gather(self, obj):
        """Every rank's object, in rank order, on every rank."""
        if not self.dist:
            return [obj]
        out = [None] * self.world
        self.dist.all_gather_object(out, obj)
        return out

    def close(self):
        if self.dist:
            self.dist.destroy_process_group()
            self.dist = None
