"""Independent replicas on several GPUs of one node (one process per GPU).

The time loop shards as independent units (sources, models): every rank
runs its own replica with its own seeded source, no collective touches the
time-stepping data path, and the only collectives there are the barrier
around the timed region and the reductions of the timing (maximum over
ranks) and of the work (sum over ranks).  Training the learned boundary's
network data-parallel is the one exchange step: each rank computes the
gradient of its own shard of face samples and the ranks average them
(allreduce_mean) before every identical optimizer step.  At the end of a run the receiver traces of every replica are
gathered on rank 0 (the reference writes each station's seismograms from the
rank that holds it, src/timeloopMod.f90:591-656; here every rank holds a whole
replica).  The process group uses NCCL on GPUs and gloo on CPUs (tests).
"""
import os
from datetime import timedelta


class Group:
    """rank, world size, local rank and the torch.distributed module (None for one process)."""

    def __init__(self, rank=0, world=1, local=0, dist=None, device="cpu"):
        self.rank, self.world, self.local, self.dist, self.device = rank, world, local, dist, device

    def barrier(self):
        if self.dist is not None:
            self.dist.barrier()

    def _reduce(self, x, op):
        if self.dist is None:
            return float(x)
        import torch
        t = torch.tensor([float(x)], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, op=op)
        return float(t.item())

    def max(self, x):
        return self._reduce(x, None if self.dist is None else self.dist.ReduceOp.MAX)

    def sum(self, x):
        return self._reduce(x, None if self.dist is None else self.dist.ReduceOp.SUM)

    def close(self):
        if self.dist is not None:
            self.dist.destroy_process_group()
            self.dist = None


def init(backend=None, timeout_s=600):
    """Group from the torchrun environment (RANK, WORLD_SIZE, LOCAL_RANK,
    MASTER_ADDR/PORT); one process without it.  backend: "nccl" (default on
    GPUs, one device per local rank) or "gloo"."""
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    if ws <= 1:
        return Group()
    import torch
    import torch.distributed as dist
    rank, local = int(os.environ["RANK"]), int(os.environ.get("LOCAL_RANK", "0"))
    backend = backend or ("nccl" if torch.cuda.is_available() else "gloo")
    if backend == "nccl":
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=timeout_s), device_id=torch.device("cuda", local))
        return Group(rank, ws, local, dist, device="cuda")
    dist.init_process_group("gloo", timeout=timedelta(seconds=timeout_s))
    return Group(rank, ws, local, dist, device="cpu")


def gather_traces(group, traces):
    """Receiver traces of every rank's replica, stacked in rank order on rank
    0: array (world, *traces.shape) there, None on the other ranks.  Every
    rank passes an array of the same shape and dtype (one collective, after
    the time loop; nothing on the data path)."""
    import numpy as np
    arr = np.ascontiguousarray(traces)
    if group.dist is None:
        return arr[None].copy()
    import torch
    t = torch.from_numpy(arr).to(group.device)
    parts = [torch.empty_like(t) for _ in range(group.world)] if group.rank == 0 else None
    group.dist.gather(t, gather_list=parts, dst=0)
    if group.rank != 0:
        return None
    return np.stack([p.cpu().numpy() for p in parts])


def allreduce_mean(group, tensor):
    """In-place mean of a tensor over the ranks (data-parallel gradients of the
    boundary network: NCCL all-reduce on GPUs, gloo on CPUs).  One process:
    unchanged."""
    if group.dist is None or group.world == 1:
        return tensor
    group.dist.all_reduce(tensor, op=group.dist.ReduceOp.SUM)
    tensor /= group.world
    return tensor


def agree_min(group, value):
    """The smallest of an integer over the ranks (so that every rank takes the
    same number of collective steps)."""
    if group.dist is None or group.world == 1:
        return int(value)
    import torch
    t = torch.tensor([int(value)], dtype=torch.int64, device=group.device)
    group.dist.all_reduce(t, op=group.dist.ReduceOp.MIN)
    return int(t.item())


def replica_seed(base, rank):
    """Seed of a rank's replica (its own source)."""
    return base + rank


def aggregate(group, units, seconds):
    """Whole-job throughput: units summed over ranks / the slowest rank's time."""
    return group.sum(units) / group.max(seconds)
