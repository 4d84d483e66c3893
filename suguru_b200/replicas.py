"""Replicas on several GPUs of one node.

The coupling step has no exchange between GPUs on this path: every rank runs
the whole workload on its own GPU, one process per GPU (torch.distributed,
NCCL on GPUs, gloo on CPU).  The whole job's rate is the units all ranks
processed over the slowest rank's time, the time reduced with a maximum over
ranks.
"""
import torch
import torch.distributed as dist


def world():
    return dist.get_world_size() if dist.is_available() and dist.is_initialized() else 1


def max_over_ranks(x):
    """The largest x over the ranks (x itself on one rank).  Every rank must call it, in the same order."""
    if world() == 1:
        return float(x)
    dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend() == "nccl" else torch.device("cpu")
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(units_per_rank, seconds_max, nranks=None):
    """Units per second of the whole job: nranks replicas of units_per_rank each over the slowest rank's time."""
    n = world() if nranks is None else nranks
    return n * units_per_rank / seconds_max
