"""Replica runs of the batched search: one process per GPU, each searching
its own copy of the query batch against its own copy of the index (the
search path has no exchange step, so there is no collective on the data
path).  The only collective is the timing: the job's time is the slowest
rank's, and the whole-job throughput counts every rank's queries."""
import datetime
import os


def init(backend="nccl", timeout_s=600):
    """Joins the process group torchrun describes (RANK, WORLD_SIZE,
    MASTER_ADDR/PORT in the environment)."""
    import torch.distributed as dist
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return dist.get_rank(), dist.get_world_size()


def job_throughput(local_ms, queries_per_rank, device=None):
    """(whole-job queries per second, slowest rank's ms) from this rank's
    timed milliseconds; every rank must call it (one MAX all-reduce)."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size() if dist.is_initialized() else 1
    t = torch.tensor([float(local_ms)], dtype=torch.float64, device=device)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    slowest = float(t.item())
    return queries_per_rank * world / (slowest / 1e3), slowest


def barrier():
    import torch.distributed as dist
    if dist.is_initialized() and dist.get_world_size() > 1:
        dist.barrier()


def finish():
    import torch.distributed as dist
    if dist.is_initialized():
        dist.destroy_process_group()
