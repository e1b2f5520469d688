"""Replicas on one node: one process per GPU, each running the whole workload
on its own device.  The pipelines have no exchange between GPUs (a query's
tables live on one device; the reference runs one query on one GPU), so
several GPUs run independent replicas: weak scaling, no data-path collective.
The ranks meet on the host (gloo) only to line up the timed region and to take
its maximum over ranks.

Launch: ``torchrun --nproc-per-node N`` (RANK, LOCAL_RANK, WORLD_SIZE and
MASTER_ADDR/MASTER_PORT from the environment; rendezvous on 127.0.0.1).
"""
import datetime
import os


def setup(timeout_s=300):
    """(world, rank, local rank); joins the host process group when world > 1."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch.distributed as dist
        if not dist.is_initialized():
            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=timeout_s))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, world):
    """The largest value of ``x`` over all ranks (every rank gets it)."""
    if world == 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(units_per_rank, ms_max, world):
    """Units of all ranks per second of the slowest rank's time."""
    return units_per_rank * world / (ms_max / 1e3)


def teardown(world):
    if world > 1:
        import torch.distributed as dist
        if dist.is_initialized():
            dist.destroy_process_group()
