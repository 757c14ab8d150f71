"""Replica data parallelism across GPUs (one process per GPU).

The state-vector path at the benchmark sizes fits one GPU, so multi-GPU runs
are replicas: each rank runs its own gradients (or serves its own share of
the requests) with no data-path collective.  The only communication is for
measurement: a barrier around the timed region and the max over ranks of the
device-timed duration, so whole-job throughput = (units over all ranks) /
(slowest rank's time).
"""
import datetime
import os


def init_from_env(backend):
    """torch.distributed from RANK / WORLD_SIZE / MASTER_ADDR / MASTER_PORT;
    returns (rank, world); a single process needs no process group."""
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if world > 1 and not dist.is_initialized():
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return rank, world


def _reduce(value, op, device):
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=op)
    return float(t.item())


def max_over_ranks(value, device="cpu"):
    import torch.distributed as dist
    return _reduce(value, dist.ReduceOp.MAX, device)


def sum_over_ranks(value, device="cpu"):
    import torch.distributed as dist
    return _reduce(value, dist.ReduceOp.SUM, device)


def barrier():
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        dist.barrier()


def shard(items, rank, world):
    """Round-robin share of `items` for `rank` (requests data-parallel across GPUs)."""
    return [x for i, x in enumerate(items) if i % world == rank]


def whole_job_throughput(units_per_rank, ms_local, device="cpu"):
    """(total units / slowest rank's seconds, slowest rank's ms)."""
    ms = max_over_ranks(ms_local, device)
    units = sum_over_ranks(units_per_rank, device)
    return units / (ms * 1e-3), ms
