"""Independent network replicas, one process per GPU (the multi-GPU mode of
this library: the step itself does not shard).  Helpers for the launcher's
environment (RANK, LOCAL_RANK, WORLD_SIZE, MASTER_ADDR/PORT), timing as the
maximum over ranks, and whole-job throughput."""
import datetime
import os


def init(backend="nccl", timeout_s=300):
    """(dist or None, rank, world, local rank); dist is torch.distributed,
    initialised from the environment when WORLD_SIZE > 1."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world <= 1:
        return None, rank, world, local
    import torch.distributed as dist
    dist.init_process_group(backend, init_method="env://", timeout=datetime.timedelta(seconds=timeout_s))
    return dist, rank, world, local


def max_over_ranks(dist, values, device="cpu"):
    """Element-wise maximum of a list of floats over all ranks (identity on
    one process)."""
    if dist is None:
        return [float(v) for v in values]
    import torch
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t.cpu().tolist()]


def throughput(world, units_per_rank, ms):
    """Whole-job rate: every rank processed units_per_rank in at most ms."""
    return world * units_per_rank / (ms / 1000.0)


def replica_seed(base, rank):
    """Seed of rank's replica (different wiring and input per rank)."""
    return base + rank


def finish(dist):
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
