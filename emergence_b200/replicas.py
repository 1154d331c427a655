"""Independent replicas on several GPUs of one node (one process per GPU).

The compressible step shards by slabs or leaf partitions, but the workloads
measured here fit one GPU, so N GPUs run N independent replicas of the same
workload (weak scaling) with no collective on the data path. torch.distributed
carries only the plumbing: the start barrier and the max over ranks of the
device-timed interval, which makes a whole-job number whose slowest rank sets
the time. Launch with torchrun (RANK, LOCAL_RANK, WORLD_SIZE, MASTER_ADDR,
MASTER_PORT in the environment); NCCL on GPUs, gloo for host-only runs.
"""
import datetime
import os


def init_from_env(backend="nccl", timeout_s=300):
    """(world, rank, local_rank) from the torchrun environment; joins the
    process group when world > 1."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch.distributed as dist
        if not dist.is_initialized():
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(value, world, device="cuda"):
    """The largest of the ranks' values (every rank gets it); `value` itself
    when there is one rank."""
    if world <= 1:
        return float(value)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(units_per_rank, world, max_ms):
    """Units processed by all ranks per second over the slowest rank's time."""
    return units_per_rank * world / (max_ms * 1e-3)


def finish(world):
    if world > 1:
        import torch.distributed as dist
        if dist.is_initialized():
            dist.destroy_process_group()
