"""Independent replicas on several GPUs: the lattice sweep does not shard
(each GPU holds whole lattices; there is no data-path collective), so N
processes run N independent chains -- one per GPU, distinct seeds -- and
only the timing is coordinated: a barrier before and after the timed
region, and the slowest rank's device time for the whole job.

Used by bench.py under torchrun; the functions take the process group
module (torch.distributed) or None for a single process, so the same code
runs with NCCL on GPUs and with gloo on CPU in the tests.
"""
import os
from datetime import timedelta


def dist_env():
    """(rank, world size, local rank) from the torchrun environment"""
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def init(backend, timeout_s=120, device=None):
    """torch.distributed with a short timeout (ranks that wait on a lost
    peer end with an error instead of hanging); None for one process"""
    rank, world, _ = dist_env()
    if world <= 1:
        return None
    import torch.distributed as dist
    kw = {"timeout": timedelta(seconds=timeout_s)}
    if device is not None:
        kw["device_id"] = device
    dist.init_process_group(backend, **kw)
    return dist


def replica_seed(rank, base=54):
    """RANDSERIES of rank r's chain: distinct per rank, rank 0 = base"""
    return base + rank


def barrier(dist):
    if dist is not None:
        dist.barrier()


def max_over_ranks(x, dist, device="cpu"):
    """the largest x over all ranks (the job's time is the slowest rank's)"""
    if dist is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(world, units_per_rank, seconds):
    """units per second of all ranks together, timed by the slowest rank"""
    return world * units_per_rank / seconds


def reference_arm_runs_here(rank):
    """the reference's CPU path is timed once per job, on rank 0"""
    return rank == 0


def finish(dist):
    if dist is not None:
        dist.destroy_process_group()
