"""Replica bookkeeping for running the audio path on N GPUs of one node, one process per GPU.

Clips are independent and the path has no exchange step, so N > 1 runs N replicas, each on its own
batch (weak scaling): the only collectives are a barrier around each timed region and a MAX
all-reduce of the ranks' times, so the job's time is its slowest rank's.  The same helpers run
with the "nccl" backend on GPUs and with "gloo" on CPU (tests).
"""
import os


def env():
    """(world size, rank, local rank) from the launcher's environment; (1, 0, 0) without one."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend, timeout_s=120):
    """Joins the process group of a multi-rank launch (no-op for one rank)."""
    import datetime
    import torch.distributed as dist
    world, _, _ = env()
    if world > 1 and not dist.is_initialized():
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return world


def barrier():
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.barrier()


def max_over_ranks(value, device="cpu"):
    """The largest of every rank's `value` (every rank gets it)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(units_per_rank, slowest_ms, world):
    """Units per second of the whole job: every rank processed `units_per_rank` and the job took
    the slowest rank's time."""
    return world * float(units_per_rank) / (float(slowest_ms) / 1e3)


def finish():
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        dist.destroy_process_group()
