"""Replica runs: one process per GPU, each decoding its own copy of the
workload (chunks are independent; the path has no exchange step, so there is
no data-path collective). The only collectives are the timing ones: a barrier
around the timed region and the maximum of the ranks' times, over whatever
process group is current (NCCL on GPUs, gloo in the CPU tests)."""
import os
from datetime import timedelta


def rank_env():
    """(rank, world, local_rank) from the launcher's environment."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend, device=None, timeout_s=120):
    """Join the process group when world > 1 (rendezvous from MASTER_ADDR /
    MASTER_PORT); a short timeout turns a missing rank into an error."""
    import torch.distributed as dist
    _, world, _ = rank_env()
    if world > 1 and not dist.is_initialized():
        kw = {"device_id": device} if device is not None and backend == "nccl" else {}
        dist.init_process_group(backend, timeout=timedelta(seconds=timeout_s), **kw)
    return world


def max_over_ranks(x, device="cpu"):
    """The largest of the ranks' values (a float), or x alone."""
    import torch
    import torch.distributed as dist
    if not dist.is_initialized() or dist.get_world_size() == 1:
        return x
    t = torch.tensor([float(x)], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_rate(units_per_rank, seconds, world):
    """Whole-job throughput: every rank's units over the slowest rank's time."""
    return world * units_per_rank / seconds


def finish():
    import torch.distributed as dist
    if dist.is_initialized():
        dist.destroy_process_group()
