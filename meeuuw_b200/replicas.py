"""Multi-GPU plumbing: one process per GPU, no data-path collective.

A single model does not shard (a 512x512 model fits one GPU; a domain decomposition would add a
halo exchange per operator apply for no gain), so N GPUs run N independent replicas, and an
ensemble's models are dealt to the GPUs balanced by element count.  The only collectives are the
timing ones: a barrier around the timed region and the maximum of the ranks' times.
"""
import os
from datetime import timedelta

import torch
import torch.distributed as dist


def world():
    """(world size, rank, local rank) from the launcher's environment (1, 0, 0 without one)."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend="nccl", timeout_s=600):
    """Join the process group when there is more than one rank; returns the world size."""
    n, _, _ = world()
    if n > 1 and not dist.is_initialized():
        dist.init_process_group(backend, timeout=timedelta(seconds=timeout_s))
    return n


def barrier(device=None):
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.barrier()
    if device is not None and torch.cuda.is_available():
        torch.cuda.synchronize()


def max_over_ranks(value, device="cpu"):
    """The largest of the ranks' values (timings are reported as the slowest rank's)."""
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value, device="cpu"):
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def throughput(units_per_rank, ms_max, device="cpu"):
    """Whole-job units per second: the units all ranks processed over the slowest rank's time."""
    return sum_over_ranks(units_per_rank, device) / (ms_max / 1000.0)


def partition(sizes, nparts):
    """Deal items (by index) to `nparts` ranks, largest first onto the least-loaded rank (LPT), so
    every rank gets a similar total size; returns one sorted index list per rank."""
    loads = [0] * nparts
    parts = [[] for _ in range(nparts)]
    for i in sorted(range(len(sizes)), key=lambda i: (-sizes[i], i)):
        r = min(range(nparts), key=lambda k: (loads[k], k))
        parts[r].append(i)
        loads[r] += sizes[i]
    return [sorted(p) for p in parts]


def finalize():
    if dist.is_available() and dist.is_initialized():
        dist.barrier()
        dist.destroy_process_group()
