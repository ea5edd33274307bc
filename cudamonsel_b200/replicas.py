"""Replicas across GPUs: one process per GPU, each transporting its own pixels.

Pixels are independent (each pixel's result depends only on its random-stream key, its beam and its
primary count), so N GPUs run N replicas of a scan with disjoint keys and no collective on the data path.
The only cross-rank step is timing: a job's time is the slowest rank's, taken with a MAX all-reduce of the
device-timed milliseconds (NCCL on GPUs, gloo in the CPU tests).
"""
import numpy as np

KEY_STRIDE = 1_000_003


def pixel_keys(rank, npix, stride=KEY_STRIDE):
    """Stream keys of one rank's pixels, disjoint across ranks: rank r takes [stride (r + 1), + npix)."""
    if npix > stride:
        raise ValueError("npix %d exceeds the key stride %d" % (npix, stride))
    return np.arange(npix, dtype=np.uint64) + np.uint64(stride * (rank + 1))


def max_over_ranks(value, device=None):
    """The largest of every rank's value (all ranks must call it; a single process returns its own)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(units_per_rank, world, ms_max):
    """Whole-job throughput (units/s) of `world` replicas that each did units_per_rank in at most ms_max."""
    return world * units_per_rank / (ms_max / 1000.0)
