"""Multi-GPU plumbing of the trace: one process per GPU, rays sharded, one exchange at the end.

Rays are independent (every ray owns its random stream), so a multi-GPU run is N
independent runs: rank r traces its own rays (weak scaling: the same number of
first-stage hits per rank, seed `rank_seed(seed, r)`), and the only collective comes
after the timed work -- counters and integer flux maps summed (exact, order free),
device times reduced with max (the job takes as long as its slowest rank).  The
reference does the same across host threads: independent contexts with seeds
seed + i*123, results concatenated (app/src/trace.cpp:709-735, pysoltrace.py:1615-1661).

The functions work with any torch.distributed backend: "nccl" with CUDA tensors on the
GPU box, "gloo" with CPU tensors in the tests.  Without an initialised process group
they return their inputs (one rank).
"""
from __future__ import annotations

import numpy as np


def rank_seed(seed: int, rank: int) -> int:
    """Seed of rank `rank`'s rays (distinct streams on every rank)."""
    return int(seed) + 1000 * int(rank)


def _dist():
    try:
        import torch.distributed as dist
    except ImportError:  # pragma: no cover - torch is part of the image
        return None
    return dist if dist.is_available() and dist.is_initialized() else None


def combine(units: float, dev_ms: float, wall_ms: float, flux: np.ndarray, device: str = "cpu"):
    """Whole-job totals of one rank's results.

    Returns (units summed over ranks, device time max over ranks, wall time max over
    ranks, flux map summed over ranks).  `device` is where the collective's tensors live
    ("cuda" for NCCL, "cpu" for gloo).
    """
    dist = _dist()
    flux = np.asarray(flux, dtype=np.int64)
    if dist is None or dist.get_world_size() == 1:
        return float(units), float(dev_ms), float(wall_ms), flux.copy()
    import torch

    s = torch.tensor([float(units)], dtype=torch.float64, device=device)
    m = torch.tensor([float(dev_ms), float(wall_ms)], dtype=torch.float64, device=device)
    f = torch.from_numpy(flux.copy()).to(device)
    dist.all_reduce(s, op=dist.ReduceOp.SUM)
    dist.all_reduce(m, op=dist.ReduceOp.MAX)
    dist.all_reduce(f, op=dist.ReduceOp.SUM)
    return s[0].item(), m[0].item(), m[1].item(), f.cpu().numpy()
