"""Replica bookkeeping for runs of independent problems on several GPUs.

Each rank (one process per GPU) draws its own problems from a rank-specific
seed and applies them with no exchange between ranks; only scalars cross at
the end: the slowest rank's device time and the total work.  The helpers
take a ``torch.distributed`` module (or ``None`` for one process), so the
same code runs over NCCL on GPUs and over gloo on CPU.
"""

from __future__ import annotations


def rank_seed(seed: int, rank: int) -> int:
    """Seed of rank ``rank``'s problem draw (rank 0 keeps ``seed``)."""
    return int(seed) + 1000 * int(rank)


def _reduce(x: float, dist, device, op_name: str) -> float:
    if dist is None:
        return float(x)
    import torch

    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=getattr(dist.ReduceOp, op_name))
    return float(t.item())


def max_over_ranks(x: float, dist=None, device="cpu") -> float:
    """Largest value over all ranks (device times are reported this way)."""
    return _reduce(x, dist, device, "MAX")


def sum_over_ranks(x: float, dist=None, device="cpu") -> float:
    """Sum over all ranks (work done by the whole job)."""
    return _reduce(x, dist, device, "SUM")


def whole_job_tflops(flops_this_rank: float, ms_this_rank: float, dist=None, device="cpu") -> float:
    """Aggregate throughput: every rank's FLOPs over the slowest rank's time."""
    flops = sum_over_ranks(flops_this_rank, dist, device)
    ms = max_over_ranks(ms_this_rank, dist, device)
    return flops / (ms * 1e-3) / 1e12
