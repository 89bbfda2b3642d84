"""Multi-GPU runs of independent H_eff problems: one process per GPU.

Two ways to spread a batch of independent problems over ranks, neither with
any exchange on the data path:
  * ``partition``: one batch is split by a greedy FLOP-balanced assignment
    (longest processing time first), each problem on exactly one rank; the
    job's work is fixed as ranks are added (strong scaling).  Results can be
    collected on rank 0 afterwards (``gather_to_root``).
  * replicas: each rank draws its own batch from a rank-specific seed
    (``rank_seed``), so per-rank work is fixed (weak scaling).
Only scalars cross during a timed run: the slowest rank's device time and
the total work.  The helpers take a ``torch.distributed`` module (or
``None`` for one process), so the same code runs over NCCL on GPUs and over
gloo on CPU.
"""

from __future__ import annotations


def partition(flops, world: int) -> list:
    """Greedy FLOP-balanced assignment of problems to ``world`` ranks.

    Problems are taken in decreasing FLOP order (ties: lower index first),
    each given to the rank with the least work so far (ties: lower rank).
    Returns, per rank, the sorted indices of its problems.  Every problem is
    assigned exactly once; with n >= world problems no rank is left empty."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(flops)), key=lambda i: (-float(flops[i]), i))
    load = [0.0] * world
    share: list = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        share[r].append(i)
        load[r] += float(flops[i])
    return [sorted(s) for s in share]


def gather_to_root(local: dict, dist=None) -> dict | None:
    """Collect every rank's ``{problem index: result}`` on rank 0 (host
    objects; after the timed region).  Returns the merged dict on rank 0 and
    None elsewhere; a problem reported by two ranks raises."""
    if dist is None:
        return dict(local)
    parts = [None] * dist.get_world_size() if dist.get_rank() == 0 else None
    dist.gather_object(local, parts, dst=0)
    if dist.get_rank() != 0:
        return None
    merged: dict = {}
    for part in parts:
        for k, v in part.items():
            if k in merged:
                raise RuntimeError(f"problem {k} was applied on two ranks")
            merged[k] = v
    return merged


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
