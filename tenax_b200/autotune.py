"""Schedule autotuner for batched H_eff applications, keyed on the sector-size
histogram.

The reference evaluates H_eff one block combination at a time and has no
schedule to tune.  Here the mixed-precision stages 1-3 can run as one fused
tcgen05 kernel (tile c extent ``c_per_tile``), as a stage-1 GEMM whose
epilogue routes the single-term W_l W_r outputs straight into the stage-4
operand (routed), or as three kernels with X1 in HBM, and which is faster
depends on the sector sizes and the MPO: the fused kernel's MMA rows are one
d sector padded to 128, its columns ``c_per_tile`` c values per MPO input
block; the routed epilogue writes each X1 row once per single-term output
that reads it.  The tuner times each candidate schedule on the actual
problems, keeps the fastest, and caches it under a key made of the device
name, the precision, a histogram of the bond sector sizes (power-of-two
buckets) with the MPO bond dimension, and a hash of the kernel library, so
later batches with the same sector profile on the same build skip the timing.
"""

from __future__ import annotations

import json
import os
from collections import Counter

import numpy as np
import torch

from tenax_b200.heff import HeffBatch, HeffOperator

DEFAULT_CACHE = os.path.join(os.path.expanduser("~"), ".cache", "tenax_b200", "heff_schedules.json")


def sector_histogram(problems) -> tuple:
    """Power-of-two histogram of the bond sector sizes of every problem's
    theta (first and last legs), with the MPO bond dimensions: the key of a
    tuned schedule."""
    hist = Counter()
    dws = set()
    for p in problems:
        idx = p.theta.indices
        for leg in (idx[0], idx[-1]):
            _, counts = np.unique(leg.charges, return_counts=True)
            for c in counts:
                hist[int(np.ceil(np.log2(max(int(c), 1))))] += 1
        dws.add(len(p.Wl.indices[0].charges))
    return tuple(sorted(hist.items())), tuple(sorted(dws))


# the schedules a tuned entry chose among: entries tuned over another set are re-tuned
SCHEDULE_SET = ("fused", "routed", "auto", "unfused")


def schedule_label(s: dict) -> str:
    return {1: f"fused c={s['c_per_tile']}", 2: "routed", -1: "auto (routed from 5e9 FLOPs)"}.get(s["fuse_mpo"],
                                                                                                "unfused")


_LIBRARY_ID = None


def library_id() -> str:
    """Content hash of the loaded CUDA library: schedules tuned on another
    build of the kernels are timed again."""
    global _LIBRARY_ID
    if _LIBRARY_ID is None:
        import hashlib

        from tenax_b200 import _capi

        with open(_capi.LIB._name, "rb") as f:
            _LIBRARY_ID = hashlib.sha256(f.read()).hexdigest()[:16]
    return _LIBRARY_ID


def cache_key(problems, precision: str) -> str:
    name = torch.cuda.get_device_name() if torch.cuda.is_available() else "cpu"
    hist, dws = sector_histogram(problems)
    return json.dumps({"device": name, "precision": precision, "dw": dws, "sectors": hist,
                       "schedules": list(SCHEDULE_SET), "library": library_id()}, sort_keys=True)


def candidates(problems, precision: str) -> list:
    """The fused kernel at the largest c extent that fits, at half of it and
    at 1, the routed stage-1 epilogue, routed or unfused per operator by its
    size (-1), and the three-kernel path."""
    p = problems[0]
    probe = HeffOperator(p.L, p.Wl, p.Wr, p.R, p.theta.indices, p.theta.keys, precision,
                         schedule={"fuse_mpo": 1, "c_per_tile": 0})
    cc = probe.schedule["c_per_tile"] if probe.schedule["fuse_mpo"] else 0
    out = []
    if cc:
        for c in sorted({cc, max(1, cc // 2), 1}, reverse=True):
            out.append({"fuse_mpo": 1, "c_per_tile": c})
    out.append({"fuse_mpo": 2, "c_per_tile": 0})
    out.append({"fuse_mpo": -1, "c_per_tile": 0})
    out.append({"fuse_mpo": 0, "c_per_tile": 0})
    return out


def time_schedule(problems, precision: str, schedule: dict, reps: int = 5, warmup: int = 2) -> float:
    """Milliseconds per batched apply of ``problems`` under ``schedule``
    (CUDA events on the current stream, after ``warmup`` applies)."""
    from tenax_b200.tensor import embed_in_keys

    ops = [HeffOperator(p.L, p.Wl, p.Wr, p.R, p.theta.indices, p.theta.keys, precision, schedule=schedule)
           for p in problems]
    if len({o.schedule["fuse_mpo"] for o in ops}) != 1 and schedule["fuse_mpo"] != -1:
        return float("inf")  # the structure does not take this schedule everywhere
    xs = [embed_in_keys(p.theta, o.keys).data for p, o in zip(problems, ops)]
    ys = [o.out_like() for o in ops]
    batch = HeffBatch(ops)
    for _ in range(warmup):
        batch.apply(xs, ys)
    st = torch.cuda.current_stream()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(st)
    for _ in range(reps):
        batch.apply(xs, ys)
    b.record(st)
    torch.cuda.synchronize()
    if batch.device_error():
        return float("inf")
    return a.elapsed_time(b) / reps


def tune(problems, precision: str, cache_path: str | None = DEFAULT_CACHE, reps: int = 5,
         force: bool = False) -> tuple:
    """(best schedule, {candidate label: ms}) for a batch of problems; the
    timings dict is empty when the schedule came from the cache."""
    key = cache_key(problems, precision)
    cache = {}
    if cache_path and os.path.exists(cache_path):
        try:
            cache = json.load(open(cache_path))
        except (OSError, ValueError):
            cache = {}
    if not force and key in cache:
        return cache[key], {}
    timings = {}
    best, best_ms = None, float("inf")
    for s in candidates(problems, precision):
        ms = time_schedule(problems, precision, s, reps=reps)
        label = schedule_label(s)
        timings[label] = round(ms, 4)
        if ms < best_ms:
            best, best_ms = s, ms
        torch.cuda.empty_cache()
    if cache_path and best is not None:
        cache[key] = best
        os.makedirs(os.path.dirname(cache_path), exist_ok=True)
        tmp = cache_path + ".tmp"
        with open(tmp, "w") as fh:
            json.dump(cache, fh, indent=1, sort_keys=True)
        os.replace(tmp, cache_path)
    return best, timings
