#!/usr/bin/env python
"""Benchmark: batched U(1) two-site H_eff matvec on B200 (FP64 drop-in vs mixed).

Workload (one step): 64 independent two-site H_eff matvecs
``abc,apqd,bpse,eqtf,dfg->cstg`` for the width-6 Heisenberg cylinder (U(1)
MPO, bond dim 26), chi drawn uniformly from {256, 512, 1024, 2048}, 30 U(1)
sectors per bond with Gaussian sizes (sigma=3, clipped to 4..256), all
problems in one launch per stage.  Synthetic seeded data; operator images
are packed once (per-site setup), theta is packed every step.

    python bench.py [--gpus N --steps K --warmup W --precision bf16x3]
    python bench.py --impl reference      # CPU baseline arm (oracle port)

Prints one JSON line on rank 0.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count()))
os.environ.setdefault("OPENBLAS_NUM_THREADS", str(os.cpu_count()))

import numpy as np  # noqa: E402

ROOT = os.path.dirname(os.path.abspath(__file__))
METRIC = "U(1) H_eff matvec TFLOP/s & DMRG sweep s at χ=2048: mixed vs FP64, |ΔE|≤1e-9"
WORKLOAD = ("batched grouped-sector contraction: 64 independent two-site H_eff matvecs, width-6 Heisenberg "
            "cylinder U(1) MPO (Dw=26), chi~U{256,512,1024,2048}, 30 U(1) sectors/bond, Gaussian sizes "
            "sigma=3 clipped 4..256, one launch per stage")
CHIS = (256, 512, 1024, 2048)
N_PROBLEMS = 64


def _peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d, "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


def _dram_view(traffic, stage_ms, peaks, peak_src):
    """The same kernel against the HBM roofline: its measured DRAM bytes per
    launch (``traffic``, from the committed ncu capture) over its CUDA-event
    stage time.  A routed stage 1 also writes the stage-4 image, so both
    bounds apply to it."""
    if not traffic or not peaks.get("hbm_gbs"):
        return None
    gbs = traffic / (stage_ms * 1e-3) / 1e9
    return {"achieved": round(gbs, 1), "peak": round(float(peaks["hbm_gbs"]), 1), "unit": "GB/s",
            "frac": round(gbs / float(peaks["hbm_gbs"]), 4), "peak_source": f"{peak_src} HBM copy",
            "basis": "measured DRAM bytes per launch / stage time"}


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled every 100 ms.

    Started before the warm-up (nvidia-smi takes a few hundred ms to print its
    first line); ``mark_start``/``mark_end`` bracket the timed region on the
    host clock and ``summary`` keeps only the samples read inside it."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.lines: list = []  # (host monotonic time read, line)
        self.ready = threading.Event()
        self.window = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "100",
                 "-i", str(self.dev)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            self.ready.wait(timeout=10.0)
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.monotonic(), line.strip()))
            self.ready.set()

    def mark_start(self):
        self.window = [time.monotonic(), None]

    def mark_end(self):
        if self.window is not None:
            self.window[1] = time.monotonic()

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        lo, hi = (self.window if self.window and self.window[1] is not None else (-1e300, 1e300))
        for t, ln in self.lines:
            if not lo <= t <= hi:
                continue
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = max(mx, float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


def run_ours(args):
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    from tenax_b200 import HeffBatch, HeffOperator, _capi
    from tenax_b200 import replicas
    from tenax_b200.tensor import embed_in_keys
    from tenax_b200.workloads import batched_problems

    dev = torch.device("cuda", local)
    if args.mode == "replicas":
        # weak scaling: every rank its own batch from a rank-specific seed
        problems = batched_problems(args.problems, CHIS, seed=replicas.rank_seed(args.seed, rank))
        share_note = f"replicas x{world} (each rank its own {args.problems}-problem batch)"
        batch_chi_counts = None
    else:
        # strong scaling: one batch split by a greedy FLOP-balanced assignment;
        # every rank builds the same batch and keeps its share
        from tenax_b200.heff import problem_flops

        problems = batched_problems(args.problems, CHIS, seed=args.seed)
        batch_chi_counts = {int(c): sum(1 for p in problems if p.chi == c) for c in CHIS}
        per_chi = {}
        for p in problems:
            if p.chi not in per_chi:
                per_chi[p.chi] = problem_flops(p)
        share = replicas.partition([per_chi[p.chi] for p in problems], world)[rank]
        problems = [problems[i] for i in share]
        torch.cuda.empty_cache()
        share_note = partition_note(world, args.problems, len(problems))
    chi_counts = {int(c): sum(1 for p in problems if p.chi == c) for c in CHIS}
    if batch_chi_counts is None:
        batch_chi_counts = chi_counts

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x: float) -> float:
        return replicas.max_over_ranks(x, dist, dev)

    def run_precision(prec, with_e2e=False, sampler=None, schedule=None):
        ops = [HeffOperator(p.L, p.Wl, p.Wr, p.R, p.theta.indices, p.theta.keys, prec, schedule=schedule)
               for p in problems]
        sizes = [o.size for o in ops]
        offs = np.concatenate([[0], np.cumsum(sizes)])
        x_all = torch.empty(int(offs[-1]), dtype=torch.float64, device=dev)
        y_all = torch.empty(int(offs[-1]), dtype=torch.float64, device=dev)
        for i, (p, o) in enumerate(zip(problems, ops)):
            x_all[offs[i]:offs[i + 1]].copy_(embed_in_keys(p.theta, o.keys).data)
        xs = [x_all[offs[i]:offs[i + 1]] for i in range(len(ops))]
        ys = [y_all[offs[i]:offs[i + 1]] for i in range(len(ops))]
        batch = HeffBatch(ops)
        flops = batch.flops
        st = torch.cuda.current_stream()
        if sampler:
            sampler.__enter__()
        # one step = one batched apply, replayed from a captured CUDA graph
        # (every stage of every problem in one graph launch) unless --no-graph
        graph = batch.capture(xs, ys) if not args.no_graph else None
        step = graph.replay if graph is not None else (lambda: batch.apply(xs, ys))
        for _ in range(args.warmup):
            step()
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        if sampler:
            sampler.mark_start()
        e0.record(st)
        for _ in range(args.steps):
            step()
        e1.record(st)
        barrier()
        if sampler:
            sampler.mark_end()
            sampler.__exit__()
        ms = max_over_ranks(e0.elapsed_time(e1) / args.steps)
        del graph
        err = batch.device_error()
        # per-stage timing (each stage re-run alone, same buffers)
        stage_ms = []
        for s in range(4):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(st)
            for _ in range(args.steps):
                _capi.check(_capi.LIB.tnx_heff_batch_apply_stage(batch.handle, s, st.cuda_stream))
            b.record(st)
            torch.cuda.synchronize()
            stage_ms.append(a.elapsed_time(b) / args.steps)
        import ctypes as C

        sf = np.zeros(3)
        tot_sf = np.zeros(3)
        for o in ops:
            _capi.check(_capi.LIB.tnx_heff_stage_flops(o.handle, sf.ctypes.data))
            tot_sf += sf
        res = {"ms": ms, "flops": flops, "stage_ms": stage_ms, "stage_flops": tot_sf.tolist(), "err": err,
               "per_problem_flops": [o.flops for o in ops], "launches": batch.launches_per_apply,
               "schedule": _batch_schedule(ops)}
        if with_e2e:
            # end to end through HeffBatch.apply_host: every step copies its
            # inputs in from pinned host memory and its outputs back; step
            # s+1's copy in and step s-1's copy out overlap step s's compute
            assert batch.total == int(offs[-1])
            host_in = [torch.empty(batch.total, dtype=torch.float64, pin_memory=True) for _ in range(2)]
            host_out = [torch.empty(batch.total, dtype=torch.float64, pin_memory=True) for _ in range(2)]
            for h in host_in:
                h.copy_(x_all.cpu())
            batch.apply_host([host_in[i % 2] for i in range(args.warmup)],
                             [host_out[i % 2] for i in range(args.warmup)])
            barrier()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(st)
            batch.apply_host([host_in[i % 2] for i in range(args.steps)],
                             [host_out[i % 2] for i in range(args.steps)])
            b.record(st)
            barrier()
            res["e2e_ms"] = max_over_ranks(a.elapsed_time(b) / args.steps)
            res["e2e_bytes"] = int(offs[-1]) * 8
            batch.apply(xs, ys)
            torch.cuda.synchronize()
            res["e2e_max_abs_diff_vs_device"] = float((host_out[(args.steps - 1) % 2] - y_all.cpu()).abs().max())
        # every problem of the batched apply against its operator applied alone
        batch.apply(xs, ys)
        torch.cuda.synchronize()
        n_eq, worst = 0, 0.0
        for o, x, y in zip(ops, xs, ys):
            y1 = o.apply(x)
            torch.cuda.synchronize()
            o.release_scratch()
            n_eq += int(torch.equal(y1, y))
            worst = max(worst, float(torch.linalg.norm(y1 - y)) / max(float(torch.linalg.norm(y1)), 1e-300))
            del y1
        res["batch_vs_single"] = {"problems": len(ops), "bitwise_equal": n_eq, "max_rel_diff": worst}
        del batch, ops, x_all, y_all, xs, ys
        torch.cuda.empty_cache()
        return res

    r64 = run_precision("fp64")
    # schedule of the mixed stages 1-3: tuned on these problems (autotune.py)
    # unless given on the command line
    tuning = None
    if args.unfused or args.routed or args.auto or args.c_per_tile or args.no_tune:
        kind = 0 if args.unfused else 2 if args.routed else -1 if args.auto else 1
        schedule = {"fuse_mpo": kind, "c_per_tile": args.c_per_tile}
    else:
        from tenax_b200 import autotune

        schedule, cand_ms = autotune.tune(problems, args.precision, cache_path=None)
        tuning = {"chosen": schedule, "candidates_ms_per_step": cand_ms,
                  "key": json.loads(autotune.cache_key(problems, args.precision))}
    sampler = ClockSampler(local)
    rmx = run_precision(args.precision, with_e2e=True, sampler=sampler, schedule=schedule)
    clocks = sampler.summary()

    # ranks draw different problems: the job's work is the sum over ranks, its
    # time the slowest rank's (the ms values above are already maxima)
    flops_all = replicas.sum_over_ranks(rmx["flops"], dist, dev)
    value = flops_all / (rmx["ms"] * 1e-3) / 1e12
    fp64_value = replicas.sum_over_ranks(r64["flops"], dist, dev) / (r64["ms"] * 1e-3) / 1e12
    peaks, peak_src = _peaks()
    # dominant GEMM stage of the mixed step
    st_ms = rmx["stage_ms"]
    fused = rmx["schedule"]["fuse_mpo"] == 1
    routed = rmx["schedule"]["fuse_mpo"] in (2, -1)
    # the fused kernel does stage 1 and the MPO; its tensor work is stage 1's
    gemm = {1: rmx["stage_flops"][0] + (rmx["stage_flops"][1] if fused else 0.0), 3: rmx["stage_flops"][2]}
    dom = max((1, 3), key=lambda s: st_ms[s])
    if fused:
        stage_names = ["pack theta panels", "fused stages 1-3 (L.theta in TMEM, W_l W_r epilogue)",
                       "none (MPO inside the fused kernel)", "stage-4 GEMM .R"]
    elif routed and rmx["schedule"]["fuse_mpo"] == -1:
        stage_names = ["pack theta", "stage-1 GEMM L.theta: routed epilogue for the routed problems, X1 for the "
                       "others", "MPO kernel: multi-term outputs (routed problems), all outputs (the others)",
                       "stage-4 GEMM .R"]
    elif routed:
        stage_names = ["pack theta", "stage-1 GEMM L.theta, epilogue routes single-term W_l W_r outputs "
                       "into the stage-4 operand", "MPO kernel: multi-term outputs from the kept X1 slots",
                       "stage-4 GEMM .R"]
    else:
        stage_names = ["pack theta", "stage-1 GEMM L.theta", "fused MPO (W_l W_r)", "stage-4 GEMM .R"]
    dom_name = ("fused stages 1-3 (tcgen05 + W_l W_r epilogue)" if fused and dom == 1
                else "stage-1 tcgen05 grouped GEMM, routed epilogue" if routed and dom == 1
                else f"{STAGE_GEMM[dom]} tcgen05 grouped GEMM")
    split = 3.0 if args.precision == "bf16x3" else 1.0
    peak = peaks["bf16_tflops"] / split if args.precision == "bf16x3" else peaks["bf16_tflops"] / 2.0
    achieved = gemm[dom] / (st_ms[dom] * 1e-3) / 1e12
    traffic = None
    tp = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if os.path.exists(tp):
        sched1 = "auto1" if rmx["schedule"]["fuse_mpo"] == -1 else "routed1"
        key = (f"{args.precision}_fused1" if fused and dom == 1 else f"{args.precision}_{sched1}" if routed and dom == 1
               else f"{args.precision}_stage{dom}")
        traffic = json.load(open(tp)).get(key)
    if rank == 0:
        out = {
            "metric": METRIC, "value": round(value, 3), "unit": "TFLOP/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(rmx["ms"], 4), "higher_is_better": True,
            "scaling": "weak" if args.mode == "replicas" else "strong",
            "vs_baseline": None, "dtype": args.precision, "data": "synthetic (seeded N(0,1) blocks; no dataset)",
            "config": bench_config(args.problems, batch_chi_counts, flops_all, share_note),
            "fp64": {"value": round(fp64_value, 3), "unit": "TFLOP/s", "ms_per_step": round(r64["ms"], 4),
                     "stage_ms": [round(x, 4) for x in r64["stage_ms"]]},
            "mixed_over_fp64": round(value / fp64_value, 3),
            "stage_ms": [round(x, 4) for x in st_ms],
            "stage_names": stage_names, "schedule": rmx["schedule"], "autotune": tuning,
            "roofline": {"bound": "tensor", "kernel": dom_name, "achieved":
                         round(achieved, 2), "peak": round(peak, 1), "unit": "TFLOP/s",
                         "frac": round(achieved / peak, 4), "peak_source": f"{peak_src} bf16 burst"
                         + (" / 3 (three products)" if split == 3 else " / 2 (tf32)"), "traffic": traffic,
                         "dram": _dram_view(traffic, st_ms[dom], peaks, peak_src)},
            "e2e": {"value": round(flops_all / (rmx["e2e_ms"] * 1e-3) / 1e12, 3), "unit": "TFLOP/s",
                    "h2d_bytes_per_step": rmx["e2e_bytes"], "d2h_bytes_per_step": rmx["e2e_bytes"],
                    "ms_per_step": round(rmx["e2e_ms"], 4), "api": "HeffBatch.apply_host (pinned host buffers; "
                    "step s+1 copied in and step s-1 copied out while step s computes)",
                    "max_abs_diff_vs_device_apply": rmx["e2e_max_abs_diff_vs_device"]},
            "gpu_launches": rmx["launches"] * args.steps, "cuda_graph": not args.no_graph,
            "device_error_flag": rmx["err"],
            "clocks": clocks,
        }
        if world == 1:
            out["parity"] = bench_parity(problems, args.precision, rmx["schedule"])
        # the timed batch's outputs against each operator applied alone (this rank's problems)
        out.setdefault("parity", {})["batch_vs_single"] = {"fp64": r64["batch_vs_single"],
                                                           args.precision: rmx["batch_vs_single"]}
        out["parity"]["ok"] = bool(out["parity"].get("ok", True) and all(
            v["bitwise_equal"] == v["problems"] for v in out["parity"]["batch_vs_single"].values()))
        if world == 1 and not args.no_cpu_baseline:
            out["cpu_baseline"] = cpu_baseline(chi_counts, seed=args.seed)
        if world == 1 and not args.no_dmrg:
            del problems
            torch.cuda.empty_cache()
            out["dmrg"] = dmrg_sweeps(chi=args.chi, sweeps=2, lanczos=args.lanczos, seed=args.seed)
        print(json.dumps(out), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def partition_note(world, n_problems, n_rank0):
    return (f"partition x{world} (one {n_problems}-problem batch split by greedy FLOP-balanced assignment; "
            f"rank 0 holds {n_rank0})")


def bench_config(n_problems, chi_counts, flops_per_step, parallelism):
    """The ``config`` object of both arms' lines: the workload, its chi mix and
    the job's FLOPs per step."""
    return {"workload": WORKLOAD, "problems": n_problems, "chi_counts": {int(k): int(v) for k, v in chi_counts.items()},
            "flops_per_step": flops_per_step,
            "flop_count": "block-sparse 4-stage sector GEMM flops from stored block dims",
            "l2": "inputs larger than L2 (operators+theta >> 126 MB); no flush", "parallelism": parallelism}


def _batch_schedule(ops) -> dict:
    """The schedule of a batch's operators; with the automatic schedule
    (routed from 5e9 FLOPs per operator, unfused below) the count of each."""
    kinds = [o.schedule["fuse_mpo"] for o in ops]
    if len(set(kinds)) == 1:
        return ops[0].schedule
    return {"fuse_mpo": -1, "c_per_tile": 0, "routed_problems": kinds.count(2), "unfused_problems": kinds.count(0)}


def bench_parity(problems, precision, schedule=None):
    """Parity on the benchmarked inputs: the first problem of each chi of the
    batch applied in FP64 and in the mixed precision on the device (relative
    Frobenius difference, mixed vs FP64), and the smallest chi's both
    results against the oracle's per-block-combination H_eff on the host."""
    import torch

    from oracle import dmrg as odmrg
    from tenax_b200 import HeffOperator
    from tenax_b200.tensor import SymmetricTensor, embed_in_keys

    firsts = {}
    for p in problems:
        firsts.setdefault(int(p.chi), p)

    def rel(a, b):
        num = sum(float(np.sum((a[k] - b.get(k, 0.0)) ** 2)) for k in a)
        num += sum(float(np.sum(b[k] ** 2)) for k in b if k not in a)
        den = sum(float(np.sum(v * v)) for v in b.values())
        return float(np.sqrt(num / max(den, 1e-300)))

    res = {"mixed_vs_fp64_device": {}, "tolerances": {"fp64": 1e-12, "bf16x3": 4e-5, "tf32": 5e-3}}
    for chi in sorted(firsts):
        p = firsts[chi]
        outs = {}
        for prec in ("fp64", precision):
            op = HeffOperator(p.L, p.Wl, p.Wr, p.R, p.theta.indices, p.theta.keys, prec,
                              schedule=None if prec == "fp64" else schedule)
            x = embed_in_keys(p.theta, op.keys)
            y = op.apply(x.data)
            torch.cuda.synchronize()
            outs[prec] = SymmetricTensor.from_flat(p.theta.indices, op.keys, y).numpy_blocks()
            if chi == min(firsts) and prec == "fp64":
                ref = odmrg.heff_matvec(*_host_problem_with_theta(p, x)).blocks
            del op
        res["mixed_vs_fp64_device"][chi] = rel(outs[precision], outs["fp64"])
        if chi == min(firsts):
            res["oracle_chi"] = chi
            res["fp64_vs_oracle"] = rel(outs["fp64"], ref)
            res[f"{precision}_vs_oracle"] = rel(outs[precision], ref)
    res["ok"] = bool(res["fp64_vs_oracle"] <= 1e-12 and res[f"{precision}_vs_oracle"] <= res["tolerances"][precision]
                     and all(v <= res["tolerances"][precision] for v in res["mixed_vs_fp64_device"].values()))
    return res


def _host_problem_with_theta(p, x):
    """Oracle tensors of a device problem with theta replaced by ``x``."""
    h = _host_problem(p)
    h[1] = _host_problem(type(p)(p.L, x, p.Wl, p.Wr, p.R, p.chi))[1]
    return h


def dmrg_sweeps(chi=2048, sweeps=2, lanczos=20, seed=0):
    """The sweep-seconds half of the metric, compactly: two-site DMRG on the
    4x6 Heisenberg cylinder at chi (the --dmrg study's workload, fewer
    sweeps), FP64 and split-BF16x3, each arm with empty plan caches.
    Returns per-sweep seconds, final energies and their difference."""
    from tenax_b200 import contraction as _contraction, dense as _dense
    from tenax_b200.dmrg import DMRGConfig, SweepStats, dmrg
    from tenax_b200.workloads import cylinder_mpo, random_symmetric_mps

    mpo = cylinder_mpo(4, 6)
    res = {"workload": f"two-site DMRG, 4x6 Heisenberg cylinder (U(1), Dw=26), chi={chi}, {sweeps} sweeps, "
                       f"{lanczos} Lanczos steps, seeded random initial MPS", "sweep_s": {}, "energy": {}}
    for prec in ("fp64", "bf16x3"):
        _contraction._PLANS.clear()
        _dense._PLANS.clear()
        mps = random_symmetric_mps(24, chi, seed=seed)
        cfg = DMRGConfig(max_bond_dim=chi, num_sweeps=sweeps, lanczos_max_iter=lanczos, convergence_tol=0.0,
                         precision=prec)
        stats: list = []
        r = dmrg(mpo, mps, cfg, stats)
        res["sweep_s"][prec] = [round(x.seconds, 3) for x in stats if isinstance(x, SweepStats)]
        res["energy"][prec] = float(r.energy)
        del r, mps
    res["dE_vs_fp64"] = res["energy"]["bf16x3"] - res["energy"]["fp64"]
    res["last_sweep_fp64_over_mixed"] = round(res["sweep_s"]["fp64"][-1] / res["sweep_s"]["bf16x3"][-1], 3)
    return res


def _host_problem(p):
    """Device problem -> oracle tensors on the host."""
    from oracle.blocksparse import Leg, OTensor

    def h(t):
        return OTensor(tuple(Leg(i.charges, int(i.flow), i.label) for i in t.indices), t.numpy_blocks())

    return [h(t) for t in (p.L, p.theta, p.Wl, p.Wr, p.R)]


STAGE_GEMM = {1: "stage-1 (L.theta)", 3: "stage-4 (.R)"}


def _load_host_module(name):
    """A pure-NumPy module of the package, loaded by file path so that the
    package (and its device library) is never imported."""
    import importlib.util

    mod_name = f"_host_{name}"
    if mod_name in sys.modules:
        return sys.modules[mod_name]
    spec = importlib.util.spec_from_file_location(mod_name, os.path.join(ROOT, "tenax_b200", f"{name}.py"))
    mod = importlib.util.module_from_spec(spec)
    sys.modules[mod_name] = mod  # dataclasses look their module up here
    spec.loader.exec_module(mod)
    return mod


class HostProblems:
    """The batch's two-site problem structures on the host, without the
    device library: the same bond sectors, key sets, flows and cylinder MPO
    sites as the GPU workload (structure depends only on chi), with seeded
    N(0,1) blocks from NumPy.  FLOPs come from the oracle's count of the
    stored block dims."""

    def __init__(self, seed: int):
        from oracle.blocksparse import Leg, OTensor

        self.sec = _load_host_module("sectors")
        am = _load_host_module("auto_mpo")
        sites = am.heisenberg_cylinder_sites(4, 6)
        self.wl, self.wr = sites[7], sites[8]
        self.W = [OTensor(tuple(Leg(c, f, l) for c, f, l in zip(s.charges, s.flows, s.labels)), s.blocks())
                  for s in (self.wl, self.wr)]
        self.gen = np.random.default_rng(seed)
        self._Leg, self._OTensor = Leg, OTensor

    def make(self, chi: int, fill: bool = True, **sector_kw):
        """(L, theta, W_l, W_r, R) oracle tensors of one chi and their FLOPs;
        ``fill=False`` gives zero-cost read-only blocks (structure only)."""
        from oracle import dmrg as odmrg

        Leg, OTensor, sec = self._Leg, self._OTensor, self.sec
        v = sec.bond_charges(int(chi), **sector_kw)

        def blocks(legs, keys):
            shapes = {k: tuple(int(np.sum(l.charges == q)) for l, q in zip(legs, k)) for k in keys}
            if not fill:
                return {k: np.broadcast_to(np.float64(0.0), sh) for k, sh in shapes.items()}
            return {k: self.gen.standard_normal(sh) for k, sh in shapes.items()}

        Lg = (Leg(v, -1, "vl"), Leg(self.wl.charges[0], -1, "wl"), Leg(v, -1, "vl_c"))
        Rg = (Leg(v, 1, "vr"), Leg(self.wr.charges[3], 1, "wr"), Leg(v, 1, "vr_c"))
        Tg = (Leg(v, 1, "vl"), Leg(sec.PHYS, 1, "p1"), Leg(sec.PHYS, 1, "p2"), Leg(v, -1, "vr"))
        L = OTensor(Lg, blocks(Lg, sec.env_keys(v, self.wl.charges[0], v)))
        R = OTensor(Rg, blocks(Rg, sec.env_keys(v, self.wr.charges[3], v)))
        T = OTensor(Tg, blocks(Tg, sec.theta_keys(v, v)))
        args = (L, T, self.W[0], self.W[1], R)
        return args, odmrg.heff_flops(*args)


def cpu_chi_schedule(n_steps: int, chis=CHIS, n_top: int = 1) -> list:
    """The bond dimension timed at each step of a CPU sample: the largest chi
    exactly ``n_top`` times (spread over the run), the other chis in
    ascending rotation on the remaining steps; every chi appears once the
    run has len(chis) steps."""
    chis = sorted(int(c) for c in chis)
    top, rest = chis[-1], chis[:-1]
    n_top = max(1, min(n_top, n_steps))
    top_at = {int(round((i + 0.5) * n_steps / n_top - 0.5)) for i in range(n_top)}
    out, j = [], 0
    for i in range(n_steps):
        if i in top_at or not rest:
            out.append(top)
        else:
            out.append(rest[j % len(rest)])
            j += 1
    return out


def time_cpu_schedule(hp: "HostProblems", schedule: list, warmup: int = 1) -> dict:
    """Time one oracle H_eff matvec per schedule entry (the reference's
    per-block-combination algorithm, algorithms/dmrg.py:1048-1151, NumPy with
    all BLAS threads).  Returns per-chi seconds and FLOPs and the loop time."""
    from oracle import dmrg as odmrg

    probs = {c: hp.make(c) for c in sorted(set(schedule))}
    small = probs[min(probs)]
    for _ in range(max(0, warmup)):
        odmrg.heff_matvec(*small[0])
    per = {c: [] for c in probs}
    t_loop = time.perf_counter()
    for c in schedule:
        t0 = time.perf_counter()
        odmrg.heff_matvec(*probs[c][0])
        per[c].append(time.perf_counter() - t0)
    loop_s = time.perf_counter() - t_loop
    return {"seconds": per, "flops": {c: probs[c][1] for c in probs}, "loop_s": loop_s}


def batch_rate(timing: dict, chi_counts: dict) -> tuple:
    """FLOP-weighted rate of a whole batch from measured per-chi matvec times
    (median per chi): sum_chi n_chi f_chi / sum_chi n_chi t_chi, with the
    per-chi rates."""
    per_chi, fl, tt = {}, 0.0, 0.0
    for c, n in chi_counts.items():
        c = int(c)
        ts = timing["seconds"].get(c)
        if not ts or n == 0:
            continue
        t = statistics.median(ts)
        f = timing["flops"][c]
        per_chi[c] = {"tflops": round(f / t / 1e12, 6), "s_per_matvec": round(t, 4), "gflop": round(f / 1e9, 3),
                      "timed": len(ts)}
        fl += n * f
        tt += n * t
    return (fl / tt / 1e12 if tt > 0 else 0.0), per_chi


def cpu_baseline(chi_counts, seed=0, n_steps=4):
    """The cpu_baseline leg: the oracle port of the reference's H_eff on the
    host cores, one matvec of each chi of the batch (the largest once), the
    batch rate FLOP-weighted from the measured per-chi times."""
    hp = HostProblems(seed + 1)
    sched = cpu_chi_schedule(n_steps)
    tm = time_cpu_schedule(hp, sched)
    rate, per_chi = batch_rate(tm, chi_counts)
    return {"value": round(rate, 6), "unit": "TFLOP/s", "cores": os.cpu_count(), "kind": "port",
            "sample": f"one oracle matvec per chi {sorted(set(sched))} ({tm['loop_s']:.1f} s); batch rate weighted "
            f"by the batch's chi counts; numpy einsum per block combination, BLAS threads={os.cpu_count()}",
            "per_chi": per_chi}


def run_reference(args):
    """CPU arm: the oracle port of the reference's H_eff on the host cores.

    Never imports the package or loads its device library: structures come
    from the pure-NumPy sector module and the AutoMPO sites, FLOPs from the
    oracle's count.  Each timed step is one matvec of the batch's structure at
    the chi the schedule gives (the largest chi once, the others in rotation);
    ``ms_per_step`` is the timed loop's own time per step, and ``value`` the
    batch rate FLOP-weighted by the batch's chi counts from the measured
    per-chi times."""
    if int(os.environ.get("RANK", "0")) != 0:
        return
    chis = np.random.default_rng(args.seed).choice(np.asarray(CHIS), size=N_PROBLEMS)
    chi_counts = {int(c): int(np.sum(chis == c)) for c in CHIS}
    hp = HostProblems(args.seed + 1)
    sched = cpu_chi_schedule(args.steps)
    tm = time_cpu_schedule(hp, sched, warmup=args.warmup)
    value, per_chi = batch_rate(tm, chi_counts)
    # the whole batch's FLOPs (structure only for a chi the schedule did not time)
    flops_of = dict(tm["flops"])
    for c in chi_counts:
        if c not in flops_of:
            flops_of[c] = hp.make(c, fill=False)[1]
    batch_flops = sum(chi_counts[c] * flops_of[c] for c in chi_counts)
    untimed = sorted(c for c in chi_counts if c not in tm["flops"] and chi_counts[c])
    sample = (f"each timed step: one oracle H_eff matvec of the batch's structure at one chi (schedule "
              f"{sched}); value = the 64-problem batch's FLOPs / its time from the measured median per-chi "
              f"matvec times; ms_per_step = the timed loop's own time per step")
    if untimed:
        sample += f"; chi {untimed} not timed in this short run, so value covers the timed chi only"
    out = {"metric": METRIC, "value": round(value, 6), "unit": "TFLOP/s",
           "n_gpus": int(os.environ.get("WORLD_SIZE", "1")), "steps": args.steps, "warmup": args.warmup,
           "ms_per_step": round(tm["loop_s"] / args.steps * 1e3, 3), "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded N(0,1) blocks)",
           "impl": "reference",
           "config": bench_config(N_PROBLEMS, chi_counts, batch_flops, partition_note(1, N_PROBLEMS, N_PROBLEMS)),
           "sample": sample, "per_chi": per_chi,
           "cpu_baseline": {"value": round(value, 6), "unit": "TFLOP/s", "cores": os.cpu_count(), "kind": "port",
                            "sample": sample},
           "e2e": {"value": round(value, 6), "unit": "TFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def run_dmrg_study(args):
    """Two-site DMRG on the width-6 Heisenberg cylinder at chi (default 2048):
    sweep seconds and energies for FP64 and the mixed precisions; matvec
    residual of the mixed H_eff against FP64 at every site; energy
    difference to the FP64 run after every sweep."""
    import torch

    from tenax_b200.dmrg import DMRGConfig, SiteStats, SweepStats, dmrg
    from tenax_b200.workloads import cylinder_mpo, random_symmetric_mps

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    Lx, Ly = args.cyl_lx, 6
    mpo = cylinder_mpo(Lx, Ly)
    out = {"study": "two-site DMRG, width-6 Heisenberg cylinder (U(1), J=1)", "sites": Lx * Ly, "chi": args.chi,
           "sweeps": args.sweeps, "lanczos_max_iter": args.lanczos, "data": "seeded random initial MPS",
           "svd": {"driver": args.svd_driver, "streams": args.svd_streams}, "runs": {}}
    fp64_e = None
    out["plans"] = "contraction plan caches cleared before every run: each arm plans its own contractions"
    from tenax_b200 import contraction as _contraction, dense as _dense

    polish = [int(x) for x in str(args.fp64_polish).split(",")]
    arms = [(p, None) if p == "fp64" else (p, k) for p in args.dmrg_precisions.split(",")
            for k in (polish if p != "fp64" else [None])]
    for prec, k_polish in arms:
        name = prec if (prec == "fp64" or len(polish) == 1) else f"{prec}/polish{k_polish}"
        _contraction._PLANS.clear()
        _dense._PLANS.clear()
        mps = random_symmetric_mps(Lx * Ly, args.chi, seed=args.seed)
        cfg = DMRGConfig(max_bond_dim=args.chi, num_sweeps=args.sweeps, lanczos_max_iter=args.lanczos,
                         convergence_tol=0.0, precision=prec, check_matvec_residual=prec != "fp64",
                         svd_driver=None if args.svd_driver == "default" else args.svd_driver,
                         svd_streams=args.svd_streams,
                         fp64_polish_steps=k_polish if k_polish is not None else DMRGConfig.fp64_polish_steps)
        stats: list = []
        phases: dict = {}
        res = dmrg(mpo, mps, cfg, stats, phases)
        sw = [s for s in stats if isinstance(s, SweepStats)]
        st = [s for s in stats if isinstance(s, SiteStats)]
        nsite = (Lx * Ly - 1) * 2
        rel = [s.matvec_rel_err for s in st if s.matvec_rel_err is not None]
        te = np.array(res.truncation_errors).reshape(len(sw), -1)
        diag = np.array([s.diag_seconds for s in st]).reshape(len(sw), nsite).sum(axis=1)
        run = {"sweep_s": [round(s.seconds - d, 3) for s, d in zip(sw, diag)],
               "diagnostic_s_excluded": [round(float(d), 3) for d in diag],
               "phase_s": {k: round(v, 3) for k, v in phases.items()},
               "energies": [float(e) for e in res.energies_per_sweep],
               "max_bond": [s.max_bond for s in sw], "matvecs_per_sweep": [s.matvecs for s in sw],
               "truncation_err_max": [float(x) for x in te.max(axis=1)],
               "site_seconds_max": round(max(s.seconds for s in st), 3)}
        if rel:
            r = np.array(rel).reshape(len(sw), nsite)
            run["matvec_rel_err_median"] = [float(np.median(x)) for x in r]
            run["matvec_rel_err_max"] = [float(np.max(x)) for x in r]
        if prec == "fp64":
            fp64_e = run["energies"]
        elif fp64_e is not None:
            run["dE_vs_fp64"] = [float(a - b) for a, b in zip(run["energies"], fp64_e)]
        if k_polish is not None:
            run["fp64_polish_steps"] = k_polish
        out["runs"][name] = run
        del res, mps
        torch.cuda.empty_cache()
    print(json.dumps(out), flush=True)


def run_dmrg_c1_study(args):
    """Config 1: two-site DMRG on the L=20 Heisenberg chain (Dw=5 MPO,
    virtual charges -4..4, chi=64, 2 sweeps, 10 Lanczos steps) from the
    fixture's MPO and random MPS (the inputs of the reference's own run,
    tests/golden/dmrg_c1_L20.npz).  Times the whole dmrg() call on the GPU
    (FP64 and split-BF16x3; the first call of a process, then a repeat) and
    the oracle's port of the reference's algorithm on the host cores, and
    compares every energy with the reference's."""
    import time

    import torch

    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    from fixture_io import unpack_tensor

    from tenax_b200.core import FlowDirection, TensorIndex, U1Symmetry
    from tenax_b200.dmrg import DMRGConfig, dmrg
    from tenax_b200.network import TensorNetwork
    from tenax_b200.tensor import SymmetricTensor

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    z = np.load(os.path.join(ROOT, "tests", "golden", "dmrg_c1_L20.npz"))
    L = 20
    host_mps = [unpack_tensor(z, f"mps{i}") for i in range(L)]
    host_mpo = [unpack_tensor(z, f"mpo{i}") for i in range(L)]
    e_ref = float(z["energy"])

    def dev(t):
        u1 = U1Symmetry()
        idx = tuple(TensorIndex(u1, l.charges, FlowDirection(l.flow), l.label) for l in t.legs)
        return SymmetricTensor(t.blocks, idx, _validate=False)

    def nets():
        mps, mpo = TensorNetwork("mps"), TensorNetwork("mpo")
        for i in range(L):
            mps.add_node(i, dev(host_mps[i]))
            mpo.add_node(i, dev(host_mpo[i]))
        return mpo, mps

    out = {"study": "config 1: two-site DMRG, L=20 Heisenberg chain, chi=64, 2 sweeps, 10 Lanczos steps",
           "data": "the reference run's own MPO and seeded random MPS (fixture)", "reference_energy": e_ref,
           "runs": {}}
    for prec in ("fp64", "bf16x3"):
        run = {}
        for label in ("first_call_s", "repeat_s"):
            mpo, mps = nets()
            cfg = DMRGConfig(max_bond_dim=64, num_sweeps=2, lanczos_max_iter=10, two_site=True, precision=prec)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            res = dmrg(mpo, mps, cfg)
            torch.cuda.synchronize()
            run[label] = round(time.perf_counter() - t0, 3)
            run["energy"] = float(res.energy)
            run["dE_vs_reference"] = float(res.energy) - e_ref
        out["runs"][prec] = run
    if not args.no_cpu_baseline:
        import oracle.dmrg as odmrg

        t0 = time.perf_counter()
        res = odmrg.dmrg(host_mpo, host_mps, max_bond_dim=64, num_sweeps=2, lanczos_max_iter=10)
        t1 = time.perf_counter() - t0
        e = float(res[0] if isinstance(res, tuple) else res)
        out["cpu_baseline"] = {"value": round(t1, 2), "unit": "s (whole run)", "cores": os.cpu_count(),
                               "kind": "port", "energy": e, "dE_vs_reference": e - e_ref,
                               "sample": "the whole config-1 run: the oracle's NumPy port of the reference's "
                                         "dmrg() with BLAS on all host cores"}
    print(json.dumps(out), flush=True)


def run_ctm_study(args):
    """Dense 1-site CTMRG (D=4, d=2, chi=80, 30 QR sweeps, square-lattice
    Heisenberg NN energy): forward and forward+gradient seconds on the GPU,
    the hand-written adjoint checked against central differences of the
    fixed-projector energy (h=1e-6, 20 random directions), the free-running
    energy, and the oracle's CPU forward (the reference's einsum order) on
    the same site tensor as the CPU baseline.  With --ctm-oracle-grad the
    oracle's torch-autograd gradient under the GPU's projectors is compared
    too (tens of seconds of CPU)."""
    import time

    import torch

    from tenax_b200.ipeps import CTMConfig, compute_energy_ctm, ctm, energy_and_grad, heisenberg_gate

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    D, d, chi, iters = 4, 2, args.ctm_chi, args.ctm_iters
    rng = np.random.default_rng(args.ctm_seed)
    A_host = rng.standard_normal((D, D, D, D, d)) / np.sqrt(2.0 * D ** 4)
    A = torch.from_numpy(A_host).cuda()
    H = heisenberg_gate()
    cfg = CTMConfig(chi=chi, max_iter=iters, conv_tol=0.0, projector_method="qr", qr_warmup_steps=0)

    def timed(fn, reps):
        ts = []
        for _ in range(reps):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            r = fn()
            torch.cuda.synchronize()
            ts.append(time.perf_counter() - t0)
        return r, ts

    def forward():
        with torch.no_grad():
            env = ctm(A, cfg)
            return float(compute_energy_ctm(A, env, H, d))

    forward()  # plans, cuSOLVER handles
    E, t_fwd = timed(forward, args.ctm_reps)
    (E_g, grad, Ps), t_grad = timed(lambda: energy_and_grad(A, H, cfg), args.ctm_reps)
    _, t_grad_fixed = timed(lambda: energy_and_grad(A, H, cfg, projectors=Ps), args.ctm_reps)

    def energy_fixed(x):
        with torch.no_grad():
            return float(compute_energy_ctm(x, ctm(x, cfg, projectors=Ps), H, d))

    h, worst, dirs = 1e-6, 0.0, []
    vr = np.random.default_rng(args.ctm_seed + 1)
    for _ in range(20):
        v = torch.from_numpy(vr.standard_normal(A.shape)).cuda()
        fd = (energy_fixed(A + h * v) - energy_fixed(A - h * v)) / (2 * h)
        ad = float((grad * v).sum())
        rel = abs(fd - ad) / max(abs(ad), 1e-3 * float(grad.norm() * v.norm()))
        worst = max(worst, rel)
        dirs.append(rel)
    out = {"study": "dense 1-site CTMRG, square-lattice S=1/2 Heisenberg, QR projectors (no warm-up)",
           "D": D, "d": d, "chi": chi, "sweeps": iters, "seed": args.ctm_seed, "data": "seeded N(0,1)/sqrt(2 D^4)",
           "energy_free_run": E, "energy_grad_run": E_g,
           "forward_s": [round(t, 4) for t in t_fwd], "forward_grad_s": [round(t, 4) for t in t_grad],
           "forward_grad_fixed_projectors_s": [round(t, 4) for t in t_grad_fixed],
           "grad_norm": float(grad.norm()),
           "fd_check": {"h": h, "directions": 20, "max_rel_err": worst, "median_rel_err": float(np.median(dirs)),
                        "projectors": "fixed (those of the gradient run)"}}
    if not args.no_cpu_baseline:
        import oracle.ctm as oc

        torch.set_num_threads(os.cpu_count() or 1)
        At = torch.from_numpy(A_host)
        t0 = time.perf_counter()
        with torch.no_grad():
            env = oc.ctm(At, chi, iters, "qr")
            E_cpu = float(oc.energy(At, env, oc.heisenberg_gate(), d))
        t_cpu = time.perf_counter() - t0
        t0 = time.perf_counter()
        E_rep = oc.energy_fixed(At, oc.heisenberg_gate(), chi, iters, [p.cpu() for p in Ps])
        out["cpu_baseline"] = {"value": round(t_cpu, 3), "unit": "s (forward, 30 sweeps + energy)",
                               "cores": torch.get_num_threads(), "kind": "port",
                               "sample": "the full forward of this workload, oracle restatement in the "
                                         "reference's einsum order (torch CPU float64)",
                               "energy_free_run": E_cpu}
        out["oracle_replay_of_gpu_projectors"] = {"dE": E_g - E_rep, "seconds": round(time.perf_counter() - t0, 3)}
        if args.ctm_oracle_grad:
            t0 = time.perf_counter()
            _, g_or, _ = oc.energy_and_grad(At, oc.heisenberg_gate(), chi, iters, projectors=[p.cpu() for p in Ps],
                                            checkpoint=True)
            out["oracle_autograd"] = {"rel_err": float((grad.cpu() - g_or).abs().max() / g_or.abs().max()),
                                      "seconds": round(time.perf_counter() - t0, 3)}
    print(json.dumps(out), flush=True)


def run_split_ctm_study(args):
    """Split CTMRG at the U(1) configuration (D=5, bond charges -2..2,
    physical {-1,+1}, chi = chi_I = 150, 40 sweeps, gradient with the sweeps
    recomputed in groups of 5) and, because the reference's re-wrap makes
    that environment identically zero, the same sizes with trivial charges.
    Reports forward and forward+gradient seconds (FP64 and split-BF16x3
    forward), peak device memory, energies, the mixed-vs-FP64 gradient
    difference, and the oracle's CPU time for one sweep (reference order)."""
    import time

    import torch

    from tenax_b200 import split_ctm as gs
    from tenax_b200.core import FlowDirection, TensorIndex, U1Symmetry
    from tenax_b200.ipeps import heisenberg_gate
    from tenax_b200.tensor import SymmetricTensor, compute_valid_blocks, block_shape

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    D, chi, iters, ck = 5, args.split_chi, args.split_iters, 5
    H = heisenberg_gate()
    u1 = U1Symmetry()
    out = {"study": "U(1) split CTMRG, square-lattice S=1/2 Heisenberg, ket/bra layers kept apart",
           "D": D, "chi": chi, "chi_I": chi, "sweeps": iters, "checkpoint_every": ck, "runs": {}}

    def site(trivial, seed):
        bond = np.zeros(D, np.int32) if trivial else np.arange(-(D // 2), D // 2 + 1, dtype=np.int32)
        phys = np.zeros(2, np.int32) if trivial else np.array([-1, 1], np.int32)
        flows = (FlowDirection.OUT, FlowDirection.IN, FlowDirection.OUT, FlowDirection.IN, FlowDirection.IN)
        idx = tuple(TensorIndex(u1, c, f, lab) for c, f, lab in
                    zip((bond, bond, bond, bond, phys), flows, ("u", "d", "l", "r", "phys")))
        rng = np.random.default_rng(seed)
        keys = sorted(k for k in compute_valid_blocks(idx) if all(s > 0 for s in block_shape(idx, k)))
        return SymmetricTensor({k: rng.standard_normal(block_shape(idx, k)) for k in keys}, idx)

    def timed(fn):
        torch.cuda.synchronize()
        torch.cuda.reset_peak_memory_stats()
        t0 = time.perf_counter()
        r = fn()
        torch.cuda.synchronize()
        return r, time.perf_counter() - t0, torch.cuda.max_memory_allocated() / 2 ** 30

    def arms(A, Ad, driver):
        """FP64 free run (recording its projectors), split-BF16x3 run replaying
        them, and forward+gradient of both with those projectors, all with
        one edge-SVD driver."""
        run = {"svd_driver": driver}
        rec: list = []
        with torch.no_grad():
            env, t, mem = timed(lambda: gs.ctm_split_tensor(A, chi, iters, conv_tol=0.0, record=rec,
                                                            svd_driver=driver))
            E = float(gs.compute_energy_split_ctm_tensor(A, env, H, 2))
        run["fp64_forward"] = {"s": round(t, 3), "peak_GiB": round(mem, 2), "energy": E,
                               "env_max_abs": max(float(x.abs().max()) for x in env)}
        with torch.no_grad():
            envm, t, mem = timed(lambda: gs.ctm_split_tensor(A, chi, iters, conv_tol=0.0, projectors=rec,
                                                             precision="bf16x3", svd_driver=driver))
            Em = float(gs.compute_energy_split_ctm_tensor(A, envm, H, 2))
        run["bf16x3_forward"] = {"s": round(t, 3), "peak_GiB": round(mem, 2), "energy": Em, "dE_vs_fp64": Em - E}
        grads = {}
        for prec in ("fp64", "bf16x3"):
            def fg():
                x = Ad.clone().requires_grad_(True)
                e = gs.ctm_split_tensor(A, chi, iters, conv_tol=0.0, projectors=rec, A_dense=x, precision=prec,
                                        checkpoint_every=ck, svd_driver=driver)
                En = gs.compute_energy_split_ctm_tensor(A, e, H, 2, A_dense=x)
                (g,) = torch.autograd.grad(En, x)
                return g

            g, t, mem = timed(fg)
            grads[prec] = g
            run[f"{prec}_forward_gradient_checkpointed"] = {"s": round(t, 3), "peak_GiB": round(mem, 2),
                                                             "grad_finite": bool(torch.isfinite(g).all()),
                                                             "grad_norm": float(g.norm())}
        g64, gmx = grads["fp64"], grads["bf16x3"]
        if torch.isfinite(g64).all() and torch.isfinite(gmx).all() and float(g64.abs().max()) > 0:
            run["grad_rel_err_bf16x3_vs_fp64"] = float((gmx - g64).abs().max() / g64.abs().max())
        return run

    out["note"] = ("the split-BF16x3 arms replay the FP64 run's projectors and compute their own edge SVDs; "
                   "inside degenerate singular-value clusters the polar driver's basis moves with the "
                   "perturbation, so the replayed projectors no longer match it: the Jacobi pair measures "
                   "the arithmetic's effect")
    for label, trivial in (("u1_charges_-2..2", False), ("trivial_charges", True)):
        A = site(trivial, args.seed + 5)
        Ad = A.todense()
        run = arms(A, Ad, "polar")
        if trivial:
            run["jacobi_pair"] = arms(A, Ad, "jacobi")
        out["runs"][label] = run
    if not args.no_cpu_baseline:
        import oracle.split_ctm as osc

        torch.set_num_threads(os.cpu_count() or 1)
        A = site(True, args.seed + 5)
        s = osc.Site(A.todense().cpu(), [i.charges for i in A.indices], [int(i.flow) for i in A.indices])
        t0 = time.perf_counter()
        with torch.no_grad():
            osc.ctm_split(s, chi, 1)
        t1 = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": round(t1 * iters, 1), "unit": "s (forward, extrapolated)",
                               "cores": torch.get_num_threads(), "kind": "port",
                               "sample": f"one sweep of the oracle restatement in the reference's order "
                                         f"(dense grown edge), {t1:.2f} s, times {iters} sweeps"}
    print(json.dumps(out), flush=True)


def run_ctm_tensor_study(args):
    """Block-sparse standard CTMRG (ctm_tensor) on a trivial-charge site
    tensor (D=4, d=2, chi=80, eigh projectors; the reference's U(1) runs
    end at an all-zero environment, so values need trivial charges): GPU
    forward seconds per sweep, the same run in FP64 and split-BF16x3, and
    the oracle (the reference's block-sparse algorithm in NumPy) timed on
    a bounded number of sweeps and replaying the GPU's projectors, with
    its energy compared."""
    import time

    import torch

    from tenax_b200.core import FlowDirection, TensorIndex, U1Symmetry
    from tenax_b200.ipeps import heisenberg_gate
    from tenax_b200.tensor import SymmetricTensor
    from tenax_b200.tensor_ctm import compute_energy_ctm_tensor, ctm_tensor

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    D, d, chi, iters = 4, 2, args.ctm_chi, args.ctm_tensor_iters
    rng = np.random.default_rng(args.ctm_seed)
    A_host = rng.standard_normal((D, D, D, D, d)) / np.sqrt(2.0 * D ** 4)
    u1 = U1Symmetry()
    flows = (FlowDirection.OUT, FlowDirection.IN, FlowDirection.OUT, FlowDirection.IN, FlowDirection.IN)
    idx = tuple(TensorIndex(u1, np.zeros(n, np.int32), f, lab)
                for n, f, lab in zip(A_host.shape, flows, ("u", "d", "l", "r", "phys")))
    A = SymmetricTensor.from_dense(A_host, idx)
    H = heisenberg_gate()
    out = {"study": "block-sparse standard CTMRG (ctm_tensor), trivial charges, eigh projectors",
           "D": D, "d": d, "chi": chi, "sweeps": iters, "seed": args.ctm_seed, "data": "seeded N(0,1)/sqrt(2 D^4)"}

    def run(**kw):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        with torch.no_grad():
            env = ctm_tensor(A, chi, iters, 0.0, **kw)
            E = float(compute_energy_ctm_tensor(A, env, H, d))
        torch.cuda.synchronize()
        return E, time.perf_counter() - t0

    run()  # plans, cuSOLVER handles
    rec: list = []
    E, t = run(record=rec)
    out["fp64"] = {"s": round(t, 4), "s_per_sweep": round(t / iters, 5), "energy": E}
    Em, tm = run(projectors=rec, precision="bf16x3")
    out["bf16x3_replay"] = {"s": round(tm, 4), "energy": Em, "dE_vs_fp64": Em - E}
    if not args.no_cpu_baseline:
        import oracle.ctm_tensor as oct
        from oracle.blocksparse import Leg, OTensor

        z = np.zeros(D, np.int32)
        legs = (Leg(z, -1, "u"), Leg(z, 1, "d"), Leg(z, -1, "l"), Leg(z, 1, "r"), Leg(np.zeros(d, np.int32), 1, "phys"))
        Ao = OTensor(legs, {(0, 0, 0, 0, 0): A_host})
        k = min(iters, args.ctm_tensor_cpu_sweeps)
        rec_o: list = []
        t0 = time.perf_counter()
        env_o = oct.ctm_tensor(Ao, chi, k, 0.0, True, "eigh", 0, rec=rec_o)
        t_cpu = time.perf_counter() - t0
        E_o = oct.energy(Ao, env_o, np.asarray(H.cpu()), d)
        with torch.no_grad():
            E_g = float(compute_energy_ctm_tensor(A, ctm_tensor(A, chi, k, 0.0, projectors=rec_o), H, d))
        out["cpu_baseline"] = {"value": round(t_cpu / k, 3), "unit": "s per sweep", "cores": os.cpu_count(),
                               "kind": "port", "sample": f"{k} sweeps of the oracle restatement (NumPy block-sparse "
                                                         f"contract, fuse and per-sector eigh, BLAS threads)"}
        out["gpu_replay_of_oracle_projectors"] = {"sweeps": k, "dE": E_g - E_o}
    print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--dmrg", action="store_true", help="run the cylinder DMRG precision study instead")
    ap.add_argument("--dmrg-c1", action="store_true",
                    help="run the config-1 chain DMRG (GPU path against the oracle's CPU port) instead")
    ap.add_argument("--chi", type=int, default=2048)
    ap.add_argument("--sweeps", type=int, default=4)
    ap.add_argument("--lanczos", type=int, default=20)
    ap.add_argument("--cyl-lx", type=int, default=4)
    ap.add_argument("--dmrg-precisions", default="fp64,bf16x3,tf32")
    ap.add_argument("--svd-driver", default="native",
                    help="per-sector SVD of the DMRG study: 'native' (tnx_svd_batch), a torch.linalg.svd driver, "
                         "or 'default'")
    ap.add_argument("--svd-streams", type=int, default=8)
    ap.add_argument("--fp64-polish", default="3",
                    help="FP64 Lanczos steps after a mixed solve (comma list: one mixed arm per value)")
    ap.add_argument("--ctm", action="store_true", help="run the dense CTMRG forward/gradient study instead")
    ap.add_argument("--ctm-chi", type=int, default=80)
    ap.add_argument("--ctm-iters", type=int, default=30)
    ap.add_argument("--ctm-seed", type=int, default=2024)
    ap.add_argument("--ctm-reps", type=int, default=3)
    ap.add_argument("--ctm-oracle-grad", action="store_true")
    ap.add_argument("--ctm-tensor", action="store_true", help="run the block-sparse CTMRG study instead")
    ap.add_argument("--ctm-tensor-iters", type=int, default=10)
    ap.add_argument("--ctm-tensor-cpu-sweeps", type=int, default=2)
    ap.add_argument("--split-ctm", action="store_true", help="run the U(1) split CTMRG study instead")
    ap.add_argument("--split-chi", type=int, default=150)
    ap.add_argument("--split-iters", type=int, default=40)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--no-graph", action="store_true", help="time eager applies instead of CUDA-graph replays")
    ap.add_argument("--unfused", action="store_true",
                    help="mixed stages 1-3 as stage-1 GEMM + X1 in HBM + MPO kernel instead of the fused kernel")
    ap.add_argument("--routed", action="store_true",
                    help="mixed stages 1-3 with the routed stage-1 epilogue, without tuning")
    ap.add_argument("--auto", action="store_true",
                    help="mixed stages 1-3 routed or unfused per problem by its size, without tuning")
    ap.add_argument("--c-per-tile", type=int, default=0, help="fused kernel: c values per tile (0 = largest that fits)")
    ap.add_argument("--no-tune", action="store_true", help="fused schedule without tuning it")
    ap.add_argument("--mode", default="partition", choices=["partition", "replicas"],
                    help="N>1: split one batch over the ranks (partition, strong scaling) or give every rank its "
                         "own batch (replicas, weak scaling)")
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="bf16x3", choices=["bf16x3", "tf32"])
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-dmrg", action="store_true", help="leave the 2-sweep chi=2048 DMRG out of the default run")
    ap.add_argument("--problems", type=int, default=N_PROBLEMS,
                    help="problems per GPU (64 = the benchmark workload; smaller only for profiling)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    sys.path.insert(0, ROOT)
    if args.dmrg:
        run_dmrg_study(args)
    elif args.dmrg_c1:
        run_dmrg_c1_study(args)
    elif args.ctm:
        run_ctm_study(args)
    elif args.split_ctm:
        run_split_ctm_study(args)
    elif args.ctm_tensor:
        run_ctm_tensor_study(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
