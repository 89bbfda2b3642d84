"""Multi-rank bookkeeping of the batched benchmark (tenax_b200.replicas) on
two gloo ranks on the CPU: per-rank problem draws differ, the reported time
is the slowest rank's and the whole-job throughput sums every rank's work."""

import json
import os
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")
dist = pytest.importorskip("torch.distributed")


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import datetime

    import torch.distributed as d

    from tenax_b200 import replicas
    from tenax_b200.workloads import draw_chis

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    d.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        seed = replicas.rank_seed(0, rank)
        chis = draw_chis(64, seed=seed).tolist()
        flops, ms = 1.0e12 * (rank + 1), 2.0 + rank
        res = {"seed": seed, "chis": chis,
               "max_ms": replicas.max_over_ranks(ms, d),
               "sum_flops": replicas.sum_over_ranks(flops, d),
               "tflops": replicas.whole_job_tflops(flops, ms, d)}
        d.barrier()
    finally:
        d.destroy_process_group()
    with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as fh:
        json.dump(res, fh)


def test_two_gloo_ranks(tmp_path):
    import torch.multiprocessing as mp

    world = 2
    mp.spawn(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    r = [json.load(open(tmp_path / f"rank{i}.json")) for i in range(world)]
    assert r[0]["seed"] == 0 and r[1]["seed"] == 1000
    assert r[0]["chis"] != r[1]["chis"]  # independent problems per rank
    for x in r:
        assert x["max_ms"] == 3.0
        assert x["sum_flops"] == 3.0e12
        assert abs(x["tflops"] - 3.0e12 / 3.0e-3 / 1e12) < 1e-9


def test_single_process_is_identity():
    from tenax_b200 import replicas

    assert replicas.max_over_ranks(2.5) == 2.5
    assert replicas.sum_over_ranks(7.0) == 7.0
    assert replicas.whole_job_tflops(1.0e12, 1.0) == pytest.approx(1000.0)
    assert replicas.rank_seed(5, 0) == 5 and replicas.rank_seed(5, 3) == 3005
    np.testing.assert_array_equal(__import__("tenax_b200.workloads", fromlist=["draw_chis"]).draw_chis(8, seed=0),
                                  np.random.default_rng(0).choice(np.asarray((256, 512, 1024, 2048)), size=8))


def test_partition_balances_the_benchmark_batch():
    """The 64-problem batch's per-problem FLOPs (structure depends only on
    chi) split over 2, 4 and 8 ranks: each problem exactly once, the busiest
    rank within 10% of the mean."""
    import importlib.util

    from tenax_b200 import replicas
    from tenax_b200.workloads import draw_chis

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    spec = importlib.util.spec_from_file_location("bench_part", os.path.join(root, "bench.py"))
    b = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(b)
    hp = b.HostProblems(0)
    per_chi = {c: hp.make(c, fill=False)[1] for c in (256, 512, 1024, 2048)}
    flops = [per_chi[int(c)] for c in draw_chis(64, seed=0)]
    for world in (1, 2, 4, 8):
        share = replicas.partition(flops, world)
        assert sorted(i for s in share for i in s) == list(range(64))
        loads = [sum(flops[i] for i in s) for s in share]
        assert max(loads) <= 1.1 * (sum(flops) / world), (world, loads)
        assert all(s for s in share)


def test_partition_edge_cases():
    from tenax_b200 import replicas

    assert replicas.partition([], 3) == [[], [], []]
    assert replicas.partition([5.0], 2) == [[0], []]
    # equal work: round robin by index
    assert replicas.partition([1.0] * 5, 2) == [[0, 2, 4], [1, 3]]
    # longest first: the big problem alone on rank 0
    assert replicas.partition([1.0, 10.0, 1.0, 1.0], 2) == [[1], [0, 2, 3]]
    with pytest.raises(ValueError):
        replicas.partition([1.0], 0)
    assert replicas.gather_to_root({3: "x"}) == {3: "x"}


def _partition_rank_main(rank, world, port, out_dir):
    """Each gloo rank applies the oracle H_eff to its share of a small batch
    and rank 0 gathers the results."""
    import datetime

    import torch.distributed as d

    from oracle import dmrg as odmrg
    from tenax_b200 import replicas

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    d.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        probs = _small_batch()
        flops = [odmrg.heff_flops(*p) for p in probs]
        mine = replicas.partition(flops, world)[rank]
        local = {i: odmrg.heff_matvec(*probs[i]).blocks for i in mine}
        merged = replicas.gather_to_root(local, d)
        d.barrier()
    finally:
        d.destroy_process_group()
    if rank == 0:
        import pickle

        with open(os.path.join(out_dir, "merged.pkl"), "wb") as fh:
            pickle.dump({"merged": merged, "shares": replicas.partition(flops, world)}, fh)


def _small_batch():
    """Six small cylinder problems (chi 40-120, 6 sectors) on the host."""
    import importlib.util

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    spec = importlib.util.spec_from_file_location("bench_small", os.path.join(root, "bench.py"))
    b = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(b)
    hp = b.HostProblems(21)
    return [hp.make(chi, n_sectors=6, lo=2, hi=64)[0] for chi in (40, 120, 64, 80, 48, 100)]


def test_partitioned_batch_on_two_gloo_ranks(tmp_path):
    """A batch split over two ranks and gathered on rank 0 equals the
    single-process results problem by problem (same arithmetic, bit for
    bit), and every problem ran on exactly one rank."""
    import pickle

    import torch.multiprocessing as mp

    from oracle import dmrg as odmrg

    world = 2
    mp.spawn(_partition_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    r = pickle.load(open(tmp_path / "merged.pkl", "rb"))
    probs = _small_batch()
    assert sorted(r["merged"]) == list(range(len(probs)))
    assert all(r["shares"])
    for i, p in enumerate(probs):
        ref = odmrg.heff_matvec(*p).blocks
        got = r["merged"][i]
        assert sorted(got) == sorted(ref)
        for k in ref:
            np.testing.assert_array_equal(got[k], ref[k])
