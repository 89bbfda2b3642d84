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
