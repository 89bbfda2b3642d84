"""The fused H_eff stages 1-3 kernel (L.theta accumulated in tensor memory,
W_l W_r applied in its epilogue) and the routed schedule (stage-1 GEMM whose
epilogue writes the single-term W_l W_r outputs into the stage-4 operand)
against the oracle and against the unfused three-kernel path (stage-1 GEMM,
X1 in HBM, MPO kernel) on the same inputs.

Tolerances (relative Frobenius error against the oracle): split-BF16x3 2e-5,
TF32 5e-3; fused against unfused: 2e-6 (BF16x3) and 1e-4 (TF32), since the
two paths sum the same FP32 products in different orders (the three-kernel
stage 1 adds a K slab's hi x hi products before its cross products, the
fused kernel interleaves them; measured up to 1.05e-6 on the 320-wide chain).  Routed against
unfused: bit for bit (the same operand images, the same MMA K order per
point, the same FP32 arithmetic for every output slot).
"""

import numpy as np
import pytest

from oracle.blocksparse import Leg, OTensor, blockwise_contract as o_blockwise

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a CUDA device", allow_module_level=True)

import tenax_b200 as tb  # noqa: E402
from tenax_b200 import workloads as W  # noqa: E402
from tenax_b200.tensor import SymmetricTensor, embed_in_keys  # noqa: E402

TOL = {"bf16x3": 2e-5, "tf32": 5e-3}
PATH_TOL = {"bf16x3": 2e-6, "tf32": 1e-4}
FUSED = {"fuse_mpo": 1, "c_per_tile": 0}
UNFUSED = {"fuse_mpo": 0, "c_per_tile": 0}
ROUTED = {"fuse_mpo": 2, "c_per_tile": 0}


def _host(t):
    return OTensor(tuple(Leg(i.charges, int(i.flow), i.label) for i in t.indices), t.numpy_blocks())


def _rel(a: dict, b: dict) -> float:
    num = sum(float(np.sum((a.get(k, 0) - b.get(k, 0)) ** 2)) for k in set(a) | set(b))
    den = sum(float(np.sum(v * v)) for v in b.values())
    return float(np.sqrt(num / max(den, 1e-300)))


def _problem(case):
    if case == "cylinder_multi_tile":  # Dw=26, sectors up to 64: several c-tiles per pair
        Wl, Wr = W.cylinder_bulk_w()
        return W.make_heff_problem(300, 300, Wl, Wr, np.random.default_rng(5), n_sectors=12, hi=64)
    if case == "tiny_sectors":  # extents 1-6: d-tiles almost all padding, c below one tile
        Wl, Wr = W.cylinder_bulk_w()
        return W.make_heff_problem(30, 30, Wl, Wr, np.random.default_rng(9), n_sectors=12, hi=6, lo=1)
    if case == "wide_chain":  # Dw=5 chain MPO, sectors up to 320: two d-tiles, several K slabs
        Wl, Wr = W.chain_bulk_w()
        return W.make_heff_problem(1400, 1400, Wl, Wr, np.random.default_rng(10), n_sectors=8, hi=320)
    if case == "cylinder_gaussian":  # the benchmark's sector shape at chi = 512
        Wl, Wr = W.cylinder_bulk_w()
        return W.make_heff_problem(512, 512, Wl, Wr, np.random.default_rng(3))
    raise ValueError(case)


def _op(p, precision, schedule):
    return tb.HeffOperator(p.L, p.Wl, p.Wr, p.R, p.theta.indices, p.theta.keys, precision, schedule=schedule)


def _apply(op, x):
    y = op.apply(x.data)
    torch.cuda.synchronize()
    assert op.device_error() == 0
    return y


@pytest.mark.parametrize("precision", ["bf16x3", "tf32"])
@pytest.mark.parametrize("case", ["cylinder_multi_tile", "tiny_sectors", "wide_chain", "cylinder_gaussian"])
def test_fused_matches_oracle_and_unfused(case, precision):
    p = _problem(case)
    fused = _op(p, precision, FUSED)
    assert fused.schedule["fuse_mpo"] == 1 and fused.schedule["c_per_tile"] >= 1
    unf = _op(p, precision, UNFUSED)
    assert unf.schedule["fuse_mpo"] == 0
    assert fused.keys == unf.keys
    x = embed_in_keys(p.theta, fused.keys)
    yf = SymmetricTensor.from_flat(p.theta.indices, fused.keys, _apply(fused, x)).numpy_blocks()
    yu = SymmetricTensor.from_flat(p.theta.indices, unf.keys, _apply(unf, x)).numpy_blocks()
    ref = o_blockwise([_host(t) for t in (p.L, x, p.Wl, p.Wr, p.R)], "abc,apqd,bpse,eqtf,dfg->cstg").blocks
    for k in yf:
        if k not in ref:
            assert np.all(yf[k] == 0.0), k
    assert _rel({k: v for k, v in yf.items() if k in ref}, ref) < TOL[precision]
    assert _rel({k: v for k, v in yu.items() if k in ref}, ref) < TOL[precision]
    assert _rel(yf, yu) < PATH_TOL[precision]


@pytest.mark.parametrize("precision", ["bf16x3", "tf32"])
@pytest.mark.parametrize("case", ["cylinder_multi_tile", "tiny_sectors", "wide_chain", "cylinder_gaussian"])
def test_routed_matches_unfused_bitwise(case, precision):
    p = _problem(case)
    rt = _op(p, precision, ROUTED)
    assert rt.schedule == ROUTED
    unf = _op(p, precision, UNFUSED)
    assert rt.keys == unf.keys
    x = embed_in_keys(p.theta, rt.keys)
    yr, yu = _apply(rt, x), _apply(unf, x)
    assert torch.equal(yr, yu)
    ref = o_blockwise([_host(t) for t in (p.L, x, p.Wl, p.Wr, p.R)], "abc,apqd,bpse,eqtf,dfg->cstg").blocks
    got = SymmetricTensor.from_flat(p.theta.indices, rt.keys, yr).numpy_blocks()
    assert _rel({k: v for k, v in got.items() if k in ref}, ref) < TOL[precision]


def test_routed_long_windows_are_exercised():
    """Tiny sectors put many row and column classes under one warp's chunk,
    so some windows exceed the 64 records a shared-memory window buffer holds
    and the epilogue reads them in pieces; the bitwise routed-vs-unfused test
    on this structure therefore covers that path.  Wide sectors keep every
    window in the buffer."""
    small = tb.HeffBatch([_op(_problem("tiny_sectors"), "bf16x3", ROUTED)])
    n, w = small.route_stats()
    assert n > 0 and w > 64, (n, w)
    unf = tb.HeffBatch([_op(_problem("tiny_sectors"), "bf16x3", UNFUSED)])
    assert unf.route_stats() == (0, 0)


def test_routed_batch_equals_individual():
    """Three problems of different chi in one routed batch: bit for bit the
    single-problem applies."""
    Wl, Wr = W.cylinder_bulk_w()
    gen = np.random.default_rng(18)
    probs = [W.make_heff_problem(c, c, Wl, Wr, gen, n_sectors=10, hi=48) for c in (120, 200, 160)]
    ops = [_op(p, "bf16x3", ROUTED) for p in probs]
    assert all(o.schedule == ROUTED for o in ops)
    xs = [embed_in_keys(p.theta, o.keys).data for p, o in zip(probs, ops)]
    singles = [o.apply(x) for o, x in zip(ops, xs)]
    batch = tb.HeffBatch(ops)
    outs = [o.out_like() for o in ops]
    batch.apply(xs, outs)
    torch.cuda.synchronize()
    assert batch.device_error() == 0
    for a, b in zip(singles, outs):
        torch.testing.assert_close(a, b, rtol=0, atol=0)


def test_routed_fp64_keeps_three_kernels():
    """FP64 has no routed epilogue: the request falls back to the unfused
    schedule, which is reported."""
    p = _problem("tiny_sectors")
    op = _op(p, "fp64", ROUTED)
    assert op.schedule == UNFUSED


@pytest.mark.parametrize("cc", [1, 2, 5])
def test_fused_tile_c_extent(cc):
    """Any c extent per tile gives the automatic choice's result (the MMA
    column range of a point does not change its K order)."""
    p = _problem("cylinder_multi_tile")
    auto = _op(p, "bf16x3", FUSED)
    fixed = _op(p, "bf16x3", {"fuse_mpo": 1, "c_per_tile": cc})
    assert fixed.schedule == {"fuse_mpo": 1, "c_per_tile": cc}
    x = embed_in_keys(p.theta, auto.keys)
    ya, yc = _apply(auto, x), _apply(fixed, x)
    assert float(torch.linalg.norm(ya - yc) / torch.linalg.norm(ya)) < 1e-6


def test_fused_batch_equals_individual():
    """Three problems of different chi in one fused batch: bit for bit the
    single-problem applies, three kernels (and a zeroing pass) per apply."""
    Wl, Wr = W.cylinder_bulk_w()
    gen = np.random.default_rng(8)
    probs = [W.make_heff_problem(c, c, Wl, Wr, gen, n_sectors=10, hi=48) for c in (120, 200, 160)]
    ops = [_op(p, "bf16x3", FUSED) for p in probs]
    assert all(o.schedule["fuse_mpo"] == 1 for o in ops)
    xs = [embed_in_keys(p.theta, o.keys).data for p, o in zip(probs, ops)]
    singles = [o.apply(x) for o, x in zip(ops, xs)]
    batch = tb.HeffBatch(ops)
    assert batch.launches_per_apply <= 4
    outs = [o.out_like() for o in ops]
    batch.apply(xs, outs)
    torch.cuda.synchronize()
    assert batch.device_error() == 0
    for a, b in zip(singles, outs):
        torch.testing.assert_close(a, b, rtol=0, atol=0)


def test_routed_and_unfused_share_a_batch():
    """Routed and unfused operators in one batch (one stage-1 launch with both
    kinds of groups, MPO tables per problem): bit for bit the single applies."""
    Wl, Wr = W.cylinder_bulk_w()
    gen = np.random.default_rng(21)
    probs = [W.make_heff_problem(c, c, Wl, Wr, gen, n_sectors=10, hi=48) for c in (120, 200, 160)]
    ops = [_op(p, "bf16x3", s) for p, s in zip(probs, (ROUTED, UNFUSED, ROUTED))]
    assert [o.schedule["fuse_mpo"] for o in ops] == [2, 0, 2]
    xs = [embed_in_keys(p.theta, o.keys).data for p, o in zip(probs, ops)]
    singles = [o.apply(x) for o, x in zip(ops, xs)]
    batch = tb.HeffBatch(ops)
    outs = [o.out_like() for o in ops]
    batch.apply(xs, outs)
    torch.cuda.synchronize()
    assert batch.device_error() == 0
    for a, b in zip(singles, outs):
        torch.testing.assert_close(a, b, rtol=0, atol=0)


@pytest.mark.parametrize("precision", ["bf16x3", "tf32"])
def test_routed_and_unfused_interleaved_tiles(precision):
    """A mixed batch with thousands of stage-1 tiles, so that every CTA of the
    persistent launch runs many tiles and routed tiles follow unfused ones
    (the window and class pipeline must advance on both kinds): bit for bit
    the single applies, and the automatic schedule gives the same bits."""
    Wl, Wr = W.cylinder_bulk_w()
    gen = np.random.default_rng(23)
    probs = [W.make_heff_problem(c, c, Wl, Wr, gen) for c in (1024, 512, 1024, 384)]
    scheds = (ROUTED, UNFUSED, ROUTED, UNFUSED)
    ops = [_op(p, precision, s) for p, s in zip(probs, scheds)]
    xs = [embed_in_keys(p.theta, o.keys).data for p, o in zip(probs, ops)]
    singles = [o.apply(x) for o, x in zip(ops, xs)]
    torch.cuda.synchronize()
    # the automatic schedule routes the two chi = 1024 operators and runs the others unfused
    auto = [_op(p, precision, None) for p in probs]
    assert [o.schedule["fuse_mpo"] for o in auto] == [2, 0, 2, 0]
    for batch in (tb.HeffBatch(ops), tb.HeffBatch(auto)):
        outs = [torch.full_like(a, float("nan")) for a in singles]
        # a first apply on other inputs leaves other values in every intermediate,
        # so a tile whose stores were skipped cannot pass on stale data
        batch.apply([-3.0 * x for x in xs], outs)
        for y in outs:
            y.fill_(float("nan"))
        batch.apply(xs, outs)
        torch.cuda.synchronize()
        assert batch.device_error() == 0
        for a, b in zip(singles, outs):
            torch.testing.assert_close(b, a, rtol=0, atol=0)


@pytest.mark.parametrize("pair", [(FUSED, UNFUSED), (ROUTED, FUSED)])
def test_mixed_schedules_cannot_share_a_batch(pair):
    p = _problem("tiny_sectors")
    a, b = _op(p, "bf16x3", pair[0]), _op(p, "bf16x3", pair[1])
    with pytest.raises(ValueError):
        tb.HeffBatch([a, b])


def test_autotune_picks_a_candidate_and_caches(tmp_path):
    """The tuner times every candidate schedule on the problems, returns the
    fastest, and a second call with the same sector profile reads it from
    the cache without timing."""
    from tenax_b200 import autotune

    Wl, Wr = W.cylinder_bulk_w()
    gen = np.random.default_rng(14)
    probs = [W.make_heff_problem(c, c, Wl, Wr, gen, n_sectors=10, hi=48) for c in (120, 200)]
    cands = autotune.candidates(probs, "bf16x3")
    assert UNFUSED in cands and ROUTED in cands and cands[0]["fuse_mpo"] == 1
    path = str(tmp_path / "tune.json")
    best, timings = autotune.tune(probs, "bf16x3", cache_path=path, reps=2)
    assert best in cands and len(timings) == len(cands)
    assert all(np.isfinite(v) and v > 0 for v in timings.values())
    again, t2 = autotune.tune(probs, "bf16x3", cache_path=path)
    assert again == best and t2 == {}
