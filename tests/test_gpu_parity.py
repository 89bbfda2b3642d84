"""GPU parity of the C-ABI contraction and H_eff paths against the oracle.

Tolerances: FP64 paths are compared block by block at rtol 1e-12 (relative
Frobenius error 1e-12 for the fused H_eff); split-BF16x3 at relative
Frobenius error 2e-5; TF32 at 5e-3.
"""

import json
import os

import numpy as np
import pytest

from fixture_io import unpack_tensor
from oracle.blocksparse import Leg, OTensor, blockwise_contract as o_blockwise
from oracle import dmrg as odmrg

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a CUDA device", allow_module_level=True)

import tenax_b200 as tb  # noqa: E402
from tenax_b200.core import FlowDirection, TensorIndex, U1Symmetry, ZnSymmetry  # noqa: E402
from tenax_b200.tensor import SymmetricTensor, embed_in_keys  # noqa: E402


def to_dev(t: OTensor) -> SymmetricTensor:
    sym = U1Symmetry() if t.modulus is None else ZnSymmetry(t.modulus)
    idx = tuple(TensorIndex(sym, l.charges, FlowDirection(l.flow), l.label) for l in t.legs)
    return SymmetricTensor(t.blocks, idx, _validate=False)


def to_host(t: SymmetricTensor) -> OTensor:
    mod = t.indices[0].symmetry.n_values() if t.indices else None
    return OTensor(tuple(Leg(i.charges, int(i.flow), i.label) for i in t.indices), t.numpy_blocks(), mod)


def rel_err(a: dict, b: dict) -> float:
    num = sum(np.sum((a.get(k, 0) - b.get(k, 0)) ** 2) for k in set(a) | set(b))
    den = sum(np.sum(v ** 2) for v in b.values())
    return float(np.sqrt(num / max(den, 1e-300)))


def test_contract_golden_fp64(golden_dir):
    z = np.load(os.path.join(golden_dir, "contract.npz"))
    for c in json.load(open(os.path.join(golden_dir, "contract.json"))):
        ins = [to_dev(unpack_tensor(z, f"{c['name']}.in{i}")) for i in range(c["n_in"])]
        ref = unpack_tensor(z, f"{c['name']}.out")
        out = tb.contract_with_subscripts(ins, c["subscripts"], None)
        got = out.numpy_blocks()
        assert sorted(got) == sorted(ref.blocks), c["name"]
        for k in got:
            np.testing.assert_allclose(got[k], ref.blocks[k], rtol=1e-12, atol=1e-13, err_msg=c["name"])


def test_labels_contract_and_errors():
    u1 = U1Symmetry()
    a = SymmetricTensor.random_normal((TensorIndex(u1, np.array([-1, 0, 1]), FlowDirection.IN, "i"),
                                       TensorIndex(u1, np.array([-1, 0, 1]), FlowDirection.OUT, "j")), key=1)
    b = SymmetricTensor.random_normal((TensorIndex(u1, np.array([-1, 0, 1]), FlowDirection.IN, "j"),
                                       TensorIndex(u1, np.array([-1, 0, 1]), FlowDirection.OUT, "k")), key=2)
    c = tb.contract(a, b)
    assert c.labels() == ("i", "k")
    ref = a.todense().cpu().numpy() @ b.todense().cpu().numpy()
    np.testing.assert_allclose(c.todense().cpu().numpy(), ref, rtol=1e-12, atol=1e-14)
    with pytest.raises(ValueError):
        tb.contract(a, b, output_labels=["j"])
    with pytest.raises(ValueError):
        tb.contract(a, a.relabel("i", "j"), b)


def _heff_fixture(golden_dir):
    z = np.load(os.path.join(golden_dir, "dmrg_pieces.npz"))
    return z, [unpack_tensor(z, f"heff.{n}") for n in ("L", "theta", "Wl", "Wr", "R")]


def test_blockwise_heff_golden(golden_dir):
    z, (L, th, Wl, Wr, R) = _heff_fixture(golden_dir)
    dL, dth, dWl, dWr, dR = map(to_dev, (L, th, Wl, Wr, R))
    out = tb.blockwise_contract([dL, dth, dWl, dWr, dR], "abc,apqd,bpse,eqtf,dfg->cstg", dth.indices)
    ref = unpack_tensor(z, "heff.out")
    got = out.numpy_blocks()
    assert sorted(got) == sorted(ref.blocks)
    assert rel_err(got, ref.blocks) < 1e-12


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("bf16x3", 2e-5), ("tf32", 5e-3)])
def test_fused_heff_golden(golden_dir, precision, tol):
    z, (L, th, Wl, Wr, R) = _heff_fixture(golden_dir)
    dL, dth, dWl, dWr, dR = map(to_dev, (L, th, Wl, Wr, R))
    op = tb.HeffOperator(dL, dWl, dWr, dR, dth.indices, dth.keys, precision)
    assert op.fused  # the U(1) two-site structure takes the fused kernels
    x = embed_in_keys(dth, op.keys)
    y = op.apply(x.data)
    torch.cuda.synchronize()
    assert op._batch.device_error() == 0
    got = SymmetricTensor.from_flat(dth.indices, op.keys, y).numpy_blocks()
    ref = unpack_tensor(z, "heff.out").blocks
    for k in got:
        if k not in ref:
            assert np.all(got[k] == 0.0), k
    assert rel_err({k: v for k, v in got.items() if k in ref}, ref) < tol


def _random_problem(chi, seed, n_sectors=12, hi=64, cylinder=True, lo=4):
    from tenax_b200 import workloads as W

    Wl, Wr = W.cylinder_bulk_w() if cylinder else W.chain_bulk_w()
    gen = np.random.default_rng(seed)
    return W.make_heff_problem(chi, chi, Wl, Wr, gen, n_sectors=n_sectors, hi=hi, lo=lo)


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("bf16x3", 2e-5)])
def test_fused_heff_random_multi_tile(precision, tol):
    # sectors up to 64 wide with Dw=26: stage-1 M spans several 128-row tiles
    p = _random_problem(300, 5, n_sectors=12, hi=64)
    op = tb.HeffOperator(p.L, p.Wl, p.Wr, p.R, p.theta.indices, p.theta.keys, precision)
    x = embed_in_keys(p.theta, op.keys)
    y = op.apply(x.data)
    torch.cuda.synchronize()
    assert op._batch.device_error() == 0
    got = SymmetricTensor.from_flat(p.theta.indices, op.keys, y).numpy_blocks()
    ref = o_blockwise([to_host(t) for t in (p.L, x, p.Wl, p.Wr, p.R)], "abc,apqd,bpse,eqtf,dfg->cstg").blocks
    assert rel_err(got, ref) < tol


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("bf16x3", 2e-5)])
@pytest.mark.parametrize("shape", ["tiny_sectors", "wide_sectors"])
def test_fused_heff_sector_extremes(shape, precision, tol):
    """Sectors of extent 1-6 (every tile mostly padding; K below one MMA step)
    and sectors up to 320 wide (several K slabs in stage 1, two N tiles)
    against the oracle's per-combination H_eff."""
    if shape == "tiny_sectors":
        p = _random_problem(30, 9, n_sectors=12, hi=6, lo=1)
    else:
        p = _random_problem(1400, 10, n_sectors=8, hi=320, cylinder=False)
    op = tb.HeffOperator(p.L, p.Wl, p.Wr, p.R, p.theta.indices, p.theta.keys, precision)
    x = embed_in_keys(p.theta, op.keys)
    y = op.apply(x.data)
    torch.cuda.synchronize()
    assert op._batch.device_error() == 0
    got = SymmetricTensor.from_flat(p.theta.indices, op.keys, y).numpy_blocks()
    ref = o_blockwise([to_host(t) for t in (p.L, x, p.Wl, p.Wr, p.R)], "abc,apqd,bpse,eqtf,dfg->cstg").blocks
    for k in got:
        if k not in ref:
            assert np.all(got[k] == 0.0), k
    assert rel_err({k: v for k, v in got.items() if k in ref}, ref) < tol


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("bf16x3", 2e-5)])
def test_heff_z3(precision, tol):
    """H_eff on Z3 charges: random charge-conserving operands with the
    two-site problem's legs and flows (L, theta, W_l, W_r, R), against the
    oracle's per-combination H_eff (blocks match by charge value,
    dmrg.py:1094-1136).  Such structures may have stage-4 groups that write
    several output charges; the operator then takes the general contraction
    path, and Lanczos on it must still reach the oracle's eigenvalue."""
    from oracle.blocksparse import random_tensor

    u = _random_problem(40, 12, n_sectors=6, hi=12, cylinder=False)
    rng = np.random.default_rng(12)
    bond = np.array([0] * 5 + [1] * 7 + [2] * 6, np.int32)
    mpo = np.array([0, 1, 2, 0, 1], np.int32)
    phys = np.array([0, 2], np.int32)
    charges = {"vl": bond, "vl_c": bond, "vr": bond, "vr_c": bond, "wl": mpo, "wr": mpo, "p1": phys, "p2": phys}

    def z3_like(t, leg_charges):
        legs = tuple(Leg(leg_charges[i], int(ix.flow), ix.label) for i, ix in enumerate(t.indices))
        return random_tensor(legs, rng, 3, 0)

    L = z3_like(u.L, [charges[i.label] for i in u.L.indices])
    R = z3_like(u.R, [charges[i.label] for i in u.R.indices])
    th = z3_like(u.theta, [charges[i.label] for i in u.theta.indices])
    # W_l (b, p, s, e) and W_r (e, q, t, f): MPO legs carry mpo charges, physical legs phys charges
    Wl = z3_like(u.Wl, [mpo, phys, phys, mpo])
    Wr = z3_like(u.Wr, [mpo, phys, phys, mpo])
    dL, dth, dWl, dWr, dR = map(to_dev, (L, th, Wl, Wr, R))
    op = tb.HeffOperator(dL, dWl, dWr, dR, dth.indices, dth.keys, precision)
    # this structure has stage-4 groups writing several output charges: it
    # must take the general path, or the fallback goes untested
    assert not op.fused
    x = embed_in_keys(dth, op.keys)
    y = op.apply(x.data)
    torch.cuda.synchronize()
    assert op.device_error() == 0
    got = SymmetricTensor.from_flat(dth.indices, op.keys, y).numpy_blocks()
    ref = o_blockwise([L, to_host(x), Wl, Wr, R], "abc,apqd,bpse,eqtf,dfg->cstg").blocks
    assert ref
    for k in got:
        if k not in ref:
            assert np.all(got[k] == 0.0), k
    assert rel_err({k: v for k, v in got.items() if k in ref}, ref) < tol
    if precision == "fp64":
        from tenax_b200 import dmrg as gd

        e, _, _ = gd.lanczos(op, dth, 8, 1e-12)
        e_ref = odmrg.lanczos(lambda v: odmrg.heff_matvec(L, v, Wl, Wr, R), th, 8, 1e-12)[0]
        assert abs(e - float(e_ref)) <= 1e-9 * max(1.0, abs(float(e_ref)))


def test_batch_equals_individual():
    probs = [_random_problem(c, s, n_sectors=10, hi=48) for c, s in ((120, 1), (200, 2), (160, 3))]
    ops = [tb.HeffOperator(p.L, p.Wl, p.Wr, p.R, p.theta.indices, p.theta.keys, "fp64") for p in probs]
    xs = [embed_in_keys(p.theta, o.keys).data for p, o in zip(probs, ops)]
    singles = [o.apply(x) for o, x in zip(ops, xs)]
    batch = tb.HeffBatch(ops)
    outs = [o.out_like() for o in ops]
    batch.apply(xs, outs)
    torch.cuda.synchronize()
    for a, b in zip(singles, outs):
        torch.testing.assert_close(a, b, rtol=0, atol=0)


@pytest.mark.parametrize("precision", ["fp64", "bf16x3"])
def test_batch_host_streaming_equals_device_apply(precision):
    """tnx_heff_batch_apply_host: five independent steps streamed from pinned
    host memory (copies overlapped with compute on their own streams) give
    bit-for-bit the outputs of device-resident applies of the same inputs."""
    probs = [_random_problem(c, s, n_sectors=10, hi=48) for c, s in ((120, 1), (200, 2), (160, 3))]
    ops = [tb.HeffOperator(p.L, p.Wl, p.Wr, p.R, p.theta.indices, p.theta.keys, precision) for p in probs]
    batch = tb.HeffBatch(ops)
    assert batch.total == sum(o.size for o in ops)
    assert list(batch.offsets) == list(np.cumsum([0] + [o.size for o in ops])[:-1])
    rng = np.random.default_rng(7)
    steps = 5
    h_in = [torch.from_numpy(rng.standard_normal(batch.total)).pin_memory() for _ in range(steps)]
    h_out = [torch.full((batch.total,), np.nan, dtype=torch.float64).pin_memory() for _ in range(steps)]
    batch.apply_host(h_in, h_out)
    torch.cuda.synchronize()
    for s in range(steps):
        x = h_in[s].cuda()
        y = torch.empty_like(x)
        xs = [x[o:o + op.size] for o, op in zip(batch.offsets, ops)]
        ys = [y[o:o + op.size] for o, op in zip(batch.offsets, ops)]
        batch.apply(xs, ys)
        torch.cuda.synchronize()
        torch.testing.assert_close(h_out[s], y.cpu(), rtol=0, atol=0)
    assert batch.device_error() == 0
    with pytest.raises(ValueError):
        batch.apply_host(h_in[:1], [torch.empty(3, dtype=torch.float64)])


def test_vector_primitives():
    from tenax_b200 import vector

    x = torch.randn(1_000_003, dtype=torch.float64, device="cuda")
    y = torch.randn(1_000_003, dtype=torch.float64, device="cuda")
    d = float(vector.dot(x, y))
    n = float(vector.nrm2(x))
    assert abs(d - float(torch.dot(x, y))) < 1e-9 * max(1.0, abs(d))
    assert abs(n - float(torch.linalg.norm(x))) < 1e-12 * n


@pytest.mark.parametrize("steps", [1, 2, 3])
def test_batch_host_streaming_short_runs(steps):
    """The streamed apply's pipeline edges: with 1, 2 or 3 steps the copy-in
    of step s+1 and copy-out of step s-1 have nothing (or one step) to overlap
    with; every output still equals the device-resident apply bit for bit."""
    probs = [_random_problem(c, s, n_sectors=8, hi=40) for c, s in ((96, 4), (140, 5))]
    ops = [tb.HeffOperator(p.L, p.Wl, p.Wr, p.R, p.theta.indices, p.theta.keys, "bf16x3") for p in probs]
    batch = tb.HeffBatch(ops)
    rng = np.random.default_rng(11 + steps)
    h_in = [torch.from_numpy(rng.standard_normal(batch.total)).pin_memory() for _ in range(steps)]
    h_out = [torch.full((batch.total,), np.nan, dtype=torch.float64).pin_memory() for _ in range(steps)]
    batch.apply_host(h_in, h_out)
    torch.cuda.synchronize()
    for s in range(steps):
        x = h_in[s].cuda()
        y = torch.empty_like(x)
        batch.apply([x[o:o + op.size] for o, op in zip(batch.offsets, ops)],
                    [y[o:o + op.size] for o, op in zip(batch.offsets, ops)])
        torch.cuda.synchronize()
        torch.testing.assert_close(h_out[s], y.cpu(), rtol=0, atol=0)
    assert batch.device_error() == 0
