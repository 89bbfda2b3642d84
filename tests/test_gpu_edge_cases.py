"""Edge cases of the block-sparse contraction on the GPU, each checked
against the oracle's restatement of the reference's filtered contraction
(contractor.py:291-484) on the same inputs: an operand with no blocks,
contracted charges that never meet, blocks of extent 1, sectors several
hundred wide (multi-tile M, N and K), Z_n charges, and the mixed-precision
generic contraction path (split-BF16x3 at 2e-5, TF32 at 5e-3 relative
Frobenius error against FP64, whose blocks match the oracle to 1e-12)."""

import numpy as np
import pytest

from oracle.blocksparse import Leg, OTensor, contract_symmetric, labels_to_subscripts, random_tensor

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a CUDA device", allow_module_level=True)

import tenax_b200 as tb  # noqa: E402
from tenax_b200.core import FlowDirection, TensorIndex, U1Symmetry, ZnSymmetry  # noqa: E402
from tenax_b200.tensor import SymmetricTensor  # noqa: E402


def to_dev(t: OTensor) -> SymmetricTensor:
    sym = U1Symmetry() if t.modulus is None else ZnSymmetry(t.modulus)
    idx = tuple(TensorIndex(sym, l.charges, FlowDirection(l.flow), l.label) for l in t.legs)
    return SymmetricTensor(t.blocks, idx, _validate=False)


def oracle(a: OTensor, b: OTensor) -> OTensor:
    subs, _ = labels_to_subscripts([a, b])
    return contract_symmetric([a, b], subs)[0]


def check(a: OTensor, b: OTensor, precision="fp64"):
    ref = oracle(a, b)
    got = tb.contract(to_dev(a), to_dev(b), precision=precision)
    assert [str(x) for x in got.labels()] == [l.label for l in ref.legs]
    assert got.keys == ref.sorted_keys()
    host = got.numpy_blocks()
    for k, blk in ref.blocks.items():
        den = max(float(np.linalg.norm(blk)), 1e-300)
        assert float(np.linalg.norm(host[k] - blk)) / den < 1e-12, k
    return got, ref


def legs(charges_flows_labels):
    return tuple(Leg(np.asarray(c, np.int32), f, lab) for c, f, lab in charges_flows_labels)


def test_operand_without_blocks():
    a = OTensor(legs([([0, 1], 1, "i"), ([0, 1], -1, "j")]), {}, None)
    b = random_tensor(legs([([0, 1], 1, "j"), ([0, 1], -1, "k")]), np.random.default_rng(1))
    got, ref = check(a, b)
    assert got.n_blocks == 0 and not ref.blocks


def test_contracted_charges_never_meet():
    rng = np.random.default_rng(2)
    a = random_tensor(legs([([3, 4], 1, "i"), ([3, 4], -1, "j")]), rng)
    b = random_tensor(legs([([-2, -1], 1, "j"), ([-2, -1], -1, "k")]), rng)
    got, _ = check(a, b)
    assert got.n_blocks == 0


def test_unit_extent_blocks():
    rng = np.random.default_rng(3)
    q = list(range(-6, 7))  # every charge once: all blocks 1 x 1 (x 1)
    a = random_tensor(legs([(q, 1, "i"), ([1, -1], 1, "p"), (q, -1, "j")]), rng)
    b = random_tensor(legs([(q, 1, "j"), ([1, -1], 1, "s"), (q, -1, "k")]), rng)
    got, _ = check(a, b)
    assert got.n_blocks > 20


def _wide_pair(rng, sizes, modulus=None):
    q = np.concatenate([np.full(n, c, np.int32) for c, n in sizes])
    a = random_tensor(legs([(q, 1, "i"), ([0, 1], 1, "p"), (q, -1, "j")]), rng, modulus)
    b = random_tensor(legs([(q, 1, "j"), ([0, 1], -1, "s"), (q, -1, "k")]), rng, modulus)
    return a, b


def test_wide_sectors_multi_tile():
    # sectors of 300..700 states: several 64/128-row image tiles in M, N and K
    a, b = _wide_pair(np.random.default_rng(4), [(0, 700), (1, 300), (2, 450)])
    check(a, b)


def test_zn_charges():
    a, b = _wide_pair(np.random.default_rng(5), [(0, 90), (1, 130), (2, 70)], modulus=3)
    check(a, b)


@pytest.mark.parametrize("precision,tol", [("bf16x3", 2e-5), ("tf32", 5e-3)])
def test_mixed_precision_generic_path(precision, tol):
    a, b = _wide_pair(np.random.default_rng(6), [(0, 260), (1, 190), (-1, 75)])
    ref = tb.contract(to_dev(a), to_dev(b), precision="fp64")
    got = tb.contract(to_dev(a), to_dev(b), precision=precision)
    assert got.keys == ref.keys
    err = float(torch.linalg.norm(got.data - ref.data) / torch.linalg.norm(ref.data))
    assert err < tol, err
