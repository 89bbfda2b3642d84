"""The device SymmetricTensor's block arithmetic against the oracle's
restatement of core/tensor.py: inner over common keys (:296-319), norm
(:863-868), scalar multiply (:923-928), key-union addition (:933-952),
transpose (:832-861), from_dense / todense (:670-781) and their errors.

Bars: keys exact; element-wise results (add, scale, transpose, dense round
trip) bit-exact, since each is one IEEE operation or a copy; the FP64
reductions (inner, norm) within 1e-13 relative."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a CUDA device", allow_module_level=True)

from oracle.blocksparse import Leg, OTensor, inner as o_inner, norm as o_norm, random_tensor, t_add, t_scale  # noqa: E402,E501
from oracle.blocksparse import todense  # noqa: E402
from tenax_b200.core import FlowDirection, TensorIndex, U1Symmetry, ZnSymmetry  # noqa: E402
from tenax_b200.tensor import SymmetricTensor, inner  # noqa: E402

CASES = {
    "u1": (None, [np.array([-1, 0, 0, 1, 2]), np.array([0, 1, 1, -1]), np.array([-2, 0, 1, 1, 0, 2])], [1, 1, -1]),
    "z3": (3, [np.array([0, 1, 2, 2]), np.array([1, 0, 2]), np.array([0, 0, 1, 2]), np.array([2, 1])],
           [1, -1, 1, -1]),
}


def _pair(name, seed):
    mod, charges, flows = CASES[name]
    legs = tuple(Leg(c.astype(np.int32), f, f"l{i}") for i, (c, f) in enumerate(zip(charges, flows)))
    rng = np.random.default_rng(seed)
    a = random_tensor(legs, rng, mod, 0)
    b = random_tensor(legs, rng, mod, 0)
    keys = sorted(b.blocks)
    for k in keys[::3]:  # b misses a third of the keys: partial overlap for inner / add
        del b.blocks[k]
    return a, b


def _dev(t: OTensor) -> SymmetricTensor:
    sym = U1Symmetry() if t.modulus is None else ZnSymmetry(t.modulus)
    idx = tuple(TensorIndex(sym, l.charges, FlowDirection(l.flow), l.label) for l in t.legs)
    return SymmetricTensor(t.blocks, idx, _validate=False)


def _same(got: SymmetricTensor, ref: OTensor):
    assert sorted(got.keys) == sorted(ref.blocks)
    host = got.numpy_blocks()
    for k, v in ref.blocks.items():
        np.testing.assert_array_equal(host[k], v)


@pytest.mark.parametrize("name", sorted(CASES))
def test_inner_norm_scale_add(name):
    a, b = _pair(name, 3)
    da, db = _dev(a), _dev(b)
    assert abs(float(inner(da, db)) - o_inner(a, b)) <= 1e-13 * max(1.0, abs(o_inner(a, b)))
    assert abs(float(da.norm()) - o_norm(a)) <= 1e-13 * o_norm(a)
    _same(da * 2.5, t_scale(a, 2.5))
    _same(da + db, t_add(a, b))
    _same(db + da, t_add(b, a))
    _same(da - db, t_add(a, t_scale(b, -1.0)))


@pytest.mark.parametrize("name", sorted(CASES))
def test_transpose_and_dense_round_trip(name):
    a, _ = _pair(name, 5)
    da = _dev(a)
    n = len(a.legs)
    perm = tuple(reversed(range(n)))
    dt = da.transpose(perm)
    assert dt.labels() == tuple(a.legs[i].label for i in perm)
    np.testing.assert_array_equal(dt.todense().cpu().numpy(), np.transpose(todense(a), perm))
    dense = todense(a)
    back = SymmetricTensor.from_dense(dense, da.indices)
    # from_dense keeps every valid key with basis states (zero blocks included)
    for k, v in back.numpy_blocks().items():
        np.testing.assert_array_equal(v, a.blocks.get(k, np.zeros_like(v)))
    back_dev = SymmetricTensor.from_dense(torch.as_tensor(dense, device="cuda"), da.indices)
    assert back_dev.keys == back.keys
    torch.testing.assert_close(back_dev.data, back.data, rtol=0, atol=0)


def test_errors():
    a, _ = _pair("u1", 7)
    da = _dev(a)
    dense = todense(a)
    # an entry outside every allowed sector
    mask = np.ones(dense.shape, bool)
    for k in a.blocks:
        pos = [np.where(l.charges == q)[0] for l, q in zip(a.legs, k)]
        mask[np.ix_(*pos)] = False
    bad = dense.copy()
    bad[tuple(np.argwhere(mask)[0])] = 1.0
    with pytest.raises(ValueError, match="outside symmetry-allowed sectors"):
        SymmetricTensor.from_dense(bad, da.indices)
    with pytest.raises(ValueError):
        SymmetricTensor.from_dense(dense[:-1], da.indices)
    with pytest.raises(TypeError):
        da + 1.0
