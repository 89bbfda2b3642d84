"""Charge algebra and leg metadata (core/symmetry.py:41-87, :182-255;
core/index.py:43-130) on CPU: U(1) adds and negates; Z_n adds and negates
mod n, also for negative inputs; fuse_many folds left to right; a leg's dual
flips its flow and dualises its charges; the reference's error texts."""

import numpy as np
import pytest

from tenax_b200.core import FlowDirection, TensorIndex, U1Symmetry, ZnSymmetry


def test_u1_charge_algebra():
    u1 = U1Symmetry()
    a, b = np.array([-3, 0, 2], np.int32), np.array([1, -1, 5], np.int32)
    np.testing.assert_array_equal(u1.fuse(a, b), [-2, -1, 7])
    np.testing.assert_array_equal(u1.dual(a), [3, 0, -2])
    np.testing.assert_array_equal(u1.fuse_many([a, b, a]), [-5, -1, 9])
    assert u1.n_values() is None and u1.identity() == 0
    assert u1 == U1Symmetry() and hash(u1) == hash(U1Symmetry())


@pytest.mark.parametrize("n", [2, 3, 5])
def test_zn_charge_algebra(n):
    z = ZnSymmetry(n)
    a = np.arange(-n, 2 * n, dtype=np.int32)
    b = np.roll(a, 3)
    np.testing.assert_array_equal(z.fuse(a, b), (a + b) % n)
    np.testing.assert_array_equal(z.dual(a), (-a) % n)
    assert np.all((z.dual(a) >= 0) & (z.dual(a) < n))
    np.testing.assert_array_equal(z.fuse_many([a, b, a]), (2 * a + b) % n)
    assert z.n_values() == n
    assert z == ZnSymmetry(n) and z != ZnSymmetry(n + 1) and z != U1Symmetry()


def test_symmetry_errors():
    with pytest.raises(ValueError, match="n must be >= 2, got 1"):
        ZnSymmetry(1)
    with pytest.raises(ValueError, match="charge_list must be non-empty"):
        U1Symmetry().fuse_many([])


def test_tensor_index():
    z3 = ZnSymmetry(3)
    idx = TensorIndex(z3, np.array([0, 1, 2, 2], np.int64), FlowDirection.IN, "a")
    assert idx.charges.dtype == np.int32 and idx.dim == 4
    d = idx.dual()
    assert d.flow == FlowDirection.OUT and d.label == "a"
    np.testing.assert_array_equal(d.charges, [0, 2, 1, 1])
    f = idx.flip_flow()
    assert f.flow == FlowDirection.OUT
    np.testing.assert_array_equal(f.charges, idx.charges)
    assert idx.relabel("b").label == "b" and idx.relabel("b").flow == FlowDirection.IN
    assert idx.charge_dims() == {0: 1, 1: 1, 2: 2}
    u = TensorIndex(U1Symmetry(), [-2, 0, 3], FlowDirection.OUT, 7)
    np.testing.assert_array_equal(u.dual().charges, [2, 0, -3])
    assert u.dual().flow == FlowDirection.IN
    with pytest.raises(ValueError, match="charges must be 1-D"):
        TensorIndex(U1Symmetry(), np.zeros((2, 2), np.int32), FlowDirection.IN, "x")
