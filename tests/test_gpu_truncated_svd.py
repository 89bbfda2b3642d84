"""GPU block-diagonal truncated SVD (tenax_b200.dmrg.truncated_svd on the
library's sector SVD batch) against the oracle's restatement of
linalg.py:75-333 on random two-site tensors.

Bars: the same kept count and bond charges in the same global order
(linalg.py:211, :242), the same U / Vh block keys, kept and full singular
values within 1e-12 of the largest, and the truncated tensor U s Vh within
1e-11 (relative Frobenius): singular vectors are compared only through it,
since their signs are the solver's choice.  Cases cover U(1) and Z2, a bond
cap, the max_truncation_err rule, both at once, normalisation (linalg.py:251)
and a sector wide enough (>= 128) to take the polar-decomposition driver."""

import zlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a CUDA device", allow_module_level=True)

from oracle.blocksparse import Leg, random_tensor, todense  # noqa: E402
from oracle import dmrg as odmrg  # noqa: E402
from tenax_b200 import dmrg as gd  # noqa: E402
from tenax_b200.core import FlowDirection, TensorIndex, U1Symmetry, ZnSymmetry  # noqa: E402
from tenax_b200.tensor import SymmetricTensor  # noqa: E402

IN, OUT = 1, -1


def _bond(charge_counts):
    return np.concatenate([np.full(n, q, np.int32) for q, n in charge_counts])


def _theta(case, rng):
    mod = case.get("modulus")
    vl, vr = _bond(case["left"]), _bond(case["right"])
    phys = np.array([1, -1] if mod is None else [0, 1], np.int32)
    legs = (Leg(vl, IN, "vl"), Leg(phys, IN, "p1"), Leg(phys, IN, "p2"), Leg(vr, OUT, "vr"))
    t = random_tensor(legs, rng, mod, 0)
    # a graded spectrum: scale each block so singular values spread over decades
    for k in list(t.blocks):
        t.blocks[k] = t.blocks[k] * 10.0 ** (-rng.uniform(0, 4))
    return t


def _to_dev(t):
    sym = U1Symmetry() if t.modulus is None else ZnSymmetry(t.modulus)
    idx = tuple(TensorIndex(sym, l.charges, FlowDirection(l.flow), l.label) for l in t.legs)
    return SymmetricTensor(t.blocks, idx, _validate=False)


CASES = {
    # physical charges are +-1, so vl and vr charges share their parity (vl + p1 + p2 = vr)
    "u1_cap": dict(left=[(-2, 6), (0, 10), (2, 5)], right=[(-2, 7), (0, 9), (2, 4)], max_sv=20),
    "u1_err": dict(left=[(-2, 6), (0, 10), (2, 5)], right=[(-2, 7), (0, 9), (2, 4)], max_err=1e-2),
    "u1_cap_err_norm": dict(left=[(-4, 3), (-2, 8), (0, 12), (2, 8), (4, 3)],
                            right=[(-4, 5), (-2, 11), (0, 13), (2, 11), (4, 5)], max_sv=37, max_err=1e-3,
                            normalize=True),
    "z2": dict(left=[(0, 9), (1, 13)], right=[(0, 11), (1, 8)], modulus=2, max_sv=25),
    # fused charge 1 has 160 rows and 160 columns: the polar-decomposition driver's range
    "u1_wide_sector": dict(left=[(0, 80), (2, 80)], right=[(0, 80), (2, 80)], max_sv=100),
}


def _widest_sector(case):
    """max over fused charges Q of min(rows, cols) of the (vl p1) x (p2 vr) sector matrix."""
    phys = (1, -1)
    rows, cols = {}, {}
    for q, n in case["left"]:
        for p in phys:
            rows[q + p] = rows.get(q + p, 0) + n
    for q, n in case["right"]:
        for p in phys:
            cols[q - p] = cols.get(q - p, 0) + n
    return max(min(rows[Q], cols.get(Q, 0)) for Q in rows)


@pytest.mark.parametrize("name", sorted(CASES))
def test_truncated_svd_matches_oracle(name):
    case = CASES[name]
    rng = np.random.default_rng(zlib.crc32(name.encode()))
    t = _theta(case, rng)
    kw = dict(max_sv=case.get("max_sv"), max_err=case.get("max_err"), normalize=case.get("normalize", False))
    U_o, s_o, V_o, sf_o = odmrg.truncated_svd(t, ["vl", "p1"], ["p2", "vr"], "bond", **kw)
    A, s, B, sf = gd.truncated_svd(_to_dev(t), ["vl", "p1"], ["p2", "vr"], "bond", kw["max_sv"], kw["max_err"],
                                   kw["normalize"], driver="native", n_streams=8)
    assert len(s) == len(s_o)
    np.testing.assert_array_equal(A.indices[-1].charges, U_o.legs[-1].charges)
    np.testing.assert_array_equal(B.indices[0].charges, V_o.legs[0].charges)
    assert sorted(A.keys) == sorted(U_o.blocks) and sorted(B.keys) == sorted(V_o.blocks)
    np.testing.assert_allclose(s, s_o, rtol=0, atol=1e-12 * s_o[0])
    np.testing.assert_allclose(sf, sf_o, rtol=0, atol=1e-12 * sf_o[0])
    if name == "u1_wide_sector":
        assert _widest_sector(case) >= gd.POLAR_MIN
    ref = np.einsum("lpb,b,bqr->lpqr", todense(U_o), s_o, todense(V_o))
    got = np.einsum("lpb,b,bqr->lpqr", A.todense().cpu().numpy(), s, B.todense().cpu().numpy())
    assert np.linalg.norm(got - ref) <= 1e-11 * np.linalg.norm(ref)
