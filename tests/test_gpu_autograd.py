"""Adjoint of the block-sparse contraction (tenax_b200.contract_ad) against
torch autograd of the same contraction on the dense forms, restricted to
each operand's stored blocks (relative 1e-12), on the reference's golden
contraction cases (U(1) and Z_3)."""

import json
import os

import numpy as np
import pytest

from fixture_io import unpack_tensor

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a CUDA device", allow_module_level=True)

from oracle.blocksparse import todense  # noqa: E402
from tenax_b200 import contract_ad  # noqa: E402
from tenax_b200.contraction import _labels_to_subscripts  # noqa: E402
from tenax_b200.core import FlowDirection, TensorIndex, U1Symmetry, ZnSymmetry  # noqa: E402
from tenax_b200.tensor import SymmetricTensor  # noqa: E402


def to_dev(t):
    sym = U1Symmetry() if t.modulus is None else ZnSymmetry(t.modulus)
    idx = tuple(TensorIndex(sym, l.charges, FlowDirection(l.flow), l.label) for l in t.legs)
    return SymmetricTensor(t.blocks, idx, _validate=False)


def blocks_of(dense, t: SymmetricTensor):
    """Dense array restricted to t's stored blocks, in t's flat layout."""
    parts = []
    for k in t.keys:
        pos = [np.nonzero(i.charges == q)[0] for i, q in zip(t.indices, k)]
        parts.append(dense[np.ix_(*pos)].ravel())
    return np.concatenate(parts) if parts else np.zeros(0)


@pytest.mark.parametrize("name", ["pair_u1", "pair_u1_perm", "mps_pair", "two_legs", "z3_pair", "outer_free"])
def test_contract_adjoint_matches_dense_autograd(golden_dir, name):
    z = np.load(os.path.join(golden_dir, "contract.npz"))
    cases = {c["name"]: c for c in json.load(open(os.path.join(golden_dir, "contract.json")))}
    c = cases[name]
    ot = [unpack_tensor(z, f"{name}.in{i}") for i in range(2)]
    a, b = (to_dev(t) for t in ot)
    a_data = a.data.clone().requires_grad_(True)
    b_data = b.data.clone().requires_grad_(True)
    a = SymmetricTensor.from_flat(a.indices, a.keys, a_data)
    b = SymmetricTensor.from_flat(b.indices, b.keys, b_data)
    out = contract_ad(a, b, output_labels=c["output_labels"])
    w = torch.from_numpy(np.random.default_rng(3).standard_normal(out.data.shape[0])).cuda()
    ga, gb = torch.autograd.grad((out.data * w).sum(), (a_data, b_data))
    # dense reference
    subs, _ = _labels_to_subscripts((a, b), c["output_labels"])
    Ad = torch.from_numpy(todense(ot[0])).requires_grad_(True)
    Bd = torch.from_numpy(todense(ot[1])).requires_grad_(True)
    Cd = torch.einsum(subs, Ad, Bd)
    Wd = SymmetricTensor.from_flat(out.indices, out.keys, w).todense().cpu()
    gad, gbd = torch.autograd.grad((Cd * Wd).sum(), (Ad, Bd))
    ra = blocks_of(gad.numpy(), a)
    rb = blocks_of(gbd.numpy(), b)
    assert np.abs(ga.cpu().numpy() - ra).max() <= 1e-12 * max(1.0, np.abs(ra).max())
    assert np.abs(gb.cpu().numpy() - rb).max() <= 1e-12 * max(1.0, np.abs(rb).max())
