"""GPU fuse_indices (tenax_b200.tensor_utils) against the reference's own
outputs: blocks and todense() bit-exact (fusion moves values only)."""

import json
import os

import numpy as np
import pytest

from fixture_io import unpack_tensor

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a CUDA device", allow_module_level=True)

from tenax_b200.core import FlowDirection, TensorIndex, U1Symmetry, ZnSymmetry  # noqa: E402
from tenax_b200.tensor import SymmetricTensor  # noqa: E402
from tenax_b200.tensor_utils import fuse_indices  # noqa: E402


def to_dev(t):
    sym = U1Symmetry() if t.modulus is None else ZnSymmetry(t.modulus)
    idx = tuple(TensorIndex(sym, l.charges, FlowDirection(l.flow), l.label) for l in t.legs)
    return SymmetricTensor(t.blocks, idx, _validate=False)


def test_fuse_matches_reference(golden_dir):
    z = np.load(os.path.join(golden_dir, "fuse.npz"))
    cases = json.load(open(os.path.join(golden_dir, "fuse.json")))
    for c in cases:
        ref = unpack_tensor(z, f"{c['name']}.out")
        for rep in range(2):
            out = fuse_indices(to_dev(unpack_tensor(z, f"{c['name']}.in")), c["axis_a"], c["axis_b"], "fused",
                               FlowDirection(c["fused_flow"]))
            assert out.keys == ref.sorted_keys(), c["name"]
            host = out.numpy_blocks()
            for k in ref.blocks:
                assert np.array_equal(host[k], ref.blocks[k]), (c["name"], k)
            assert np.array_equal(out.todense().cpu().numpy(), z[f"{c['name']}.out_dense"]), c["name"]
            assert out.labels()[min(c["axis_a"], c["axis_b"])] == "fused"
