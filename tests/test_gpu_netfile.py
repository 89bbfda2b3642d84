"""NetworkBlueprint.launch() on the GPU against the reference's own results
(tests/golden/netfile.npz from network/netfile.py): blocks bit-for-bit in
structure and FP64 values to 1e-12, the reference's empty N-operand result
for a 3-chain without ORDER, and the pairwise flag's full contraction."""

import json
import os

import numpy as np
import pytest

from fixture_io import unpack_tensor

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a CUDA device", allow_module_level=True)

from tenax_b200 import netfile as nf  # noqa: E402
from tenax_b200.core import FlowDirection, TensorIndex, U1Symmetry  # noqa: E402
from tenax_b200.tensor import SymmetricTensor  # noqa: E402


def to_dev(t):
    idx = tuple(TensorIndex(U1Symmetry(), l.charges, FlowDirection(l.flow), l.label) for l in t.legs)
    return SymmetricTensor(t.blocks, idx, _validate=False)


@pytest.fixture(scope="module")
def fix(golden_dir):
    z = np.load(os.path.join(golden_dir, "netfile.npz"))
    with open(os.path.join(golden_dir, "netfile.json")) as fh:
        meta = json.load(fh)
    ins = {n: to_dev(unpack_tensor(z, f"in.{n}")) for n in ("A", "B", "C", "Bring")}
    return z, meta, ins


def _check(got, ref):
    assert [str(x) for x in got.labels()] == [l.label for l in ref.legs]
    assert got.keys == ref.sorted_keys()
    host = got.numpy_blocks()
    for k, blk in ref.blocks.items():
        np.testing.assert_allclose(host[k], blk, rtol=0, atol=1e-12 * max(1.0, float(np.abs(blk).max())))


SLOTS = {"pair": ("A", "B"), "chain3": ("A", "B", "C"), "chain3_order": ("A", "B", "C"),
         "chain3_order_right": ("A", "B", "C"), "ring_scalar": ("A", "Bring")}


@pytest.mark.parametrize("name", sorted(SLOTS))
def test_launch_matches_reference(fix, name):
    z, meta, ins = fix
    bp = nf.NetworkBlueprint(meta["parse"][name]["source"])
    bp.put_tensors(dict(zip(bp.tensor_names, [ins[s] for s in SLOTS[name]])))
    assert bp.is_ready()
    _check(bp.launch(), unpack_tensor(z, f"out.{name}"))


def test_label_order_and_transpose(fix):
    z, meta, ins = fix
    bp = nf.NetworkBlueprint(meta["parse"]["pair"]["source"])
    bp.put_tensor("A", ins["A"].relabels({"i": "x", "j": "y"}), label_order=["x", "y"])
    bp.put_tensor("B", ins["B"].transpose((1, 0)))
    _check(bp.launch(), unpack_tensor(z, "out.pair_label_order"))
    with pytest.raises(ValueError, match="don't match blueprint"):
        bp.put_tensor("A", ins["C"])


def test_pairwise_flag_contracts_the_chain(fix):
    z, meta, ins = fix
    bp = nf.NetworkBlueprint(meta["parse"]["chain3"]["source"])
    bp.put_tensors({"A": ins["A"], "B": ins["B"], "C": ins["C"]})
    assert bp.launch().n_blocks == 0  # the reference's filtered 3-operand contraction
    full = bp.launch(pairwise=True)
    _check(full, unpack_tensor(z, "out.chain3_order_right"))  # same labels (i, l), other association
    tn = bp.to_tensor_network()
    assert tn.n_nodes() == 3 and tn.n_edges() == 2
