"""Fermionic symmetries on the GPU engine against the reference's own
outputs (tests/golden/fermion.*): label contractions carry the exchange sign
of the leg reordering (contraction/contractor.py:206-285, :460-470),
transposes the Koszul sign (core/tensor.py:32-50, :836-862) and daggers the
twist phase (core/tensor.py:795-820), for FermionParity and FermionicU1.
Keys exact, FP64 values at rtol 1e-12; split-BF16x3 contractions within 2e-5
relative Frobenius error."""

import json
import os

import numpy as np
import pytest

from fixture_io import unpack_tensor

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a CUDA device", allow_module_level=True)

import tenax_b200 as tb  # noqa: E402
from tenax_b200.core import FermionicU1, FermionParity, FlowDirection, TensorIndex  # noqa: E402
from tenax_b200.tensor import SymmetricTensor  # noqa: E402


def _cases(golden_dir):
    return json.load(open(os.path.join(golden_dir, "fermion.json")))


def _dev(z, name, sym):
    t = unpack_tensor(z, name)
    idx = tuple(TensorIndex(sym, l.charges, FlowDirection(l.flow), l.label) for l in t.legs)
    return SymmetricTensor(t.blocks, idx, _validate=False), t


def _sym(c):
    return FermionParity() if c["symmetry"] == "fermion_parity" else FermionicU1()


def _assert_blocks(got: dict, ref: dict, name, rtol=1e-12):
    assert sorted(got) == sorted(ref), name
    for k in got:
        np.testing.assert_allclose(got[k], ref[k], rtol=rtol, atol=1e-13, err_msg=f"{name} {k}")


def test_fermion_contractions_match_reference(golden_dir):
    z = np.load(os.path.join(golden_dir, "fermion.npz"))
    n = 0
    for c in _cases(golden_dir):
        if c["kind"] != "contract":
            continue
        sym = _sym(c)
        ins = [_dev(z, f"{c['name']}.in{i}", sym)[0] for i in range(c["n_in"])]
        ref = unpack_tensor(z, f"{c['name']}.out")
        out = tb.contract_with_subscripts(ins, c["subscripts"], None)
        _assert_blocks(out.numpy_blocks(), ref.blocks, c["name"])
        # the label API gives the same tensor
        via_labels = tb.contract(*ins, output_labels=c["output_labels"])
        _assert_blocks(via_labels.numpy_blocks(), ref.blocks, c["name"] + " (labels)")
        n += 1
    assert n == 10


def test_fermion_contraction_mixed_precision(golden_dir):
    z = np.load(os.path.join(golden_dir, "fermion.npz"))
    for c in _cases(golden_dir):
        if c["kind"] != "contract":
            continue
        ins = [_dev(z, f"{c['name']}.in{i}", _sym(c))[0] for i in range(c["n_in"])]
        ref = unpack_tensor(z, f"{c['name']}.out").blocks
        got = tb.contract_with_subscripts(ins, c["subscripts"], None, precision="bf16x3").numpy_blocks()
        num = sum(float(np.sum((got[k] - ref[k]) ** 2)) for k in ref)
        den = sum(float(np.sum(v * v)) for v in ref.values())
        assert sorted(got) == sorted(ref) and np.sqrt(num / den) < 2e-5, c["name"]


def test_fermion_transpose_and_dagger_match_reference(golden_dir):
    z = np.load(os.path.join(golden_dir, "fermion.npz"))
    kinds = set()
    for c in _cases(golden_dir):
        if c["kind"] == "contract":
            continue
        t, _ = _dev(z, f"{c['name']}.in0", _sym(c))
        ref = unpack_tensor(z, f"{c['name']}.out")
        out = t.transpose(tuple(c["axes"])) if c["kind"] == "transpose" else t.dagger()
        _assert_blocks(out.numpy_blocks(), ref.blocks, c["name"])
        for got_leg, ref_leg in zip(out.indices, ref.legs):
            np.testing.assert_array_equal(got_leg.charges, ref_leg.charges)
            assert int(got_leg.flow) == int(ref_leg.flow)
        kinds.add(c["kind"])
    assert kinds == {"transpose", "dagger"}


def test_fermion_custom_grading_is_rejected():
    sym = FermionicU1(grading=lambda q: int(q) % 3 == 1)
    q = np.array([0, 1, -1], np.int32)
    a = SymmetricTensor.random_normal((TensorIndex(sym, q, FlowDirection.IN, "i"),
                                       TensorIndex(sym, q, FlowDirection.OUT, "j")), key=3)
    b = SymmetricTensor.random_normal((TensorIndex(sym, q, FlowDirection.IN, "j"),
                                       TensorIndex(sym, q, FlowDirection.OUT, "k")), key=4)
    with pytest.raises(NotImplementedError):
        tb.contract(a, b)
