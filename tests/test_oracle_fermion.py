"""The oracle's fermionic restatement against the reference's own outputs
(tests/golden/fermion.*, produced by executing the reference's source):
label contractions with the exchange sign of the leg reordering
(contraction/contractor.py:206-285, :460-470), transposes with the Koszul
sign (core/tensor.py:32-50, :836-862) and daggers with the twist phase
(core/tensor.py:795-820), for FermionParity and FermionicU1.  Values at
rtol 1e-12, keys exact."""

import json
import os

import numpy as np

from fixture_io import unpack_tensor
from oracle.blocksparse import contract_symmetric, dagger, transpose


def _load(golden_dir, name):
    t = unpack_tensor(np.load(os.path.join(golden_dir, "fermion.npz")), name)
    t.fermionic = True
    return t


def _close(got, ref, name):
    assert sorted(got.blocks) == sorted(ref.blocks), name
    for k in got.blocks:
        np.testing.assert_allclose(got.blocks[k], ref.blocks[k], rtol=1e-12, atol=1e-13, err_msg=f"{name} {k}")


def test_fermion_oracle_matches_reference(golden_dir):
    cases = json.load(open(os.path.join(golden_dir, "fermion.json")))
    kinds = set()
    for c in cases:
        ref = _load(golden_dir, f"{c['name']}.out")
        if c["kind"] == "contract":
            ins = [_load(golden_dir, f"{c['name']}.in{i}") for i in range(c["n_in"])]
            got, _ = contract_symmetric(ins, c["subscripts"])
        elif c["kind"] == "transpose":
            got = transpose(_load(golden_dir, f"{c['name']}.in0"), c["axes"])
        else:
            got = dagger(_load(golden_dir, f"{c['name']}.in0"))
            for lg, lr in zip(got.legs, ref.legs):
                np.testing.assert_array_equal(lg.charges, lr.charges)
                assert lg.flow == lr.flow
        _close(got, ref, c["name"])
        kinds.add(c["kind"])
    assert kinds == {"contract", "transpose", "dagger"}


def test_signs_are_not_trivial(golden_dir):
    """The fixtures exercise the sign: the same contraction without it
    differs from the reference on some block."""
    cases = [c for c in json.load(open(os.path.join(golden_dir, "fermion.json"))) if c["kind"] == "contract"]
    differs = 0
    for c in cases:
        ins = [_load(golden_dir, f"{c['name']}.in{i}") for i in range(c["n_in"])]
        for t in ins:
            t.fermionic = False
        got, _ = contract_symmetric(ins, c["subscripts"])
        ref = _load(golden_dir, f"{c['name']}.out")
        if any(not np.allclose(got.blocks[k], ref.blocks[k]) for k in ref.blocks):
            differs += 1
    assert differs >= len(cases) // 2
