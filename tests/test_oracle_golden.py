"""Pin the oracle (NumPy restatement) to the reference's own outputs.

The fixtures were produced by executing the reference's source under a NumPy
stand-in for jax (tests/golden/make_golden.py).
"""

import json
import os

import numpy as np
import pytest

from fixture_io import unpack_tensor
from oracle.blocksparse import blockwise_contract, contract_symmetric, valid_blocks
from oracle import dmrg as odmrg


def assert_tensor_close(a, b, rtol=1e-12, atol=1e-13):
    assert sorted(a.blocks) == sorted(b.blocks)
    for k in a.blocks:
        np.testing.assert_allclose(a.blocks[k], b.blocks[k], rtol=rtol, atol=atol)


def test_valid_blocks_order(golden_dir):
    cases = json.load(open(os.path.join(golden_dir, "valid_blocks.json")))
    for c in cases:
        keys = valid_blocks(c["charges"], c["flows"], c["modulus"], c["target"])
        assert [list(k) for k in keys] == c["keys"], c["name"]


def test_contract_symmetric_cases(golden_dir):
    z = np.load(os.path.join(golden_dir, "contract.npz"))
    cases = json.load(open(os.path.join(golden_dir, "contract.json")))
    for c in cases:
        ins = [unpack_tensor(z, f"{c['name']}.in{i}") for i in range(c["n_in"])]
        ref = unpack_tensor(z, f"{c['name']}.out")
        out, _ = contract_symmetric(ins, c["subscripts"])
        assert len(out.blocks) == c["n_out_blocks"], c["name"]
        assert_tensor_close(out, ref)


def test_heff_env_lanczos_svd(golden_dir):
    z = np.load(os.path.join(golden_dir, "dmrg_pieces.npz"))
    L, th, Wl, Wr, R = (unpack_tensor(z, f"heff.{n}") for n in ("L", "theta", "Wl", "Wr", "R"))
    for t in (L, th, Wl, Wr, R):
        assert len(t.blocks) > 0, "fixture operands must be non-empty"
    out = odmrg.heff_matvec(L, th, Wl, Wr, R)
    assert len(out.blocks) > 0
    assert_tensor_close(out, unpack_tensor(z, "heff.out"))
    newL = odmrg.update_left_env(L, unpack_tensor(z, "envl.A"), Wl)
    assert_tensor_close(newL, unpack_tensor(z, "envl.out"))
    newR = odmrg.update_right_env(R, unpack_tensor(z, "envr.B"), Wr)
    assert_tensor_close(newR, unpack_tensor(z, "envr.out"))
    e, vec, _, _ = odmrg.lanczos(lambda v: odmrg.heff_matvec(L, v, Wl, Wr, R), th, 8, 1e-12)
    assert abs(e - float(z["lanczos.energy"])) < 1e-12
    ref_vec = unpack_tensor(z, "lanczos.vec")
    assert_tensor_close(vec, ref_vec, rtol=1e-9, atol=1e-11)
    U, s, Vh, err = odmrg.svd_and_truncate_site(ref_vec, 2, 5)
    np.testing.assert_allclose(s, z["svd.s"], rtol=1e-12)
    assert abs(err - float(z["svd.err"])) < 1e-12
    # gauge-invariant comparison: U s Vh products per key
    Ur, Vr = unpack_tensor(z, "svd.U"), unpack_tensor(z, "svd.Vh")
    assert sorted(U.blocks) == sorted(Ur.blocks) and sorted(Vh.blocks) == sorted(Vr.blocks)
    np.testing.assert_array_equal(U.legs[-1].charges, Ur.legs[-1].charges)


def test_auto_mpo_matches_reference(golden_dir):
    """The host MPO builder reproduces the reference's symmetric AutoMPO."""
    from tenax_b200.auto_mpo import heisenberg_chain_sites, heisenberg_cylinder_sites

    z = np.load(os.path.join(golden_dir, "mpo.npz"))
    for prefix, sites in (("cyl", heisenberg_cylinder_sites(3, 6)), ("chain", heisenberg_chain_sites(7))):
        for i, s in enumerate(sites):
            ref = unpack_tensor(z, f"{prefix}{i}")
            for leg, q in zip(ref.legs, s.charges):
                np.testing.assert_array_equal(leg.charges, q)
            blocks = s.blocks()
            assert sorted(blocks) == sorted(ref.blocks), (prefix, i)
            for k in blocks:
                np.testing.assert_array_equal(blocks[k], ref.blocks[k])


def test_oracle_dmrg_config1_energy(golden_dir):
    """Full config-1 DMRG (L=20, chi=64, 2 sweeps, 10 Lanczos steps) from the
    reference's own initial MPS: converged energy within 1e-9."""
    z = np.load(os.path.join(golden_dir, "dmrg_c1_L20.npz"))
    mps = [unpack_tensor(z, f"mps{i}") for i in range(20)]
    mpo = [unpack_tensor(z, f"mpo{i}") for i in range(20)]
    e, es, _, te = odmrg.dmrg(mpo, mps, 64, 2, lanczos_max_iter=10)
    assert abs(e - float(z["energy"])) <= 1e-9
    assert len(te) == len(z["truncation_errors"])
