"""The block-sparse CTMRG oracle against the reference's own outputs
(tests/golden/ctm_tensor.npz, written by make_golden.py from
algorithms/_ctm_tensor.py)."""

import json
import os

import numpy as np
import pytest

from oracle import ctm_tensor as oc
from oracle.blocksparse import todense
from tests.golden.fixture_io import unpack_tensor

HERE = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module")
def gold():
    z = np.load(os.path.join(HERE, "ctm_tensor.npz"))
    with open(os.path.join(HERE, "ctm_tensor.json")) as fh:
        meta = json.load(fh)
    return z, meta


def _cases(meta, with_error=False):
    return [n for n, m in meta.items() if "bond_charges" in m and (("error" in m) == with_error)]


def _projectors(z, name, n):
    return [z[f"{name}.P{i}"] for i in range(n)]


def _check_env(z, name, env, dense, atol=1e-10):
    for f in oc.FIELDS:
        if dense:
            np.testing.assert_allclose(todense(env[f]), z[f"{name}.{f}"], atol=atol, rtol=0, err_msg=f)
            continue
        ref = unpack_tensor(z, f"{name}.{f}")
        assert sorted(env[f].blocks) == sorted(ref.blocks), f"{name}.{f}: block keys differ"
        assert [l.label for l in env[f].legs] == [l.label for l in ref.legs]
        for lg, lr in zip(env[f].legs, ref.legs):
            assert lg.flow == lr.flow
            np.testing.assert_array_equal(lg.charges, lr.charges)
        for k, blk in ref.blocks.items():
            np.testing.assert_allclose(env[f].blocks[k], blk, atol=atol, rtol=0, err_msg=f"{name}.{f}{k}")


def test_replay_matches_reference(gold):
    z, meta = gold
    H = z["H"]
    for name in _cases(meta):
        m = meta[name]
        A = unpack_tensor(z, f"{name}.A")
        Ps = _projectors(z, name, 4 * m["iters"])
        env = oc.ctm_tensor(A, m["chi"], m["iters"], 0.0, True, m["method"], m["warmup"], m["dense"], Ps)
        _check_env(z, name, env, m["dense"])
        assert abs(oc.energy(A, env, H, 2) - m["energy"]) < 1e-10, name


def test_free_run_projectors_match_reference(gold):
    """Without replay the oracle computes the reference's projectors: the
    kept subspace P P^T agrees with the reference's until the first cut
    through a degenerate eigenvalue cluster, after which both runs follow
    their own (equally valid) choice -- the reference's CTM is not a smooth
    function of its input, which is why parity is pinned by replay."""
    z, meta = gold
    for name in _cases(meta):
        m = meta[name]
        A = unpack_tensor(z, f"{name}.A")
        rec = []
        env = oc.ctm_tensor(A, m["chi"], m["iters"], 0.0, True, m["method"], m["warmup"], m["dense"], rec=rec)
        ref = _projectors(z, name, 4 * m["iters"])
        assert len(rec) == len(ref)
        agree = [P.shape == R.shape and np.abs(P @ P.T - R @ R.T).max() < 1e-8 for P, R in zip(rec, ref)]
        assert agree[0] and agree[1], name  # the first moves start from the identity environment
        if name.startswith(("u1", "z2")):
            assert oc.energy(A, env, z["H"], 2) == m["energy"] == 0.0  # the reference's symmetric runs give 0


def test_error_case_matches_reference(gold):
    z, meta = gold
    for name in _cases(meta, with_error=True):
        m = meta[name]
        A = unpack_tensor(z, f"{name}.A")
        with pytest.raises(ValueError) as ei:
            oc.ctm_tensor(A, m["chi"], m["iters"], 0.0, True, m["method"], m["warmup"], m["dense"])
        assert str(ei.value) == m["error"]


def test_checkerboard_replay_matches_reference(gold):
    z, meta = gold
    name = "cb_d2_chi6"
    m = meta[name]
    A, B = unpack_tensor(z, f"{name}.A"), unpack_tensor(z, f"{name}.B")
    Ps = _projectors(z, name, 8 * m["iters"])
    envs = oc.ctm_tensor_multisite({(0, 0): A, (1, 0): B}, oc.CHECKERBOARD, m["chi"], m["iters"], 0.0,
                                   projectors=Ps)
    for s, c in (("A", (0, 0)), ("B", (1, 0))):
        for f in oc.FIELDS:
            ref = unpack_tensor(z, f"{name}.env{s}.{f}")
            assert sorted(envs[c][f].blocks) == sorted(ref.blocks)
            np.testing.assert_allclose(todense(envs[c][f]), todense(ref), atol=1e-10, rtol=0)
    E = oc.energy_2site(A, B, envs[(0, 0)], envs[(1, 0)], z["H"], 2)
    assert abs(E - m["energy"]) < 1e-10


def test_invalid_projector_method_raises(gold):
    z, meta = gold
    A = unpack_tensor(z, "triv_d2_chi6.A")
    with pytest.raises(ValueError, match="Unknown projector_method"):
        oc.ctm_tensor(A, 4, 1, method="invalid")
