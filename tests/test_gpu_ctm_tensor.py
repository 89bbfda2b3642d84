"""GPU block-sparse standard CTMRG (tenax_b200.ctm_tensor) against the
reference's own outputs (tests/golden/ctm_tensor.npz from
algorithms/_ctm_tensor.py) and the reference's own checks
(tests/test_ctm_tensor.py).

The reference CTM is not a smooth function of its input (degenerate
eigenvalue clusters are cut by the truncation), so values are pinned by
replaying the reference's recorded projectors: with them the block
structure must be identical (keys, charges, flows, labels) and the values
agree to 1e-10 in FP64."""

import json
import os

import numpy as np
import pytest

from fixture_io import unpack_tensor

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a CUDA device", allow_module_level=True)

from oracle import ctm_tensor as oc  # noqa: E402
from oracle.blocksparse import todense  # noqa: E402
from tenax_b200 import tensor_ctm as gc  # noqa: E402
from tenax_b200 import ipeps  # noqa: E402
from tenax_b200.core import FlowDirection, TensorIndex, U1Symmetry, ZnSymmetry  # noqa: E402
from tenax_b200.tensor import SymmetricTensor  # noqa: E402

FIELDS = ("C1", "C2", "C3", "C4", "T1", "T2", "T3", "T4")


def to_dev(t):
    sym = U1Symmetry() if t.modulus is None else ZnSymmetry(t.modulus)
    idx = tuple(TensorIndex(sym, l.charges, FlowDirection(l.flow), l.label) for l in t.legs)
    return SymmetricTensor(t.blocks, idx, _validate=False)


@pytest.fixture(scope="module")
def fix(golden_dir):
    z = np.load(os.path.join(golden_dir, "ctm_tensor.npz"))
    with open(os.path.join(golden_dir, "ctm_tensor.json")) as fh:
        return z, json.load(fh)


def _site(z, name, dense):
    A = unpack_tensor(z, f"{name}.A")
    return (todense(A) if dense else to_dev(A)), A


def _check(z, prefix, env, dense, atol=1e-10):
    for f in FIELDS:
        t = getattr(env, f)
        if dense:
            np.testing.assert_allclose(t.todense().cpu().numpy(), z[f"{prefix}.{f}"], atol=atol, rtol=0)
            continue
        ref = unpack_tensor(z, f"{prefix}.{f}")
        assert t.keys == ref.sorted_keys(), f"{prefix}.{f}: block structure differs"
        assert list(t.labels()) == [l.label for l in ref.legs]
        for i, l in zip(t.indices, ref.legs):
            assert int(i.flow) == l.flow
            np.testing.assert_array_equal(i.charges, l.charges)
        host = t.numpy_blocks()
        for k, blk in ref.blocks.items():
            np.testing.assert_allclose(host[k], blk, atol=atol, rtol=0, err_msg=f"{prefix}.{f}{k}")


CASES = ["triv_d2_chi6", "triv_d3_chi10", "triv_d2_chi5_qr", "dense_d2_chi6", "dense_d2_chi4_qr", "u1_d3_chi8",
         "z2_d3_chi6"]


@pytest.mark.parametrize("name", CASES)
def test_replay_matches_reference(fix, name):
    z, meta = fix
    m = meta[name]
    A, _ = _site(z, name, m["dense"])
    Ps = [z[f"{name}.P{i}"] for i in range(4 * m["iters"])]
    env = gc.ctm_tensor(A, m["chi"], m["iters"], 0.0, True, m["method"], m["warmup"], projectors=Ps)
    _check(z, name, env, m["dense"])
    E = float(gc.compute_energy_ctm_tensor(A, env, z["H"], 2))
    assert abs(E - m["energy"]) < 1e-10


@pytest.mark.parametrize("name", CASES)
def test_projectors_match_reference(fix, name):
    """Free run: the first projector has the reference's shape, orthonormal
    columns and captures the same weight tr(P^T rho P) of the first move's
    density matrix (the choice of vectors inside a degenerate eigenvalue
    cluster is the solver's own, so P itself is not compared)."""
    z, meta = fix
    m = meta[name]
    A, A_o = _site(z, name, m["dense"])
    rec = []
    env = gc.ctm_tensor(A, m["chi"], m["iters"], 0.0, True, m["method"], m["warmup"], record=rec)
    assert len(rec) == 4 * m["iters"]
    P, R = rec[0].cpu().numpy(), z[f"{name}.P0"]
    assert P.shape == R.shape
    np.testing.assert_allclose(P.T @ P, np.eye(P.shape[1]), atol=1e-10)
    env0 = oc.init_env(A_o, m["chi"], m["dense"])
    g1, g2, _ = oc.grow(env0, env0, oc.double_layer(A_o), "left")
    M = np.concatenate([todense(g1), todense(g2)], axis=1)
    rho = M @ M.T  # the QR branch diagonalises the same matrix through R R^T
    w_gpu, w_ref = np.trace(P.T @ rho @ P), np.trace(R.T @ rho @ R)
    assert abs(w_gpu - w_ref) <= 1e-10 * max(1.0, abs(w_ref))
    if not name.startswith(("triv", "dense")):
        assert float(gc.compute_energy_ctm_tensor(A, env, z["H"], 2)) == 0.0


def test_error_case_matches_reference(fix):
    z, meta = fix
    name = "u1_d2_chi6_err"
    m = meta[name]
    A, _ = _site(z, name, False)
    with pytest.raises(ValueError) as ei:
        gc.ctm_tensor(A, m["chi"], m["iters"], 0.0, True, m["method"], m["warmup"])
    assert str(ei.value) == m["error"]


def test_checkerboard_replay_matches_reference(fix):
    z, meta = fix
    name = "cb_d2_chi6"
    m = meta[name]
    A, B = to_dev(unpack_tensor(z, f"{name}.A")), to_dev(unpack_tensor(z, f"{name}.B"))
    Ps = [z[f"{name}.P{i}"] for i in range(8 * m["iters"])]
    env_A, env_B = gc.ctm_tensor_2site(A, B, m["chi"], m["iters"], 0.0, projectors=Ps)
    _check(z, f"{name}.envA", env_A, False)
    _check(z, f"{name}.envB", env_B, False)
    E = float(gc.compute_energy_ctm_tensor_2site(A, B, env_A, env_B, z["H"], 2))
    assert abs(E - m["energy"]) < 1e-10


def _peps(D, d, seed):
    rng = np.random.RandomState(seed)
    x = rng.standard_normal((D, D, D, D, d))
    return x / (np.linalg.norm(x) + 1e-10)


def test_single_sweep_matches_dense_ctm():
    """One sweep of the block-sparse CTM on a dense site tensor against one
    sweep of the dense CTM: corner singular values within 1e-10 (the
    reference's test_ctm_tensor.py:247-282)."""
    A = _peps(2, 2, 42)
    chi = 6
    env_t = gc.ctm_tensor(A, chi, 1, 0.0, True, "eigh", 0)
    cfg = ipeps.CTMConfig(chi=chi, max_iter=1, conv_tol=0.0, renormalize=True, projector_method="eigh",
                          qr_warmup_steps=0)
    env_d = ipeps.ctm(torch.as_tensor(A), cfg)
    for i, f in enumerate(FIELDS[:4]):
        s_t = torch.linalg.svdvals(getattr(env_t, f).todense()).sort().values
        s_d = torch.linalg.svdvals(env_d[i]).sort().values
        np.testing.assert_allclose(s_t.cpu().numpy(), s_d.cpu().numpy(), atol=1e-10, err_msg=f)


def test_symmetric_energy_matches_dense():
    """Trivial-charge SymmetricTensor run against the dense-input run,
    energies within 1e-4 (the reference's test_ctm_tensor.py:290-316).  The
    two branches do the same arithmetic, so the runs agree although a
    40-sweep run's energy moves by O(1) under a 1e-14 change of A."""
    A = _peps(2, 2, 99)
    sym = U1Symmetry()
    idx = tuple(TensorIndex(sym, np.zeros(2, np.int32), f, label=l)
                for f, l in zip((FlowDirection.OUT, FlowDirection.IN, FlowDirection.OUT, FlowDirection.IN,
                                 FlowDirection.IN), ("u", "d", "l", "r", "phys")))
    A_sym = SymmetricTensor.from_dense(A, idx)
    H = ipeps.heisenberg_gate()
    E_d = float(gc.compute_energy_ctm_tensor(A, gc.ctm_tensor(A, 6, 40, 1e-8), H, 2))
    E_s = float(gc.compute_energy_ctm_tensor(A_sym, gc.ctm_tensor(A_sym, 6, 40, 1e-8), H, 2))
    assert np.isfinite(E_d) and abs(E_s - E_d) < 1e-4


def test_mixed_precision_replay_close_to_fp64(fix):
    z, meta = fix
    name = "triv_d3_chi10"
    m = meta[name]
    A, _ = _site(z, name, False)
    Ps = [z[f"{name}.P{i}"] for i in range(4 * m["iters"])]
    e64 = gc.ctm_tensor(A, m["chi"], m["iters"], 0.0, projectors=Ps)
    emx = gc.ctm_tensor(A, m["chi"], m["iters"], 0.0, projectors=Ps, precision="bf16x3")
    for f in FIELDS:
        a, b = getattr(e64, f), getattr(emx, f)
        assert a.keys == b.keys
        # three BF16 products (hi*hi + hi*lo + lo*hi) leave ~2^-16 relative per product
        assert float((a.data - b.data).abs().max()) < 5e-5 * max(1.0, float(a.data.abs().max())), f


def test_invalid_projector_method_raises():
    with pytest.raises(ValueError, match="Unknown projector_method"):
        gc.ctm_tensor(_peps(2, 2, 42), 4, 1, projector_method="invalid")
