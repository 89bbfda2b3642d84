"""GPU U(1) split-CTMRG (tenax_b200.split_ctm) against the reference's runs.

* Replaying the reference's projectors and edge-split SVDs reproduces its
  environments and energy to 1e-12 -- including the U(1) cases, where the
  reference's environment is exactly zero after the first sweep.
* Projectors computed on the GPU equal the reference's where the eigenvalue
  gap at the cut is clear (1e-10 on P P^T).
* Gradient with the projectors fixed: equal to torch autograd of the oracle
  with its broadened edge-split adjoint (1e-10) and to central differences
  (h = 1e-6, relative 1e-6) on a case whose edge spectra have no nonzero
  degeneracy across the truncation; recomputing groups of sweeps
  (checkpointing) changes nothing.  The reference's own reverse pass (plain
  SVD and sqrt) is NaN on these runs: their first moves start from an
  identity-like environment with exactly degenerate and zero singular values.
* The mixed-precision (split-BF16x3) forward moves the energy by < 2e-5.
"""

import json
import os

import numpy as np
import pytest

from fixture_io import unpack_tensor

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a CUDA device", allow_module_level=True)

from oracle import split_ctm as osc  # noqa: E402
from oracle.blocksparse import todense  # noqa: E402
from tenax_b200 import split_ctm as gs  # noqa: E402
from tenax_b200.core import FlowDirection, TensorIndex, U1Symmetry  # noqa: E402
from tenax_b200.tensor import SymmetricTensor  # noqa: E402

DEV = torch.device("cuda:0")
ALL = ("triv_d2_chi6", "triv_d3_chi8", "u1_d3_chi6", "u1_d3_chi9")


@pytest.fixture(scope="module")
def fix(golden_dir):
    return (np.load(os.path.join(golden_dir, "split_ctm.npz")),
            json.load(open(os.path.join(golden_dir, "split_ctm.json"))))


def case(fix, name):
    z, meta = fix
    m = meta[name]
    t = unpack_tensor(z, f"{name}.A")
    u1 = U1Symmetry()
    idx = tuple(TensorIndex(u1, l.charges, FlowDirection(l.flow), l.label) for l in t.legs)
    A = SymmetricTensor(t.blocks, idx, _validate=False)
    n = m["iters"]
    Ps = [torch.from_numpy(z[f"{name}.P{i}"]).to(DEV) for i in range(8 * n)]
    svds = [tuple(torch.from_numpy(z[f"{name}.svd{k}{i}"]).to(DEV) for k in ("U", "s", "Vh")) for i in range(4 * n)]
    return m, t, A, Ps, svds, torch.from_numpy(z["H"]).to(DEV)


@pytest.mark.parametrize("name", ALL)
def test_replay_matches_reference(fix, name):
    z, _ = fix
    m, _, A, Ps, svds, H = case(fix, name)
    with torch.no_grad():
        env = gs.ctm_split_tensor(A, m["chi"], m["iters"], conv_tol=0.0, projectors=Ps, svds=svds)
        E = float(gs.compute_energy_split_ctm_tensor(A, env, H, 2))
    assert abs(E - m["energy"]) <= 1e-12
    for nm, x in zip(gs.SplitCTMTensorEnv._fields, env):
        ref = z[f"{name}.{nm}"]
        assert float(np.abs(x.cpu().numpy() - ref).max()) <= 1e-12 * max(1.0, float(np.abs(ref).max())), nm
    if name.startswith("u1"):
        assert E == 0.0 and all(float(x.abs().max()) == 0.0 for x in env)


@pytest.mark.parametrize("name", ("triv_d2_chi6", "triv_d3_chi8"))
def test_projectors_match_reference(fix, name):
    """Replaying the reference's run, the projector the GPU computes from
    the same grown corners spans the reference's subspace at every move
    whose eigenvalue gap at the cut exceeds 1e-6 of the largest eigenvalue
    (the identity-like start makes the first moves exactly degenerate)."""
    m, _, A, Ps, svds, _ = case(fix, name)
    chi = m["chi"]
    checked = []

    def probe(i, first, second):
        for g1, g2, Pref in (first, second):
            rho = g1 @ g1.T + g2 @ g2.T
            lam = torch.linalg.eigvalsh(0.5 * (rho + rho.T)).flip(0)
            k = min(chi, lam.shape[0])
            if k < lam.shape[0] and float(lam[0]) > 0 and float((lam[k - 1] - lam[k]) / lam[0]) > 1e-6:
                P = gs._projector(g1, g2, chi)
                checked.append(float((P @ P.T - Pref @ Pref.T).abs().max()))

    with torch.no_grad():
        gs.ctm_split_tensor(A, chi, m["iters"], conv_tol=0.0, projectors=Ps, svds=svds, probe=probe)
    assert len(checked) >= 4 and max(checked) < 1e-10, checked


def test_gradient_matches_oracle_and_fd(fix):
    """The projectors are the reference's recorded ones: a free run's
    projectors depend on the gauge its edge SVDs chose inside degenerate
    clusters, and so does the conditioning of the fixed-projector energy."""
    m, t, A, rec, _, H = case(fix, "triv_d2_chi6")
    n, chi = m["iters"], m["chi"]
    Ad = A.todense()

    def energy(x, grad=False, **kw):
        env = gs.ctm_split_tensor(A, chi, n, conv_tol=0.0, projectors=rec, A_dense=x, **kw)
        return gs.compute_energy_split_ctm_tensor(A, env, H, 2, A_dense=x)

    x = Ad.clone().requires_grad_(True)
    (g,) = torch.autograd.grad(energy(x), x)
    x2 = Ad.clone().requires_grad_(True)
    (g_ck,) = torch.autograd.grad(energy(x2, checkpoint_every=2), x2)
    assert float((g_ck - g).abs().max()) <= 1e-13 * float(g.abs().max())
    # oracle autograd under the same projectors, through the broadened edge-split adjoint
    a0 = torch.from_numpy(todense(t)).requires_grad_(True)
    site = osc.Site(a0, [l.charges for l in t.legs], [l.flow for l in t.legs])
    E0 = osc.energy(site, osc.ctm_split(site, chi, n, projectors=[p.cpu() for p in rec], broadened=True), H.cpu())
    (g0,) = torch.autograd.grad(E0, a0)
    assert float((g.cpu() - g0).abs().max()) <= 1e-10 * float(g0.abs().max())
    # central differences of the fixed-projector energy
    rng = np.random.default_rng(7)
    h = 1e-6
    with torch.no_grad():
        for _ in range(10):
            v = torch.from_numpy(rng.standard_normal(tuple(Ad.shape))).to(DEV)
            fd = (float(energy(Ad + h * v)) - float(energy(Ad - h * v))) / (2 * h)
            ad = float((g * v).sum())
            assert abs(fd - ad) <= 1e-6 * max(abs(ad), 1e-3 * float(g.norm() * v.norm()))


def test_mixed_forward_close_to_fp64(fix):
    """Same projectors, edge SVDs computed: the split-BF16x3 edge projection
    moves the energy by less than 2e-5 (about 2^-16 relative per product,
    the three-product scheme's accuracy)."""
    m, _, A, _, _, H = case(fix, "triv_d2_chi6")
    rec: list = []
    with torch.no_grad():
        e64 = gs.ctm_split_tensor(A, m["chi"], m["iters"], conv_tol=0.0, record=rec)
        emx = gs.ctm_split_tensor(A, m["chi"], m["iters"], conv_tol=0.0, projectors=rec, precision="bf16x3")
        E64 = float(gs.compute_energy_split_ctm_tensor(A, e64, H, 2))
        Emx = float(gs.compute_energy_split_ctm_tensor(A, emx, H, 2))
    assert abs(Emx - E64) <= 2e-5


def test_svd_driver_choice(fix):
    """Both edge-SVD drivers give the same environment when nothing forces a
    basis choice (the fixture's edges are 12 x 12, below the polar driver's
    size, so both run Jacobi); an unknown driver is a ValueError."""
    m, _, A, _, _, H = case(fix, "triv_d2_chi6")
    with torch.no_grad():
        ep = gs.ctm_split_tensor(A, m["chi"], m["iters"], conv_tol=0.0, svd_driver="polar")
        ej = gs.ctm_split_tensor(A, m["chi"], m["iters"], conv_tol=0.0, svd_driver="jacobi")
    for a, b in zip(ep, ej):
        assert torch.equal(a, b)
    with pytest.raises(ValueError, match="svd_driver"):
        gs.ctm_split_tensor(A, m["chi"], 1, conv_tol=0.0, svd_driver="gesvd")
