"""GPU CTMRG (tenax_b200.ipeps) against the reference's runs and the oracle.

Parity is defined with the projectors fixed (the reference's CTM on random
site tensors is chaotic under rounding; see tests/test_oracle_ctm.py):
  * replaying the reference's own projectors reproduces its environments and
    energy to 1e-12;
  * projectors computed on the GPU span the reference's kept subspace where
    the eigenvalue gap at the cut exceeds 1e-6 (1e-10 on P P^T);
  * the hand-written adjoint equals torch autograd of the oracle under the
    same projectors (relative 1e-10) and central finite differences of the
    fixed-projector energy (h = 1e-6, 20 random directions, relative 1e-6);
  * the renormalisation kernels and the dense contraction adjoints match
    torch float64 references (1e-13).
"""

import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a CUDA device", allow_module_level=True)

from oracle import ctm as oc  # noqa: E402
from tenax_b200 import ipeps as gc  # noqa: E402
from tenax_b200 import dense  # noqa: E402

DEV = torch.device("cuda:0")
NAMES = ("C1", "C2", "C3", "C4", "T1", "T2", "T3", "T4")
SMALL = ("qr_small", "eigh_small", "qr_mid", "qr_warm")


@pytest.fixture(scope="module")
def ctm_fix(golden_dir):
    return (np.load(os.path.join(golden_dir, "ctm.npz")),
            json.load(open(os.path.join(golden_dir, "ctm.json"))))


def _case(fix, name, device=DEV):
    z, meta = fix
    m = meta[name]
    A = torch.from_numpy(z[f"{name}.A"])
    Ps = [torch.from_numpy(z[f"{name}.P{i}"]) for i in range(4 * m["iters"])] if name != "c4" else None
    cfg = gc.CTMConfig(chi=m["chi"], max_iter=m["iters"], conv_tol=0.0, projector_method=m["method"],
                       qr_warmup_steps=m["warmup"])
    return m, A, Ps, cfg


def _rel(a, b):
    return float(((a - b).abs().max() / b.abs().max()).detach())


def test_renormalize_kernels_match_torch():
    g = torch.Generator(device="cpu").manual_seed(1)
    sizes = [1, 7, 6400, 102400, 33, 1000, 65537, 12]
    xs = [torch.randn(n, generator=g, dtype=torch.float64) for n in sizes]
    xs[4][[3, 17]] = 5.0  # tie for the maximum
    xs[5][[0, 999]] = torch.tensor([-4.0, 4.0], dtype=torch.float64)  # tie with opposite signs
    xs[7].zero_()  # all zero: m = 0
    xs = [x.to(DEV).requires_grad_(True) for x in xs]
    gys = [torch.randn(n, generator=g, dtype=torch.float64).to(DEV) for n in sizes]
    ys = gc._Renormalize.apply(*xs)
    grads = torch.autograd.grad(ys, xs, gys)
    xr = [x.detach().clone().requires_grad_(True) for x in xs]
    yr = [x / (x.abs().max() + gc.EPS) for x in xr]
    gr = torch.autograd.grad(yr, xr, gys)
    for y, r in zip(ys, yr):
        assert torch.allclose(y, r, rtol=1e-15, atol=0)
    for a, b in zip(grads, gr):
        assert float((a - b).abs().max()) <= 1e-13 * max(1.0, float(b.abs().max()))


@pytest.mark.parametrize("subs,shapes", [
    ("ab,buc->auc", [(12, 9), (9, 5, 12)]),
    ("pxwB,txsw->pBst", [(6, 5, 5, 7), (5, 5, 5, 5)]),
    ("psA,pBst->AtB", [(6, 5, 7), (6, 7, 5, 5)]),
    ("udlrs,UDLRt->uUdDlLrRst", [(2, 2, 2, 2, 2), (2, 2, 2, 2, 2)]),
    ("dfgst,fgdwx->stwx", [(4, 9, 9, 2, 2), (9, 9, 4, 2, 2)]),
])
def test_dense_contract_and_adjoint(subs, shapes):
    g = torch.Generator(device="cpu").manual_seed(2)
    a, b = (torch.randn(s, generator=g, dtype=torch.float64).to(DEV).requires_grad_(True) for s in shapes)
    out = dense.contract(subs, a, b)
    ref = torch.einsum(subs, a, b)
    assert _rel(out, ref) < 1e-13
    w = torch.randn(out.shape, generator=g, dtype=torch.float64).to(DEV)
    ga, gb = torch.autograd.grad(out, (a, b), w)
    ra, rb = torch.autograd.grad(ref, (a, b), w)
    assert _rel(ga, ra) < 1e-13 and _rel(gb, rb) < 1e-13


@pytest.mark.parametrize("name", SMALL)
def test_replay_reference_projectors(ctm_fix, name):
    z, _ = ctm_fix
    m, A, Ps, cfg = _case(ctm_fix, name)
    with torch.no_grad():
        env = gc.ctm(A.to(DEV), cfg, projectors=[p.to(DEV) for p in Ps])
        E = float(gc.compute_energy_ctm(A.to(DEV), env, gc.heisenberg_gate(), 2))
    assert abs(E - m["energy"]) <= 1e-12
    for x, nm in zip(env, NAMES):
        ref = torch.from_numpy(z[f"{name}.{nm}"])
        assert float((x.cpu() - ref).abs().max()) <= 1e-12 * float(ref.abs().max()), nm


@pytest.mark.parametrize("name", SMALL)
def test_gpu_projectors_span_reference_subspace(ctm_fix, name):
    m, A, Ps, cfg = _case(ctm_fix, name)
    Ad = A.to(DEV)
    with torch.no_grad():
        a = gc.build_double_layer(Ad)
        env = gc.initialize_env(a, m["chi"])
        warm = m["warmup"] if m["method"] == "qr" else 0
        checked = 0
        for it in range(m["iters"]):
            meth = "eigh" if it < warm else m["method"]
            for i in range(4):
                c1, c2, _, slots, _ = gc._MOVE_SPECS[i]
                Cg1 = dense.einsum(c1, env[slots[0]], env[slots[1]])
                Cg2 = dense.einsum(c2, env[slots[2]], env[slots[3]])
                n = Cg1.shape[0] * Cg1.shape[1]
                gap = oc.truncation_gap(Cg1.reshape(n, -1).cpu(), Cg2.reshape(n, -1).cpu(), m["chi"], meth)
                Pref = Ps[4 * it + i]
                if gap > 1e-6:
                    P = gc._projector(Cg1, Cg2, m["chi"], meth).cpu()
                    assert float((P @ P.T - Pref @ Pref.T).abs().max()) < 1e-10
                    checked += 1
                env, _ = gc.ctm_move(env, a, i, m["chi"], meth, Pref.to(DEV))
            env = gc.renormalize_env(env)
        assert checked >= 4 * m["iters"] - 2


@pytest.mark.parametrize("name", SMALL)
def test_adjoint_matches_oracle_autograd(ctm_fix, name):
    m, A, Ps, cfg = _case(ctm_fix, name)
    E1, g1, _ = gc.energy_and_grad(A.to(DEV), gc.heisenberg_gate(), cfg, projectors=[p.to(DEV) for p in Ps])
    E0, g0, _ = oc.energy_and_grad(A, oc.heisenberg_gate(), m["chi"], m["iters"], m["method"], m["warmup"],
                                   projectors=Ps)
    assert abs(E1 - E0) <= 1e-12
    assert _rel(g1.cpu(), g0) <= 1e-10


def test_adjoint_matches_fixed_projector_fd(ctm_fix):
    """Central differences h=1e-6 on 20 random directions of the energy with
    the projectors of the unperturbed run held fixed."""
    m, A, _, cfg = _case(ctm_fix, "qr_mid")
    Ad = A.to(DEV)
    H = gc.heisenberg_gate()
    E, g, Ps = gc.energy_and_grad(Ad, H, cfg)

    def energy(x):
        with torch.no_grad():
            env = gc.ctm(x, cfg, projectors=Ps)
            return float(gc.compute_energy_ctm(x, env, H, 2))

    assert abs(energy(Ad) - E) <= 1e-13
    rng = np.random.default_rng(20)
    h = 1e-6
    worst = 0.0
    for _ in range(20):
        v = torch.from_numpy(rng.standard_normal(A.shape)).to(DEV)
        fd = (energy(Ad + h * v) - energy(Ad - h * v)) / (2 * h)
        ad = float((g * v).sum())
        worst = max(worst, abs(fd - ad) / max(abs(ad), 1e-3 * float(g.norm() * v.norm())))
    assert worst <= 1e-6, worst


def test_c4_free_run_replays_in_oracle(ctm_fix):
    """D=4, chi=80, 30 QR sweeps: the GPU's own projectors, replayed in the
    oracle, give the same energy (1e-10); the free-running energy lies in
    the band the reference's chaotic iteration visits (|dE| < 1e-2)."""
    m, A, _, cfg = _case(ctm_fix, "c4")
    rec: list = []
    with torch.no_grad():
        env = gc.ctm(A.to(DEV), cfg, record=rec)
        E = float(gc.compute_energy_ctm(A.to(DEV), env, gc.heisenberg_gate(), 2))
    Eo = oc.energy_fixed(A, oc.heisenberg_gate(), m["chi"], m["iters"], [p.cpu() for p in rec])
    assert abs(E - Eo) <= 1e-10
    assert abs(E - m["energy"]) < 1e-2
