"""The oracle's broadened edge-split adjoint (oracle.split_ctm.BroadenedSVD,
SqrtZeroSafe), which the GPU split-CTM gradient is checked against.

* On a generic truncated SVD it equals central differences: Townsend's
  reverse mode over all triplets is exact when nothing is degenerate.
* On the reference's own split-CTM run (its recorded projectors, trivial
  charges, D=2, chi=6) the fixed-projector energy's gradient is finite and
  equals central differences (relative 1e-6), although the first moves have
  exactly degenerate and zero kept singular values."""

import json
import os

import numpy as np
import torch

from oracle import split_ctm as osc
from oracle.blocksparse import todense
from tests.golden.fixture_io import unpack_tensor

HERE = os.path.join(os.path.dirname(__file__), "golden")


def test_broadened_svd_adjoint_matches_central_differences():
    gen = torch.Generator().manual_seed(0)
    m, n, k = 9, 7, 4
    M0 = torch.randn(m, n, dtype=torch.float64, generator=gen)
    W1 = torch.randn(m, m, dtype=torch.float64, generator=gen)
    W2 = torch.randn(n, n, dtype=torch.float64, generator=gen)

    def loss(M, broadened):
        U, s, Vh = osc.BroadenedSVD.apply(M) if broadened else torch.linalg.svd(M, full_matrices=False)
        U, s, Vh = U[:, :k], s[:k], Vh[:k]
        return (W1 * (U @ U.T)).sum() + (W2 * (Vh.T @ Vh)).sum() + ((U @ torch.diag(s) @ Vh) ** 3).sum()

    x = M0.clone().requires_grad_(True)
    (g,) = torch.autograd.grad(loss(x, True), x)
    h = 1e-6
    for _ in range(4):
        v = torch.randn(m, n, dtype=torch.float64, generator=gen)
        fd = (float(loss(M0 + h * v, False)) - float(loss(M0 - h * v, False))) / (2 * h)
        ad = float((g * v).sum())
        assert abs(fd - ad) <= 1e-6 * max(abs(ad), 1.0)


def test_fixed_projector_gradient_on_reference_run():
    z = np.load(os.path.join(HERE, "split_ctm.npz"))
    meta = json.load(open(os.path.join(HERE, "split_ctm.json")))
    name = "triv_d2_chi6"
    m = meta[name]
    t = unpack_tensor(z, f"{name}.A")
    n, chi = m["iters"], m["chi"]
    H = torch.from_numpy(z["H"])
    Ps = [torch.from_numpy(z[f"{name}.P{i}"]) for i in range(8 * n)]
    a0 = torch.from_numpy(todense(t))

    def energy(x):
        site = osc.Site(x, [l.charges for l in t.legs], [l.flow for l in t.legs])
        return osc.energy(site, osc.ctm_split(site, chi, n, projectors=list(Ps), broadened=True), H)

    x = a0.clone().requires_grad_(True)
    e = energy(x)
    assert abs(float(e.detach()) - m["energy"]) < 1e-10  # same forward as the plain split
    (g,) = torch.autograd.grad(e, x)
    assert torch.isfinite(g).all()
    rng = np.random.default_rng(7)
    h = 1e-6
    with torch.no_grad():
        for _ in range(5):
            v = torch.from_numpy(rng.standard_normal(tuple(a0.shape)))
            fd = (float(energy(a0 + h * v)) - float(energy(a0 - h * v))) / (2 * h)
            ad = float((g * v).sum())
            assert abs(fd - ad) <= 1e-6 * max(abs(ad), 1e-3 * float(g.norm() * v.norm()))
