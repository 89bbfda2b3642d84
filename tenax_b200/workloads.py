"""Seeded synthetic two-site H_eff problems (host structure + device data).

A problem is (L, theta, W_l, W_r, R) with the flow/charge conventions of
tenax's symmetric DMRG (algorithms/dmrg.py:1165-1299):
  L[a,b,c]: keys with q_a = q_b + q_c      (environment of the left block)
  theta[a,p,q,d]: q_d = q_a + q_p + q_q    (flows IN, IN, IN, OUT)
  R[d,f,g]: keys with q_d = q_f + q_g
W_l, W_r are bulk sites of the Heisenberg cylinder MPO (width 6, J=1).
Bond sectors: ``n_sectors`` U(1) charges of one parity, sizes proportional
to exp(-q^2 / (2 sigma^2)) clipped to [lo, hi] and adjusted to sum to chi.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch

from tenax_b200.auto_mpo import heisenberg_chain_sites, heisenberg_cylinder_sites, to_symmetric
from tenax_b200.core import FlowDirection, TensorIndex, U1Symmetry
from tenax_b200.sectors import PHYS, bond_charges, env_keys, sector_sizes, theta_keys  # noqa: F401
from tenax_b200.tensor import SymmetricTensor, _device, block_shape

U1 = U1Symmetry()


@dataclass
class HeffProblem:
    L: SymmetricTensor
    theta: SymmetricTensor
    Wl: SymmetricTensor
    Wr: SymmetricTensor
    R: SymmetricTensor
    chi: int


def _fill(indices, keys, gen, dtype=torch.float64):
    sizes = [int(np.prod(block_shape(indices, k))) for k in keys]
    n = int(sum(sizes))
    dev = _device()
    if isinstance(gen, np.random.Generator):
        data = torch.from_numpy(gen.standard_normal(n)).to(dev)
    else:
        data = torch.randn(n, generator=gen, dtype=torch.float64, device=dev)
    return SymmetricTensor.from_flat(indices, keys, data)


def make_heff_problem(chi_l: int, chi_r: int, Wl: SymmetricTensor, Wr: SymmetricTensor, gen,
                      parity: int = 1, **kw) -> HeffProblem:
    vl = bond_charges(chi_l, parity=parity, **kw)
    vr = bond_charges(chi_r, parity=parity, **kw)
    mpo_l = Wl.indices[0].charges
    mpo_r = Wr.indices[3].charges
    Lidx = (TensorIndex(U1, vl, FlowDirection.OUT, "vl"), TensorIndex(U1, mpo_l, FlowDirection.OUT, "wl"),
            TensorIndex(U1, vl, FlowDirection.OUT, "vl_c"))
    Ridx = (TensorIndex(U1, vr, FlowDirection.IN, "vr"), TensorIndex(U1, mpo_r, FlowDirection.IN, "wr"),
            TensorIndex(U1, vr, FlowDirection.IN, "vr_c"))
    Tidx = (TensorIndex(U1, vl, FlowDirection.IN, "vl"), TensorIndex(U1, PHYS, FlowDirection.IN, "p1"),
            TensorIndex(U1, PHYS, FlowDirection.IN, "p2"), TensorIndex(U1, vr, FlowDirection.OUT, "vr"))
    L = _fill(Lidx, env_keys(vl, mpo_l, vl), gen)
    R = _fill(Ridx, env_keys(vr, mpo_r, vr), gen)
    th = _fill(Tidx, theta_keys(vl, vr), gen)
    return HeffProblem(L, th, Wl, Wr, R, chi_l)


def cylinder_bulk_w(Lx: int = 4, Ly: int = 6, site: int = 7):
    """Device W_l, W_r: two neighbouring bulk sites of the width-Ly cylinder MPO."""
    sites = heisenberg_cylinder_sites(Lx, Ly)
    return to_symmetric(sites[site]), to_symmetric(sites[site + 1])


def chain_bulk_w(L: int = 20, site: int = 9):
    sites = heisenberg_chain_sites(L)
    return to_symmetric(sites[site]), to_symmetric(sites[site + 1])


def mps_bond_sectors(L: int, j: int, chi: int, sigma: float = 3.0) -> np.ndarray:
    """Charges of MPS bond j (after j+1 spin-1/2 sites) of a total-Sz=0 state.

    Sector q (parity of j+1) holds at most min(C(n_l, (n_l+q)/2), C(n_r, (n_r-q)/2))
    states; sizes follow exp(-q^2/(2 sigma^2)) scaled to a total of
    min(chi, available), capped per sector.
    """
    from math import comb

    nl, nr = j + 1, L - j - 1
    qs, caps = [], []
    for q in range(-nl, nl + 1):
        if (q + nl) % 2 or abs(q) > nr:
            continue
        c = min(comb(nl, (nl + q) // 2), comb(nr, (nr - q) // 2))
        if c > 0:
            qs.append(q)
            caps.append(c)
    qs, caps = np.array(qs), np.array(caps)
    total = int(min(chi, caps.sum()))
    g = np.exp(-(qs.astype(np.float64) ** 2) / (2 * sigma * sigma))

    def sizes(s):
        return np.minimum(caps, np.maximum(1, np.rint(s * g))).astype(np.int64)

    a, b = 0.0, 1e12
    for _ in range(200):
        m = 0.5 * (a + b)
        if sizes(m).sum() < total:
            a = m
        else:
            b = m
    sz = sizes(b)
    order = np.argsort(-g, kind="stable")
    while sz.sum() > total:
        for i in order[::-1]:
            if sz.sum() <= total:
                break
            if sz[i] > 1:
                sz[i] -= 1
    while sz.sum() < total:
        for i in order:
            if sz.sum() >= total:
                break
            if sz[i] < caps[i]:
                sz[i] += 1
    return np.concatenate([np.full(int(s), int(q), np.int32) for q, s in zip(qs, sz) if s > 0])


def random_symmetric_mps(L: int, chi: int, seed: int = 0):
    """Seeded random U(1) MPS (total Sz = 0) with the tenax label/flow
    conventions (algorithms/dmrg.py:1481-1523): sites (v IN, p IN, v OUT),
    2-leg boundaries, blocks N(0,1) in sorted-key order, each site divided by
    its Frobenius norm.  Returns a ``TensorNetwork``."""
    from tenax_b200.network import TensorNetwork
    from tenax_b200.tensor import compute_valid_blocks

    rng = np.random.default_rng(seed)
    bonds = [mps_bond_sectors(L, j, chi) for j in range(L - 1)]
    net = TensorNetwork(name=f"random_symmetric_mps_L{L}_chi{chi}")
    for i in range(L):
        p = TensorIndex(U1, PHYS, FlowDirection.IN, f"p{i}")
        if i == 0:
            idx = (p, TensorIndex(U1, bonds[0], FlowDirection.OUT, f"v0_1"))
        elif i == L - 1:
            idx = (TensorIndex(U1, bonds[i - 1], FlowDirection.IN, f"v{i - 1}_{i}"), p)
        else:
            idx = (TensorIndex(U1, bonds[i - 1], FlowDirection.IN, f"v{i - 1}_{i}"), p,
                   TensorIndex(U1, bonds[i], FlowDirection.OUT, f"v{i}_{i + 1}"))
        keys = sorted(k for k in compute_valid_blocks(idx) if all(s > 0 for s in block_shape(idx, k)))
        n = int(sum(int(np.prod(block_shape(idx, k))) for k in keys))
        data = rng.standard_normal(n)
        data /= np.linalg.norm(data)
        net.add_node(i, SymmetricTensor.from_flat(idx, keys, torch.from_numpy(data).to(_device())))
    for i in range(L - 1):
        net.connect(i, f"v{i}_{i + 1}", i + 1, f"v{i}_{i + 1}")
    return net


def cylinder_mpo(Lx: int = 4, Ly: int = 6):
    """Heisenberg cylinder MPO (J=1, U(1), uncompressed) as a ``TensorNetwork``."""
    from tenax_b200.network import TensorNetwork

    net = TensorNetwork(name=f"cylinder_{Lx}x{Ly}")
    for i, s in enumerate(heisenberg_cylinder_sites(Lx, Ly)):
        net.add_node(i, to_symmetric(s))
    return net


def draw_chis(n: int, chis=(256, 512, 1024, 2048), seed: int = 0) -> np.ndarray:
    """The bond dimensions of a batch: n draws, uniform over ``chis``, from a seeded generator."""
    return np.random.default_rng(seed).choice(np.asarray(chis), size=n)


def batched_problems(n: int = 64, chis=(256, 512, 1024, 2048), seed: int = 0, gen_backend: str = "torch",
                     **kw) -> list:
    """The batched grouped-sector workload: n independent two-site problems,
    chi drawn uniformly from ``chis`` with a seeded generator."""
    Wl, Wr = cylinder_bulk_w()
    draw = draw_chis(n, chis, seed)
    if gen_backend == "torch":
        gen = torch.Generator(device=_device())
        gen.manual_seed(seed)
    else:
        gen = np.random.default_rng(seed + 1)
    return [make_heff_problem(int(c), int(c), Wl, Wr, gen, **kw) for c in draw]
