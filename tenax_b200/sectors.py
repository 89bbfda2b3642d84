"""Sector structure of the synthetic two-site H_eff problems (pure NumPy).

Bond charges with Gaussian sector sizes, the environment and theta key
sets, and the physical charges of a spin-1/2 site, with the flow/charge
conventions of tenax's symmetric DMRG (algorithms/dmrg.py:1165-1299):
  L[a,b,c]: keys with q_a = q_b + q_c
  theta[a,p,q,d]: q_d = q_a + q_p + q_q   (flows IN, IN, IN, OUT)
  R[d,f,g]: keys with q_d = q_f + q_g
This module imports nothing but NumPy, so host-only tools (the CPU timing of
the reference's algorithm) can build the same structures without loading
the device library.
"""

from __future__ import annotations

import numpy as np

PHYS = np.array([1, -1], np.int32)


def sector_sizes(chi: int, n_sectors: int = 30, sigma: float = 3.0, lo: int = 4, hi: int = 256,
                 parity: int = 1) -> tuple:
    """(charges, sizes) of one bond; deterministic integer rounding."""
    k = np.arange(n_sectors) - n_sectors // 2
    q = (parity % 2) + 2 * k
    g = np.exp(-(q.astype(np.float64) ** 2) / (2 * sigma * sigma))
    if chi < n_sectors * lo or chi > n_sectors * hi:
        raise ValueError(f"chi={chi} cannot be split into {n_sectors} sectors of size [{lo},{hi}]")

    def sizes(s):
        return np.clip(np.rint(s * g), lo, hi).astype(np.int64)

    a, b = 0.0, float(chi) * 1e6
    for _ in range(200):
        m = 0.5 * (a + b)
        if sizes(m).sum() < chi:
            a = m
        else:
            b = m
    sz = sizes(b)
    order = np.argsort(-g, kind="stable")
    while sz.sum() > chi:
        for i in order[::-1]:
            if sz.sum() <= chi:
                break
            if sz[i] > lo:
                sz[i] -= 1
    while sz.sum() < chi:
        for i in order:
            if sz.sum() >= chi:
                break
            if sz[i] < hi:
                sz[i] += 1
    return q.astype(np.int32), sz


def bond_charges(chi: int, parity: int = 1, **kw) -> np.ndarray:
    q, sz = sector_sizes(chi, parity=parity, **kw)
    return np.concatenate([np.full(int(s), int(c), np.int32) for c, s in zip(q, sz)])


def env_keys(leg0, mpo, leg2):
    """Keys (q0, qb, q2) with q0 = qb + q2."""
    s0 = set(np.unique(leg0).tolist())
    keys = []
    for qb in np.unique(mpo):
        for q2 in np.unique(leg2):
            if int(qb + q2) in s0:
                keys.append((int(qb + q2), int(qb), int(q2)))
    return sorted(keys)



def theta_keys(vl, vr) -> list:
    """Keys (q_a, q_p, q_q, q_d) of a two-site theta with q_d = q_a + q_p + q_q."""
    sr = set(np.unique(vr).tolist())
    return sorted((int(a), int(p), int(q), int(a + p + q)) for a in np.unique(vl) for p in PHYS for q in PHYS
                  if int(a + p + q) in sr)
