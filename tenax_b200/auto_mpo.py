"""Finite-automaton MPO construction with U(1) bond charges (host side).

Builds the same MPO as tenax ``algorithms/auto_mpo.py`` with
``compress=False``: bond state 0 = "done", the last state = "vacuum", one
state per term in flight across the bond (ordered by term), W tensors of
shape (D_l, d, d, D_r) with legs (IN bond, IN top, OUT bottom, OUT bond),
and bond charges equal to the charge transferred by the term's operators to
the left of the bond.  Output is host numpy (``MPOSite``); ``to_symmetric``
uploads a site as a ``SymmetricTensor``.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np


def spin_half_ops() -> dict:
    return {
        "Sz": np.array([[0.5, 0.0], [0.0, -0.5]]),
        "Sp": np.array([[0.0, 1.0], [0.0, 0.0]]),
        "Sm": np.array([[0.0, 0.0], [1.0, 0.0]]),
        "Id": np.eye(2),
    }


@dataclass
class MPOSite:
    W: np.ndarray              # (D_l, d, d, D_r) dense
    charges: tuple             # (left bond, phys, phys, right bond) int32 charge arrays
    flows: tuple = (1, 1, -1, -1)
    labels: tuple = ()

    def blocks(self) -> dict:
        """All conservation-valid non-empty sectors (zero-valued ones included)."""
        out = {}
        cl, cp, cb, cr = self.charges
        for ql in np.unique(cl):
            for qp in np.unique(cp):
                for qb in np.unique(cb):
                    qr = ql + qp - qb
                    if qr not in set(cr.tolist()):
                        continue
                    idx = [np.where(cl == ql)[0], np.where(cp == qp)[0], np.where(cb == qb)[0], np.where(cr == qr)[0]]
                    out[(int(ql), int(qp), int(qb), int(qr))] = self.W[np.ix_(*idx)]
        return out


def _op_charge(op: np.ndarray, phys: np.ndarray) -> int:
    q = None
    for i, j in zip(*np.nonzero(np.abs(op) > 1e-14)):
        t = int(phys[i]) - int(phys[j])
        if q is None:
            q = t
        elif q != t:
            raise ValueError(f"Operator mixes charge sectors: found transfers {q} and {t}.")
    return 0 if q is None else q


def build_auto_mpo_sites(terms, L: int, d: int = 2, site_ops: dict | None = None, phys=None) -> list:
    """``terms``: (coeff, op_name, site, op_name, site, ...) tuples."""
    ops = site_ops or spin_half_ops()
    phys = np.array([1, -1], np.int32) if phys is None else np.asarray(phys, np.int32)
    ident = np.eye(d)
    parsed = []
    for t in terms:
        coeff, args = complex(t[0]), t[1:]
        pairs = sorted(((int(args[k + 1]), ops[args[k]]) for k in range(0, len(args), 2)), key=lambda x: x[0])
        sites = [s for s, _ in pairs]
        if len(set(sites)) != len(sites):
            raise ValueError(f"Duplicate sites in term: {sites}")
        parsed.append((coeff, pairs))
    if not parsed:
        raise ValueError("No terms")
    # state index of each in-flight term at each bond
    states = []
    for j in range(L - 1):
        st, nxt = {}, 1
        for tid, (_, pairs) in enumerate(parsed):
            if pairs[0][0] <= j < pairs[-1][0]:
                st[tid] = nxt
                nxt += 1
        states.append(st)
    cplx = any(c.imag != 0 for c, _ in parsed)
    sites_out = []
    for i in range(L):
        Dl = 1 if i == 0 else len(states[i - 1]) + 2
        Dr = 1 if i == L - 1 else len(states[i]) + 2
        W = np.zeros((Dl, d, d, Dr), dtype=np.complex128 if cplx else np.float64)
        vac_l = 0 if i == 0 else Dl - 1
        vac_r = Dr - 1
        if L > 1:
            if i == 0:
                W[0, :, :, vac_r] = ident
            elif i == L - 1:
                W[0, :, :, 0] = ident
            else:
                W[0, :, :, 0] = ident
                W[vac_l, :, :, vac_r] = ident
        for tid, (coeff, pairs) in enumerate(parsed):
            lo, hi = pairs[0][0], pairs[-1][0]
            if i < lo or i > hi:
                continue
            op = dict(pairs).get(i, ident)
            c = coeff if cplx else coeff.real
            if lo == hi:
                W[vac_l, :, :, 0] += c * op
            elif i == lo:
                W[vac_l, :, :, states[i][tid]] += c * op
            elif i == hi:
                W[states[i - 1][tid], :, :, 0] += op
            else:
                W[states[i - 1][tid], :, :, states[i][tid]] = op
        sites_out.append(W)
    # bond charges
    bond_q = []
    for j in range(L - 1):
        q = np.zeros(len(states[j]) + 2, np.int32)
        for tid, s in states[j].items():
            q[s] = sum(_op_charge(op, phys) for site, op in parsed[tid][1] if site <= j)
        bond_q.append(q)
    out = []
    for i, W in enumerate(sites_out):
        ql = np.zeros(W.shape[0], np.int32) if i == 0 else bond_q[i - 1]
        qr = np.zeros(W.shape[3], np.int32) if i == L - 1 else bond_q[i]
        labels = ("w_left_0" if i == 0 else f"w{i - 1}_{i}", f"mpo_top_{i}", f"mpo_bot_{i}",
                  "w_right" if i == L - 1 else f"w{i}_{i + 1}")
        out.append(MPOSite(W, (ql, phys, phys, qr), labels=labels))
    return out


def heisenberg_chain_sites(L: int, Jz: float = 1.0, Jxy: float = 1.0, hz: float = 0.0) -> list:
    """Spin-1/2 XXZ chain (tenax algorithms/dmrg.py:1373-1412)."""
    terms = []
    for i in range(L - 1):
        terms += [(Jz, "Sz", i, "Sz", i + 1), (Jxy / 2, "Sp", i, "Sm", i + 1), (Jxy / 2, "Sm", i, "Sp", i + 1)]
    if hz != 0.0:
        terms += [(hz, "Sz", i) for i in range(L)]
    if not terms:
        terms = [(0.0, "Sz", 0)]
    return build_auto_mpo_sites(terms, L)


def cylinder_bonds(Lx: int, Ly: int) -> list:
    """Nearest-neighbour bonds of an Lx x Ly cylinder (periodic in y), each
    bond once, column-major sites i = x*Ly + y."""
    bonds = []
    for x in range(Lx):
        for y in range(Ly):
            i, j = x * Ly + y, x * Ly + (y + 1) % Ly
            bonds.append((min(i, j), max(i, j)))
            if x < Lx - 1:
                bonds.append((x * Ly + y, (x + 1) * Ly + y))
    return bonds


def heisenberg_cylinder_sites(Lx: int, Ly: int, J: float = 1.0) -> list:
    terms = []
    for i, j in cylinder_bonds(Lx, Ly):
        terms += [(J, "Sz", i, "Sz", j), (J / 2, "Sp", i, "Sm", j), (J / 2, "Sm", i, "Sp", j)]
    return build_auto_mpo_sites(terms, Lx * Ly)


def to_symmetric(site: MPOSite):
    """Upload one MPO site as a device ``SymmetricTensor``."""
    from tenax_b200.core import FlowDirection, TensorIndex, U1Symmetry
    from tenax_b200.tensor import SymmetricTensor

    u1 = U1Symmetry()
    idx = tuple(TensorIndex(u1, c, FlowDirection(f), lab) for c, f, lab in zip(site.charges, site.flows, site.labels))
    return SymmetricTensor(site.blocks(), idx)
