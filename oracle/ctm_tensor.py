"""Float64 NumPy restatement of tenax's block-sparse standard CTMRG
(``algorithms/_ctm_tensor.py``), with its energy.

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).

Tensors are ``oracle.blocksparse.OTensor`` objects and every step is the
reference's own operation on them: label contractions with the filtered
block-sparse semantics (``contract_symmetric``), ``fuse_indices`` with the
pair-grouped sector layout, the per-sector eigh projector with its global
``(-lambda, -index)`` truncation, ``from_dense(tol=inf)`` re-wraps and the
max-abs renormalisation that re-wraps every tensor over all its valid
blocks.  Environments are dicts ``{"C1": OTensor, ..., "T4": OTensor}``.

Every projector can be supplied (replay) and every computed one recorded,
as the dense ``P`` the reference passes to ``jax.lax.stop_gradient``
(:185, :247, :282); a run given the reference's recorded projectors
reproduces its environments to rounding.
"""

from __future__ import annotations

import numpy as np
import torch

from oracle import ctm as dense_ctm
from oracle.blocksparse import (
    Leg,
    OTensor,
    block_shape,
    contract_symmetric,
    fuse_indices,
    fused_charges,
    labels_to_subscripts,
    todense,
    valid_blocks,
)

EPS = 1e-15  # tenax core/__init__.py:15
IN, OUT = 1, -1
FIELDS = ("C1", "C2", "C3", "C4", "T1", "T2", "T3", "T4")

# corner (label_a, label_b, flow_a, flow_b, reference axis of A for the charges)
# (_split_ctm_tensor.py:262-267)
CORNER_SPECS = {
    "C1": ("c1_d", "c1_r", IN, OUT, 1),
    "C2": ("c2_l", "c2_d", IN, OUT, 0),
    "C3": ("c3_u", "c3_l", OUT, IN, 1),
    "C4": ("c4_r", "c4_u", OUT, IN, 0),
}
# edge (label chi1, label D^2, label chi2, flows, A axis for the chi charges,
# A axis fused into the D^2 leg) (_ctm_tensor.py:395-405)
EDGE_SPECS = {
    "T1": ("t1_l", "u2", "t1_r", IN, IN, OUT, 3, 0),
    "T2": ("t2_u", "r2", "t2_d", OUT, OUT, IN, 0, 3),
    "T3": ("t3_r", "d2", "t3_l", OUT, OUT, IN, 3, 1),
    "T4": ("t4_d", "l2", "t4_u", IN, IN, OUT, 1, 2),
}

# One move per direction (_ctm_tensor.py:586-759):
#   (corner, its leg relabelled to the edge's, perpendicular edge, fused pair)
#   x 2, the parallel edge with its two fused pairs, and the output relabels.
MOVES = {
    "left": dict(
        c1=("C1", ("c1_r", "t1_l"), "T1", ("c1_d", "u2")),
        c2=("C4", ("c4_u", "t3_r"), "T3", ("c4_r", "d2")),
        edge=("T4", ("t4_d", "u2"), ("t4_u", "d2")),
        out=(("C1", {"chi_new": "c1_d", "t1_r": "c1_r"}), ("C4", {"chi_new": "c4_r", "t3_l": "c4_u"}),
             ("T4", {"chi_new": "t4_d", "chi_new_r": "t4_u", "r2": "l2"}))),
    "right": dict(
        c1=("C2", ("c2_l", "t1_r"), "T1", ("c2_d", "u2")),
        c2=("C3", ("c3_u", "t3_l"), "T3", ("c3_l", "d2")),
        edge=("T2", ("t2_u", "u2"), ("t2_d", "d2")),
        out=(("C2", {"chi_new": "c2_l", "t1_l": "c2_d"}), ("C3", {"chi_new": "c3_u", "t3_r": "c3_l"}),
             ("T2", {"chi_new": "t2_u", "chi_new_r": "t2_d", "l2": "r2"}))),
    "top": dict(
        c1=("C1", ("c1_d", "t4_d"), "T4", ("c1_r", "l2")),
        c2=("C2", ("c2_d", "t2_u"), "T2", ("c2_l", "r2")),
        edge=("T1", ("t1_l", "l2"), ("t1_r", "r2")),
        out=(("C1", {"chi_new": "c1_d", "t4_u": "c1_r"}), ("C2", {"chi_new": "c2_l", "t2_d": "c2_d"}),
             ("T1", {"chi_new": "t1_l", "chi_new_r": "t1_r", "d2": "u2"}))),
    "bottom": dict(
        c1=("C4", ("c4_r", "t4_u"), "T4", ("c4_u", "l2")),
        c2=("C3", ("c3_l", "t2_d"), "T2", ("c3_u", "r2")),
        edge=("T3", ("t3_r", "l2"), ("t3_l", "r2")),
        out=(("C4", {"chi_new": "c4_r", "t4_d": "c4_u"}), ("C3", {"chi_new": "c3_u", "t2_u": "c3_l"}),
             ("T3", {"chi_new": "t3_r", "chi_new_r": "t3_l", "u2": "d2"}))),
}
DIRECTIONS = ("left", "right", "top", "bottom")


# ---------------------------------------------------------------------------
# tensor helpers
# ---------------------------------------------------------------------------

def relabels(t: OTensor, mapping: dict) -> OTensor:
    return OTensor(tuple(Leg(l.charges, l.flow, mapping.get(l.label, l.label)) for l in t.legs), t.blocks,
                   t.modulus)


def bar(t: OTensor) -> OTensor:
    """Flip every flow, keep charges and values (core/tensor.py ``bar``)."""
    return OTensor(tuple(Leg(l.charges, -l.flow, l.label) for l in t.legs), t.blocks, t.modulus)


def contract(*ts: OTensor) -> OTensor:
    """Label contraction, free labels in order of appearance
    (contractor.py:490-531 -> :291-484)."""
    subs, _ = labels_to_subscripts(ts)
    out, _ = contract_symmetric(list(ts), subs)
    return out


def fuse_by_label(t: OTensor, la, lb, fused, flow) -> OTensor:
    """(_ctm_tensor.py:65-76)"""
    lab = t.labels()
    return fuse_indices(t, lab.index(la), lab.index(lb), fused, flow)


def from_dense(arr: np.ndarray, legs, modulus) -> OTensor:
    """Every valid block with non-empty legs, cut from ``arr``
    (core/tensor.py:670-732 with tol=inf)."""
    charges = [l.charges for l in legs]
    blocks = {}
    for k in sorted(valid_blocks(charges, [l.flow for l in legs], modulus)):
        pos = [np.where(np.asarray(c) == q)[0] for c, q in zip(charges, k)]
        if not all(len(p) for p in pos):
            continue
        blocks[k] = np.array(arr[np.ix_(*pos)], dtype=np.float64)
    return OTensor(tuple(legs), blocks, modulus)


def derive_charges(base, n):
    """(_split_ctm_tensor.py:251-257)"""
    base = np.asarray(base, dtype=np.int32)
    if n <= len(base):
        return base[:n].copy()
    return np.tile(base, n // len(base) + 1)[:n].astype(np.int32)


# ---------------------------------------------------------------------------
# double layer and initial environment
# ---------------------------------------------------------------------------

def double_layer(A: OTensor, open_phys: bool = False) -> OTensor:
    """sum_phys A bar(A), ket/bra pairs fused (u,U)->u2 IN, (d,D)->d2 OUT,
    (l,L)->l2 IN, (r,R)->r2 OUT (_ctm_tensor.py:346-392)."""
    m = {"u": "U", "d": "D", "l": "L", "r": "R"}
    if open_phys:
        m["phys"] = "phys_bra"
    a8 = contract(A, relabels(bar(A), m))
    a = fuse_by_label(a8, "u", "U", "u2", IN)
    a = fuse_by_label(a, "d", "D", "d2", OUT)
    a = fuse_by_label(a, "l", "L", "l2", IN)
    return fuse_by_label(a, "r", "R", "r2", OUT)


def init_env(A: OTensor, chi: int, dense: bool = False) -> dict:
    """Identity corners, identity-like edges (_ctm_tensor.py:408-583).

    ``dense``: the DenseTensor branch (trivial charges, corners
    eye(min(chi, D^2)) zero-padded, _split_ctm_tensor.py:64-80)."""
    D = A.legs[0].dim
    D2 = D * D
    mod = A.modulus
    env = {}
    for name, (la, lb, fa, fb, ref) in CORNER_SPECS.items():
        if dense:
            q = np.zeros(chi, np.int32)
            C = np.zeros((chi, chi))
            m = min(chi, D2)
            C[:m, :m] = np.eye(m)
        else:
            leg = A.legs[ref]
            q = derive_charges(fused_charges(leg, Leg(leg.charges, -leg.flow), fa, mod), chi)
            C = np.eye(chi)
        env[name] = from_dense(C, (Leg(q, fa, la), Leg(q.copy(), fb, lb)), mod)
    for name, (l1, l2, l3, f1, f2, f3, rc, rd) in EDGE_SPECS.items():
        T = np.zeros((chi, D2, chi))
        for i in range(min(chi, D2)):
            T[i, :, i] += 1.0
        if dense:
            qc, qd = np.zeros(chi, np.int32), np.zeros(D2, np.int32)
        else:
            qc = derive_charges(A.legs[rc].charges, chi)
            leg = A.legs[rd]
            qd = fused_charges(leg, Leg(leg.charges, -leg.flow), f2, mod)
        env[name] = from_dense(T, (Leg(qc, f1, l1), Leg(qd, f2, l2), Leg(qc.copy(), f3, l3)), mod)
    return env


# ---------------------------------------------------------------------------
# projector
# ---------------------------------------------------------------------------

def eigh_projector_symmetric(C1g: OTensor, C4g: OTensor, chi: int) -> np.ndarray:
    """Per-sector density matrices and global truncation; returns the dense
    projector (_ctm_tensor.py:79-192).

    For each fused charge q: rho_q = sum M M^T over the blocks of C1g then
    C4g carrying q, M the block reshaped to (d_q, -1) with d_q counted on
    C1g's fused leg (so C4g blocks of another height raise numpy's
    reshape ValueError, as in the reference); rho_q symmetrised, eigh.
    Eigenpairs sorted by (-lambda, -index) over all sectors, the first chi
    kept; sector q's kept vectors (indices descending) fill consecutive
    columns, sectors in increasing q, at q's rows of the fused leg."""
    fpos = C1g.labels().index("fused")
    cpos = 1 - fpos
    fleg = C1g.legs[fpos]
    fused_total = fleg.dim

    def group(Cg):
        g: dict = {}
        for key, blk in Cg.blocks.items():
            g.setdefault(int(key[fpos]), []).append((int(key[cpos]), blk))
        return g

    g1, g4 = group(C1g), group(C4g)
    charges = np.asarray(fleg.charges)
    rows = {q: np.where(charges == q)[0] for q in sorted(set(g1) | set(g4))}
    sectors = {}
    for q in sorted(set(g1) | set(g4)):
        dq = len(rows[q])
        if dq == 0:
            continue
        rho = np.zeros((dq, dq))
        for entries in (g1.get(q, []), g4.get(q, [])):
            for _, blk in entries:
                M = blk.reshape(dq, -1) if fpos == 0 else blk.reshape(-1, dq).T
                rho = rho + M @ M.conj().T
        rho = 0.5 * (rho + rho.conj().T)
        w, v = np.linalg.eigh(rho)
        sectors[q] = (v, w)
    pairs = [(float(val), q, i) for q, (_, w) in sectors.items() for i, val in enumerate(w)]
    pairs.sort(key=lambda x: (-x[0], -x[2]))
    n_keep = min(chi, len(pairs))
    keep: dict = {}
    for _, q, i in pairs[:n_keep]:
        keep.setdefault(q, []).append(i)
    P = np.zeros((fused_total, n_keep))
    col = 0
    for q in sorted(keep):
        idx = sorted(keep[q], reverse=True)
        P[np.ix_(rows[q], np.arange(col, col + len(idx)))] = sectors[q][0][:, idx]
        col += len(idx)
    return P


def dense_projector(C1g: OTensor, C4g: OTensor, chi: int, method: str) -> np.ndarray:
    """Dense projector of the densified grown corners (_ctm_tensor.py:231-289):
    QR of [C1g C4g] then eigh of R R^T, or eigh of C1g C1g^T + C4g C4g^T;
    the top-k eigenvectors in decreasing order."""
    a, b = todense(C1g), todense(C4g)
    if method == "qr":
        Q, R = np.linalg.qr(np.concatenate([a, b], axis=1))
        rho = R @ R.conj().T
        rho = 0.5 * (rho + rho.conj().T)
        w, v = np.linalg.eigh(rho)
        k = min(chi, len(w))
        return Q @ v[:, -k:][:, ::-1]
    rho = a @ a.conj().T + b @ b.conj().T
    rho = 0.5 * (rho + rho.conj().T)
    w, v = np.linalg.eigh(rho)
    k = min(chi, len(w))
    return v[:, -k:][:, ::-1]


def projector(C1g: OTensor, C4g: OTensor, chi: int, method: str, dense: bool) -> np.ndarray:
    """Method dispatch (_ctm_tensor.py:195-296): 'qr' always dense; 'eigh'
    per sector when both corners have blocks (and the inputs are symmetric),
    else dense."""
    if method not in ("eigh", "qr"):
        raise ValueError(f"Unknown projector_method={method!r}; expected 'eigh' or 'qr'.")
    if method == "eigh" and not dense and C1g.blocks and C4g.blocks:
        return eigh_projector_symmetric(C1g, C4g, chi)
    return dense_projector(C1g, C4g, chi, method)


def wrap_projector(P: np.ndarray, fleg: Leg, modulus) -> OTensor:
    """P (fused, chi_new) with trivial chi_new charges flowing OUT, re-wrapped
    with from_dense(tol=inf) (_ctm_tensor.py:187-191, :253-264, :284-296)."""
    legs = (Leg(fleg.charges, fleg.flow, "fused"), Leg(np.zeros(P.shape[1], np.int32), OUT, "chi_new"))
    return from_dense(P, legs, modulus)


def apply_projector(P, C1g, C4g, Tg, fl, fr):
    """P^T C1g, P^T C4g, P^T Tg P (_ctm_tensor.py:299-338)."""
    Pb = bar(P)
    C1n = contract(Pb, C1g)
    C4n = contract(Pb, C4g)
    step = contract(relabels(Pb, {"fused": fl}), Tg)
    Tn = contract(step, relabels(P, {"fused": fr, "chi_new": "chi_new_r"}))
    return C1n, C4n, Tn


# ---------------------------------------------------------------------------
# moves, sweeps, driver
# ---------------------------------------------------------------------------

def grow(env_self: dict, env_nb: dict, a: OTensor, direction: str):
    """The two grown corners (fused, col) and the grown edge (fl, fr, D^2)
    of one move (_ctm_tensor.py:586-759)."""
    mv = MOVES[direction]
    grown = []
    for cname, (old, new), ename, (fa, fb) in (mv["c1"], mv["c2"]):
        g = contract(relabels(env_self[cname], {old: new}), env_nb[ename])
        grown.append(fuse_by_label(g, fa, fb, "fused", IN))
    ename, (la, lb), (ra, rb) = mv["edge"]
    Tg = fuse_by_label(contract(env_self[ename], a), la, lb, "fl", IN)
    return grown[0], grown[1], fuse_by_label(Tg, ra, rb, "fr", OUT)


def move(env_self: dict, env_nb: dict, a: OTensor, chi: int, method: str, direction: str, dense: bool = False,
         P_in=None, rec=None) -> dict:
    """One directional move (_ctm_tensor.py:586-759)."""
    mv = MOVES[direction]
    g1, g2, Tg = grow(env_self, env_nb, a, direction)
    grown = [g1, g2]
    Pd = P_in if P_in is not None else projector(grown[0], grown[1], chi, method, dense)
    if rec is not None:
        rec.append(np.array(Pd))
    P = wrap_projector(np.asarray(Pd), grown[0].legs[grown[0].labels().index("fused")], a.modulus)
    new = apply_projector(P, grown[0], grown[1], Tg, "fl", "fr")
    out = dict(env_self)
    for (name, mp), t in zip(mv["out"], new):
        out[name] = relabels(t, mp)
    return out


def normalize(t: OTensor) -> OTensor:
    """x / (max|x| + EPS) over the dense form, re-wrapped over every valid
    block (_ctm_tensor.py:767-779)."""
    d = todense(t)
    m = np.max(np.abs(d)) if d.size else 0.0
    return from_dense(d / (m + EPS), t.legs, t.modulus)


def sweep(env, a, chi, renormalize, method, dense=False, projectors=None, rec=None):
    """Left, right, top, bottom, then renormalise (_ctm_tensor.py:796-808)."""
    for i, dr in enumerate(DIRECTIONS):
        env = move(env, env, a, chi, method, dr, dense, None if projectors is None else projectors[i], rec)
    if renormalize:
        env = {k: normalize(v) for k, v in env.items()}
    return env


def sv_diff(s_new, s_old):
    """(_ctm_tensor.py:861-865)"""
    s1 = s_new / (np.sum(s_new) + 1e-15)
    s2 = s_old / (np.sum(s_old) + 1e-15)
    return float(np.max(np.abs(s1 - s2)))


def ctm_tensor(A: OTensor, chi, max_iter=100, conv_tol=1e-8, renormalize=True, method="eigh", warmup=3,
               dense=False, projectors=None, rec=None):
    """(_ctm_tensor.py:868-917).  ``projectors``: flat list, four per sweep."""
    a = double_layer(A)
    env = init_env(A, chi, dense)
    n = 0

    def run(env, m):
        nonlocal n
        ps = None if projectors is None else projectors[4 * n: 4 * n + 4]
        n += 1
        return sweep(env, a, chi, renormalize, m, dense, ps, rec)

    if method == "qr" and warmup > 0:
        w = min(warmup, max_iter)
        for _ in range(w):
            env = run(env, "eigh")
        max_iter -= w
    prev = None
    for _ in range(max_iter):
        env = run(env, method)
        sv = np.linalg.svd(todense(env["C1"]), compute_uv=False)
        if prev is not None and sv_diff(sv, prev) < conv_tol:
            break
        prev = sv
    return env


CHECKERBOARD = {(0, 0): {d: (1, 0) for d in DIRECTIONS}, (1, 0): {d: (0, 0) for d in DIRECTIONS}}


def ctm_tensor_multisite(sites: dict, neighbors: dict, chi, max_iter=100, conv_tol=1e-8, renormalize=True,
                         method="eigh", warmup=3, dense=False, projectors=None, rec=None):
    """Multisite sweeps: per direction, every site in sorted order moves with
    its neighbour's environment and double layer (_ctm_tensor.py:836-858,
    :920-974).  ``projectors``: flat list in call order."""
    dls = {c: double_layer(A) for c, A in sites.items()}
    envs = {c: init_env(A, chi, dense) for c, A in sites.items()}
    it = iter(projectors) if projectors is not None else None

    def run(envs, m):
        for dr in DIRECTIONS:
            for c in sorted(envs):
                nb = neighbors[c][dr]
                envs[c] = move(envs[c], envs[nb], dls[nb], chi, m, dr, dense,
                               None if it is None else next(it), rec)
        if renormalize:
            envs = {c: {k: normalize(v) for k, v in e.items()} for c, e in envs.items()}
        return envs

    if method == "qr" and warmup > 0:
        w = min(warmup, max_iter)
        for _ in range(w):
            envs = run(envs, "eigh")
        max_iter -= w
    prev: dict = {}
    for _ in range(max_iter):
        envs = run(envs, method)
        conv = True
        for c in sorted(envs):
            sv = np.linalg.svd(todense(envs[c]["C1"]), compute_uv=False)
            if c not in prev or sv_diff(sv, prev[c]) >= conv_tol:
                conv = False
            prev[c] = sv
        if conv:
            break
    return envs


# ---------------------------------------------------------------------------
# energy
# ---------------------------------------------------------------------------

def dense_env(env: dict):
    """(_ctm_tensor.py:1021-1034)"""
    return tuple(torch.from_numpy(todense(env[k])) for k in FIELDS)


def energy(A: OTensor, env: dict, H, d: int) -> float:
    """Densify and evaluate the dense CTM energy (_ctm_tensor.py:1037-1069)."""
    Ad = torch.from_numpy(todense(A))
    Ht = torch.as_tensor(np.asarray(H, dtype=np.float64)).reshape(d, d, d, d)
    with torch.no_grad():
        return float(dense_ctm.energy(Ad, dense_env(env), Ht, d))


def energy_2site(A: OTensor, B: OTensor, env_A: dict, env_B: dict, H, d: int) -> float:
    """(_ctm_tensor.py:1072-1109 -> ipeps.py:1552-1662)"""
    Ad, Bd = torch.from_numpy(todense(A)), torch.from_numpy(todense(B))
    Ht = torch.as_tensor(np.asarray(H, dtype=np.float64)).reshape(d, d, d, d)
    with torch.no_grad():
        return float(dense_ctm.energy_2site(Ad, Bd, dense_env(env_A), dense_env(env_B), Ht, d))


def site_tensor(D, bond_charges, phys_charges, seed, modulus=None) -> OTensor:
    """Site tensor (u, d, l, r, phys) with flows (OUT, IN, OUT, IN, IN),
    N(0,1) blocks over the valid keys in sorted order from numpy's seeded
    generator."""
    rng = np.random.default_rng(seed)
    b = np.asarray(bond_charges, np.int32)
    p = np.asarray(phys_charges, np.int32)
    legs = (Leg(b, OUT, "u"), Leg(b.copy(), IN, "d"), Leg(b.copy(), OUT, "l"), Leg(b.copy(), IN, "r"),
            Leg(p, IN, "phys"))
    blocks = {}
    for k in sorted(valid_blocks([l.charges for l in legs], [l.flow for l in legs], modulus)):
        shp = block_shape([l.charges for l in legs], k)
        if all(s > 0 for s in shp):
            blocks[k] = rng.standard_normal(shp)
    return OTensor(legs, blocks, modulus)
