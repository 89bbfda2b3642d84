"""Float64 restatement of tenax's U(1) split-CTMRG (ket and bra layers kept
apart), with its energy.

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).  Follows
``algorithms/_split_ctm_tensor.py``; torch CPU float64, so autograd gives the
reverse-mode gradient with the projectors detached (the reference's
``stop_gradient``, :448).

Symmetric tensors are carried in dense form.  This is exact for the
reference's operations:
  * every ``SymmetricTensor.from_dense(..., tol=inf)`` re-wrap with
    charge-tiled legs (:1082-1181, :147-248) keeps the charge-conserving
    entries and drops the rest, so it is a multiplication by the 0/1 mask of
    the legs' charges and flows;
  * a symmetric contraction of conserving operands equals the dense
    contraction of their dense forms;
  * ``fuse_indices(...).todense()`` (:522-541 etc.) is the natural reshape
    with rows moved by ``oracle.blocksparse.fused_row_map``.
Each move keeps the reference's order of operations, including the dense
grown edge of shape (chi D^2, D^2, chi D^2) (:464-504) and the
three-factor projection ``einsum("ia,idj,jb->adb")``.

Every projector and every edge-split SVD can be supplied (replay): a run
given the reference's recorded ones reproduces its environments to rounding.
"""

from __future__ import annotations

import math

import numpy as np
import torch

from oracle.blocksparse import Leg, fused_row_map

EPS = 1e-15  # tenax core/__init__.py:15
LOG_EPS = 1e-250  # tenax core/__init__.py:16

NAMES = ("C1", "C2", "C3", "C4", "T1_ket", "T1_bra", "T2_ket", "T2_bra", "T3_ket", "T3_bra", "T4_ket", "T4_bra")
IN, OUT = 1, -1

# leg flows and the site-tensor axis the chi/I charges (and, for edges, the
# D charges) are tiled from (_split_ctm_tensor.py:260-355)
CORNERS = {"C1": ((IN, OUT), 1), "C2": ((IN, OUT), 0), "C3": ((OUT, IN), 1), "C4": ((OUT, IN), 0)}
KET = {"T1": ((IN, IN, OUT), 3, 0), "T2": ((OUT, OUT, IN), 0, 3), "T3": ((OUT, OUT, IN), 3, 1),
       "T4": ((IN, IN, OUT), 1, 2)}
BRA = {"T1": ((IN, OUT, IN), 3, 0), "T2": ((OUT, IN, OUT), 0, 3), "T3": ((OUT, IN, OUT), 3, 1),
       "T4": ((IN, OUT, IN), 1, 2)}


def derive_charges(base, n):
    """Tile the base charges to length n (_split_ctm_tensor.py:251-257)."""
    base = np.asarray(base, dtype=np.int32)
    if n <= len(base):
        return base[:n].copy()
    return np.tile(base, n // len(base) + 1)[:n].astype(np.int32)


class Site:
    """Site tensor A[u, d, l, r, s] (dense float64) with its leg charges and
    flows; the bra layer is A with all flows reversed (``bar()``)."""

    def __init__(self, dense, charges, flows, modulus=None):
        self.A = dense
        self.charges = [np.asarray(c, dtype=np.int32) for c in charges]
        self.flows = list(flows)
        self.modulus = modulus
        self.D = dense.shape[0]
        self.d = dense.shape[4]


def env_legs(site: Site, chi: int, chi_I: int) -> dict:
    """(charges, flows) of every environment leg; fixed for the whole run
    because every re-wrap tiles the same base charges (:1082-1181)."""
    q = site.charges
    legs = {}
    for name, (fl, ref) in CORNERS.items():
        c = derive_charges(q[ref], chi)
        legs[name] = [(c, fl[0]), (c.copy(), fl[1])]
    for name, (fl, rc, rd) in KET.items():
        legs[name + "_ket"] = [(derive_charges(q[rc], chi), fl[0]), (q[rd].copy(), fl[1]),
                               (derive_charges(q[rc], chi_I), fl[2])]
    for name, (fl, rc, rd) in BRA.items():
        legs[name + "_bra"] = [(derive_charges(q[rc], chi_I), fl[0]), (q[rd].copy(), fl[1]),
                               (derive_charges(q[rc], chi), fl[2])]
    return legs


def charge_mask(legs, modulus=None) -> torch.Tensor:
    """1 where sum(flow * charge) is the identity, else 0."""
    tot = np.zeros([len(c) for c, _ in legs], dtype=np.int64)
    for ax, (c, f) in enumerate(legs):
        shp = [1] * len(legs)
        shp[ax] = len(c)
        tot = tot + int(f) * np.asarray(c, dtype=np.int64).reshape(shp)
    if modulus is not None:
        tot = np.mod(tot, modulus)
    return torch.from_numpy((tot == 0).astype(np.float64))


def init_env(site: Site, chi: int, chi_I: int):
    """Identity corners and identity-like edges, masked (:147-248, :358-428)."""
    legs = env_legs(site, chi, chi_I)
    D = site.D
    env = {}
    for n in ("C1", "C2", "C3", "C4"):
        env[n] = torch.eye(chi, dtype=torch.float64) * charge_mask(legs[n], site.modulus)
    m = min(min(chi, D), min(chi_I, D))
    for n in ("T1", "T2", "T3", "T4"):
        tk = torch.zeros(chi, D, chi_I, dtype=torch.float64)
        tb = torch.zeros(chi_I, D, chi, dtype=torch.float64)
        for i in range(m):
            tk[i, :, i] = 1.0
            tb[i, :, i] = 1.0
        env[n + "_ket"] = tk * charge_mask(legs[n + "_ket"], site.modulus)
        env[n + "_bra"] = tb * charge_mask(legs[n + "_bra"], site.modulus)
    return env, legs


def projector(C1g, C2g, chi):
    """Leading eigenvectors of C1g C1g^H + C2g C2g^H (:431-449)."""
    rho = C1g @ C1g.conj().T + C2g @ C2g.conj().T
    rho = 0.5 * (rho + rho.conj().T)
    _, vecs = torch.linalg.eigh(rho)
    k = min(chi, vecs.shape[0])
    return vecs[:, -k:].flip(1)


def fuse_dense(x, ax_a, ax_b, leg_a, leg_b, modulus):
    """fuse_indices(x, ax_a, ax_b, IN).todense() for a 3-leg grown corner
    whose remaining leg is the last one: rows = fused legs, cols = last."""
    other = [i for i in range(3) if i not in (ax_a, ax_b)][0]
    nat = x.permute(ax_a, ax_b, other).reshape(x.shape[ax_a] * x.shape[ax_b], x.shape[other])
    m = fused_row_map(Leg(leg_a[0], leg_a[1]), Leg(leg_b[0], leg_b[1]), IN, modulus)
    inv = np.empty_like(m)
    inv[m] = np.arange(len(m))
    return nat[torch.from_numpy(inv)]


# Lorentzian width of the broadened SVD adjoint (algorithms/ad_utils.py:80)
BROADENING = 1e-12


class BroadenedSVD(torch.autograd.Function):
    """Thin SVD whose reverse pass stays finite on degenerate spectra.

    The reference differentiates ``jnp.linalg.svd`` and ``jnp.sqrt`` directly
    (:1069-1071).  The first moves of every split CTM start from an
    identity-like environment whose edges have exactly degenerate pairs and
    exactly zero kept singular values, so that reverse pass is NaN there.
    This adjoint is the one a finite gradient of the fixed-projector energy
    needs.  It is Townsend's reverse mode ("Differentiating the singular value
    decomposition", 2016) over all min(m, n) triplets.  The factor
    1/(s_j^2 - s_i^2) is replaced by the Lorentzian d/(d^2 + eps^2),
    d = s_j^2 - s_i^2, with the reference's eps (Francuz et al., PRR 7,
    013237).  The caller truncates by slicing, so the coupling to the
    discarded triplets is exact."""

    @staticmethod
    def forward(ctx, A):
        U, s, Vh = torch.linalg.svd(A, full_matrices=False)
        ctx.save_for_backward(U, s, Vh)
        return U, s, Vh

    @staticmethod
    def backward(ctx, dU, ds, dVh):
        U, s, Vh = ctx.saved_tensors
        V = Vh.T
        m, n, r = U.shape[0], V.shape[0], s.shape[0]
        dU = torch.zeros_like(U) if dU is None else dU
        ds = torch.zeros_like(s) if ds is None else ds
        dV = torch.zeros_like(V) if dVh is None else dVh.T
        d = s[None, :] ** 2 - s[:, None] ** 2
        F = d / (d * d + BROADENING ** 2)
        F = F * (1.0 - torch.eye(r, dtype=s.dtype))
        a = U.T @ dU
        b = V.T @ dV
        inner = (F * (a - a.T)) @ torch.diag(s) + torch.diag(ds) + torch.diag(s) @ (F * (b - b.T))
        dA = U @ inner @ Vh
        s_inv = torch.where(s > BROADENING, 1.0 / s, torch.zeros_like(s))
        if m > r:
            dA = dA + ((dU - U @ a) @ torch.diag(s_inv)) @ Vh
        if n > r:
            dA = dA + U @ (torch.diag(s_inv) @ (dV - V @ b).T)
        return dA


class SqrtZeroSafe(torch.autograd.Function):
    """sqrt(s) with derivative 0 at s == 0: the exactly zero singular values
    of the first moves stay zero for every site tensor."""

    @staticmethod
    def forward(ctx, s):
        r = torch.sqrt(s)
        ctx.save_for_backward(r)
        return r

    @staticmethod
    def backward(ctx, g):
        (r,) = ctx.saved_tensors
        safe = torch.where(r > 0, r, torch.ones_like(r))
        return torch.where(r > 0, g / (2.0 * safe), torch.zeros_like(g))


def svd_split(T_full, chi_I, usv=None, broadened=False):
    """(chi, D^2, chi) -> ket (chi, D, k), bra (k, D, chi) (:1058-1074).

    ``broadened`` differentiates through ``BroadenedSVD`` and ``SqrtZeroSafe``
    instead of the plain SVD and sqrt; the forward values are the same."""
    chi, D2 = T_full.shape[0], T_full.shape[1]
    D = math.isqrt(D2)
    T_mat = T_full.reshape(chi, D, D, chi).reshape(chi * D, D * chi)
    if usv is not None:
        U, s, Vh = usv
    elif broadened:
        U, s, Vh = BroadenedSVD.apply(T_mat)
    else:
        U, s, Vh = torch.linalg.svd(T_mat, full_matrices=False)
    k = min(chi_I, s.shape[0])
    r = SqrtZeroSafe.apply(s[:k]) if broadened else torch.sqrt(s[:k])
    return (U[:, :k] * r[None, :]).reshape(chi, D, k), (r[:, None] * Vh[:k, :]).reshape(k, D, chi)


# Per move: first layer ("ket"/"bra"), corner growth subscripts and the
# axes of the fusion, the mid-corner growth with the second layer, the
# combined-projector subscripts, edge name, contracted site leg, and the
# dense output order of the grown edge (reference labels) as site-leg names.
MOVES = {
    "left": dict(first="ket", c1=("C1", "T1_ket", "ab,bux->aux", (0, 1)), c2=("C4", "T3_ket", "ba,bdx->adx", (0, 1)),
                 m1=("T1_bra", "ac,cdb->adb"), m2=("T3_bra", "ac,cdb->adb"), pf="auJ,JUb->auUb",
                 edge="T4", leg="l", out=("x", "u", "U", "r", "R", "y", "d", "D"), new=("C1", "C4")),
    "right": dict(first="bra", c1=("C2", "T1_bra", "ba,xub->axu", (0, 2)), c2=("C3", "T3_bra", "ab,xdb->axd", (0, 2)),
                  m1=("T1_ket", "af,buf->aub"), m2=("T3_ket", "af,hdf->adh"), pf="aUJ,Jub->auUb",
                  edge="T2", leg="r", out=("x", "u", "U", "l", "L", "y", "d", "D"), new=("C2", "C3")),
    "top": dict(first="ket", c1=("C1", "T4_ket", "ba,blx->alx", (0, 1)), c2=("C2", "T2_ket", "ab,brx->arx", (0, 1)),
                m1=("T4_bra", "ac,cdb->adb"), m2=("T2_bra", "ac,cdb->adb"), pf="auJ,JUb->auUb",
                edge="T1", leg="u", out=("x", "l", "L", "d", "D", "y", "r", "R"), new=("C1", "C2")),
    "bottom": dict(first="bra", c1=("C4", "T4_bra", "ab,xlb->axl", (0, 2)), c2=("C3", "T2_bra", "ba,xrb->axr", (0, 2)),
                   m1=("T4_ket", "af,blf->alb"), m2=("T2_ket", "af,erf->are"), pf="aUJ,Jub->auUb",
                   edge="T3", leg="d", out=("x", "l", "L", "u", "U", "y", "r", "R"), new=("C4", "C3")),
}
ORDER = ("left", "right", "top", "bottom")
_SITE = "udlr"


def corner_fused_legs(name, legs):
    """Charges/flows of the two fused legs of a move's grown corners: the
    corner's free leg and the edge's D leg (in grown-corner order)."""
    mv = MOVES[name]
    out = []
    for cname, ename, subs, (fa, fb) in (mv["c1"], mv["c2"]):
        lhs, o = subs.split("->")
        sc, se = lhs.split(",")
        src = {}
        for ch, lg in zip(sc, legs[cname]):
            src[ch] = lg
        for ch, lg in zip(se, legs[ename]):
            src.setdefault(ch, lg) if ch in sc else src.__setitem__(ch, lg)
        out.append((src[o[fa]], src[o[fb]]))
    return out


def grow_edge(site: Site, T_ket, T_bra, leg, out_order):
    """Dense grown edge (chi D^2, D^2, chi D^2) from the separate layers
    (_split_ctm_tensor.py:464-504): ket = T_ket . A over the site leg,
    bra = T_bra . A over the same leg, summed over the interlayer bond and
    the physical index."""
    free = [c for c in _SITE if c != leg]
    ks = "x" + leg + "I"
    kA = "".join(leg if c == leg else c for c in _SITE) + "s"
    bs = "I" + leg.upper() + "y"
    bA = "".join(leg.upper() if c == leg else c.upper() for c in _SITE) + "s"
    ket = torch.einsum(f"{ks},{kA}->xI{''.join(free)}s", T_ket, site.A)
    bra = torch.einsum(f"{bs},{bA}->Iy{''.join(c.upper() for c in free)}s", T_bra, site.A)
    g = torch.einsum(f"xI{''.join(free)}s,Iy{''.join(c.upper() for c in free)}s->{''.join(out_order)}", ket, bra)
    chi, D = T_ket.shape[0], site.D
    return g.reshape(chi * D * D, D * D, chi * D * D)


def move(env, legs, site: Site, name, chi, chi_I, projectors=None, svds=None, rec_p=None, rec_svd=None,
         broadened=False):
    """One directional move (_split_ctm_tensor.py:512-1050)."""
    mv = MOVES[name]
    mod = site.modulus
    (c1n, e1n, s1, (a1, b1)), (c2n, e2n, s2, (a2, b2)) = mv["c1"], mv["c2"]
    (fl1a, fl1b), (fl2a, fl2b) = corner_fused_legs(name, legs)
    g1 = fuse_dense(torch.einsum(s1, env[c1n], env[e1n]), a1, b1, fl1a, fl1b, mod)
    g2 = fuse_dense(torch.einsum(s2, env[c2n], env[e2n]), a2, b2, fl2a, fl2b, mod)
    P1 = (projectors.pop(0) if projectors else projector(g1.detach(), g2.detach(), chi)).detach()
    mid1, mid2 = P1.conj().T @ g1, P1.conj().T @ g2
    h1 = torch.einsum(mv["m1"][1], mid1, env[mv["m1"][0]]).reshape(-1, chi)
    h2 = torch.einsum(mv["m2"][1], mid2, env[mv["m2"][0]]).reshape(-1, chi)
    P2 = (projectors.pop(0) if projectors else projector(h1.detach(), h2.detach(), chi)).detach()
    if rec_p is not None:
        rec_p.extend([P1, P2])
    new = dict(env)
    for cn, h in zip(mv["new"], (h1, h2)):
        new[cn] = (P2.conj().T @ h) * charge_mask(legs[cn], mod)
    D = site.D
    P1_3 = P1.reshape(chi, D, -1)
    P2_3 = P2.reshape(P1_3.shape[2], D, -1)
    Pf = torch.einsum(mv["pf"], P1_3, P2_3)
    Pf = Pf.reshape(chi * D * D, Pf.shape[3])
    e = mv["edge"]
    Tg = grow_edge(site, env[e + "_ket"], env[e + "_bra"], mv["leg"], mv["out"])
    Tn = torch.einsum("ia,idj,jb->adb", Pf, Tg, Pf)
    usv = svds.pop(0) if svds else None
    tk, tb = svd_split(Tn, chi_I, usv, broadened)
    if rec_svd is not None:
        rec_svd.append(Tn.detach())
    new[e + "_ket"] = tk * charge_mask(legs[e + "_ket"], mod)
    new[e + "_bra"] = tb * charge_mask(legs[e + "_bra"], mod)
    return new


def renormalize(env):
    """Corners by their max-abs (+LOG_EPS); each ket/bra pair by the
    geometric mean of their max-abs (+EPS) (:1209-1240)."""
    out = dict(env)
    for n in ("C1", "C2", "C3", "C4"):
        out[n] = env[n] * (1.0 / (env[n].abs().max() + LOG_EPS))
    for n in ("T1", "T2", "T3", "T4"):
        k, b = env[n + "_ket"], env[n + "_bra"]
        shared = torch.sqrt(k.abs().max() * b.abs().max()) + EPS
        out[n + "_ket"] = k * (1.0 / shared)
        out[n + "_bra"] = b * (1.0 / shared)
    return out


def ctm_split(site: Site, chi, iters, chi_I=None, projectors=None, svds=None, rec_p=None, broadened=False):
    """Fixed-count split CTM (ctm_split_tensor with conv_tol=0, :1243-1289).
    ``broadened``: the edge split's reverse pass through ``BroadenedSVD``."""
    chi_I = chi if chi_I is None else chi_I
    env, legs = init_env(site, chi, chi_I)
    ps = list(projectors) if projectors is not None else None
    sv = list(svds) if svds is not None else None
    for _ in range(iters):
        for name in ORDER:
            env = move(env, legs, site, name, chi, chi_I, ps, sv, rec_p, broadened=broadened)
        env = renormalize(env)
    return env


def to_standard(env):
    """Ket/bra edges merged over the interlayer bond (:1292-1313)."""
    chi = env["C1"].shape[0]

    def merge(k, b):
        D = k.shape[1]
        return torch.einsum("auc,cUb->auUb", k, b).reshape(chi, D * D, chi)

    return (env["C1"], env["C2"], env["C3"], env["C4"], merge(env["T1_ket"], env["T1_bra"]),
            merge(env["T2_ket"], env["T2_bra"]), merge(env["T3_ket"], env["T3_bra"]),
            merge(env["T4_ket"], env["T4_bra"]))


def energy(site: Site, env, H):
    """compute_energy_split_ctm_tensor (:1316-1351) via the dense energy."""
    from oracle.ctm import energy as dense_energy

    return dense_energy(site.A, to_standard(env), H, site.d)
