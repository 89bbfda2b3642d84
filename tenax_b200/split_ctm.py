"""U(1) split-CTMRG on the GPU (ket and bra layers kept apart).

Same function as tenax ``algorithms/_split_ctm_tensor.py``
(``ctm_split_tensor`` :1243-1289, ``compute_energy_split_ctm_tensor``
:1316-1351, ``SplitCTMTensorEnv`` :37-56), on float64 CUDA tensors.

Representation.  The reference re-wraps every new corner and edge with
``SymmetricTensor.from_dense(..., tol=inf)`` over legs whose charges are A's
bond charges tiled to chi / chi_I (:251-257, :1082-1181): the tensor keeps
exactly the charge-conserving entries.  Those leg charges never change, so
each environment tensor is held here in dense form and the re-wrap is a
product with its fixed 0/1 charge mask; a symmetric contraction of such
operands is the dense contraction of their dense forms.  Growing a corner
fuses two legs and densifies the result (``fuse_indices(..).todense()``,
:522-541); that is the natural reshape with rows moved by the fused-row map
the library's planner computes (``tnx_fuse_row_map``, integer-exact against
the reference).  So every move is a short chain of dense contractions on the
library's engine (FP64 DMMA or split-BF16x3 / TF32 tcgen05), projectors and
the edge SVD in FP64 through cuSOLVER, and a few masked products.

The grown edge (chi D^2, D^2, chi D^2) of the reference (:464-504) is never
formed: with P the combined projector (chi D^2, chi),

    T'[A,(m,M),B] = sum P[x,r,R,A] ket[x,I,{r,c,m},s] bra[I,y,{R,C,M},s] P[y,c,C,B]

is evaluated as P.ket, then .bra (over R, I, s), then .P -- 55 GFLOP per
move at D=5, chi=150 instead of 105, and 112 MB of intermediate instead of
2.8 GB.  ket = T_ket.A and bra = T_bra.A contract one site leg each.

Differentiation.  Everything except the projectors (held fixed: the
reference's stop_gradient, :448) is differentiable: engine contractions
carry their hand-written adjoints (``tenax_b200.dense.Contract``), the masks
and row moves are linear, and the edge split has a hand-written SVD adjoint
that stays finite on the degenerate spectra the identity-like initial
environment produces (``_SVD``).
``checkpoint_every`` recomputes groups of sweeps in the backward pass.
"""

from __future__ import annotations

import ctypes as C
import math
from typing import NamedTuple

import numpy as np
import torch
import torch.utils.checkpoint

from tenax_b200 import _capi
from tenax_b200.dense import contract, einsum
from tenax_b200.ipeps import CTMEnvironment, compute_energy_ctm
from tenax_b200.linalg import POLAR_MIN, svd as linalg_svd

EPS = 1e-15  # tenax core/__init__.py:15
LOG_EPS = 1e-250  # tenax core/__init__.py:16
IN, OUT = 1, -1


class SplitCTMTensorEnv(NamedTuple):
    """Corners (chi, chi); ket edges (chi, D, chi_I); bra edges (chi_I, D, chi)
    (_split_ctm_tensor.py:37-56).  Dense CUDA tensors, zero outside the
    charge-conserving blocks of the tiled leg charges."""

    C1: torch.Tensor
    C2: torch.Tensor
    C3: torch.Tensor
    C4: torch.Tensor
    T1_ket: torch.Tensor
    T1_bra: torch.Tensor
    T2_ket: torch.Tensor
    T2_bra: torch.Tensor
    T3_ket: torch.Tensor
    T3_bra: torch.Tensor
    T4_ket: torch.Tensor
    T4_bra: torch.Tensor


_FIELDS = SplitCTMTensorEnv._fields
# leg flows of each environment tensor and the site axis whose charges its
# chi / chi_I legs (and, for edges, its D leg) carry (_split_ctm_tensor.py:260-355)
_CORNER = {"C1": ((IN, OUT), 1), "C2": ((IN, OUT), 0), "C3": ((OUT, IN), 1), "C4": ((OUT, IN), 0)}
_KET = {"T1": ((IN, IN, OUT), 3, 0), "T2": ((OUT, OUT, IN), 0, 3), "T3": ((OUT, OUT, IN), 3, 1),
        "T4": ((IN, IN, OUT), 1, 2)}
_BRA = {"T1": ((IN, OUT, IN), 3, 0), "T2": ((OUT, IN, OUT), 0, 3), "T3": ((OUT, IN, OUT), 3, 1),
        "T4": ((IN, OUT, IN), 1, 2)}

# Per move (:512-1050): which layer is absorbed first, the two corner
# growths (corner, edge, dense subscripts, fused axes), the growths of the
# mid-corners with the other layer, the combined-projector subscripts, the
# edge and its contracted site leg, the site legs of the edge's rows / middle /
# columns (lower case: ket layer, upper: bra), and the corners replaced.
_MOVES = (
    dict(c1=("C1", "T1_ket", "ab,bux->aux", (0, 1)), c2=("C4", "T3_ket", "ba,bdx->adx", (0, 1)),
         m1=("T1_bra", "ac,cdb->adb"), m2=("T3_bra", "ac,cdb->adb"), pf="auJ,JUb->auUb",
         edge="T4", leg="l", rows="uU", mid="rR", cols="dD", new=("C1", "C4")),
    dict(c1=("C2", "T1_bra", "ba,xub->axu", (0, 2)), c2=("C3", "T3_bra", "ab,xdb->axd", (0, 2)),
         m1=("T1_ket", "af,buf->aub"), m2=("T3_ket", "af,hdf->adh"), pf="aUJ,Jub->auUb",
         edge="T2", leg="r", rows="uU", mid="lL", cols="dD", new=("C2", "C3")),
    dict(c1=("C1", "T4_ket", "ba,blx->alx", (0, 1)), c2=("C2", "T2_ket", "ab,brx->arx", (0, 1)),
         m1=("T4_bra", "ac,cdb->adb"), m2=("T2_bra", "ac,cdb->adb"), pf="auJ,JUb->auUb",
         edge="T1", leg="u", rows="lL", mid="dD", cols="rR", new=("C1", "C2")),
    dict(c1=("C4", "T4_bra", "ab,xlb->axl", (0, 2)), c2=("C3", "T2_bra", "ba,xrb->axr", (0, 2)),
         m1=("T4_ket", "af,blf->alb"), m2=("T2_ket", "af,erf->are"), pf="aUJ,Jub->auUb",
         edge="T3", leg="d", rows="lL", mid="uU", cols="rR", new=("C4", "C3")),
)
_SITE = "udlr"


def _derive(base, n):
    """A's charges tiled to length n (_split_ctm_tensor.py:251-257)."""
    base = np.asarray(base, dtype=np.int32)
    return base[:n].copy() if n <= len(base) else np.tile(base, n // len(base) + 1)[:n].astype(np.int32)


class _Structure:
    """Leg charges/flows, charge masks and fused-row moves of one run."""

    def __init__(self, charges, flows, modulus, chi, chi_I, device):
        self.modulus = modulus
        q = [np.asarray(c, dtype=np.int32) for c in charges]
        self.legs = {}
        for n, (fl, ref) in _CORNER.items():
            c = _derive(q[ref], chi)
            self.legs[n] = [(c, fl[0]), (c, fl[1])]
        for n, (fl, rc, rd) in _KET.items():
            self.legs[n + "_ket"] = [(_derive(q[rc], chi), fl[0]), (q[rd], fl[1]), (_derive(q[rc], chi_I), fl[2])]
        for n, (fl, rc, rd) in _BRA.items():
            self.legs[n + "_bra"] = [(_derive(q[rc], chi_I), fl[0]), (q[rd], fl[1]), (_derive(q[rc], chi), fl[2])]
        self.mask = {n: self._mask(self.legs[n], device) for n in _FIELDS}
        self.moves = []
        for mv in _MOVES:
            inv = []
            for cname, ename, subs, (fa, fb) in (mv["c1"], mv["c2"]):
                lhs, o = subs.split("->")
                sc, se = lhs.split(",")
                src = dict(zip(se, self.legs[ename]))
                src.update(zip(sc, self.legs[cname]))
                inv.append(self._row_move(src[o[fa]], src[o[fb]], device))
            self.moves.append(inv)

    def _mask(self, legs, device):
        tot = np.zeros([len(c) for c, _ in legs], dtype=np.int64)
        for ax, (c, f) in enumerate(legs):
            shp = [1] * len(legs)
            shp[ax] = len(c)
            tot = tot + int(f) * c.astype(np.int64).reshape(shp)
        if self.modulus is not None:
            tot = np.mod(tot, self.modulus)
        return torch.from_numpy((tot == 0).astype(np.float64)).to(device)

    def _row_move(self, leg_a, leg_b, device):
        (qa, fa), (qb, fb) = leg_a, leg_b
        qa, qb = np.ascontiguousarray(qa, np.int32), np.ascontiguousarray(qb, np.int32)
        m = np.zeros(len(qa) * len(qb), dtype=np.int64)
        _capi.check(_capi.LIB.tnx_fuse_row_map(qa.ctypes.data, len(qa), int(fa), qb.ctypes.data, len(qb), int(fb), IN,
                                               0 if self.modulus is None else int(self.modulus), m.ctypes.data))
        inv = np.empty_like(m)
        inv[m] = np.arange(len(m))
        return torch.from_numpy(inv).to(device)


def _site(A):
    """(dense A on the GPU, leg charges, leg flows, modulus) of a site tensor:
    a tenax_b200 SymmetricTensor, or a dense array (trivial charges)."""
    from tenax_b200.tensor import SymmetricTensor

    if isinstance(A, SymmetricTensor):
        if A.ndim != 5:
            raise ValueError("split CTM takes 5-leg site tensors (u, d, l, r, phys)")
        return (A.todense(), [i.charges for i in A.indices], [int(i.flow) for i in A.indices],
                A.indices[0].symmetry.n_values())
    a = A if isinstance(A, torch.Tensor) else torch.as_tensor(np.asarray(A, dtype=np.float64))
    a = a.to(device="cuda", dtype=torch.float64)
    if a.ndim != 5:
        raise ValueError("split CTM takes 5-leg site tensors (u, d, l, r, phys)")
    return a, [np.zeros(n, np.int32) for n in a.shape], [OUT, IN, OUT, IN, IN], None


def initialize_split_ctm_tensor_env(A, chi: int, chi_I: int) -> SplitCTMTensorEnv:
    """Identity corners and identity-like edges (_split_ctm_tensor.py:358-428)."""
    a, q, f, mod = _site(A)
    S = _Structure(q, f, mod, chi, chi_I, a.device)
    return _init(S, a.shape[0], chi, chi_I, a.device)


def _init(S: _Structure, D, chi, chi_I, dev) -> SplitCTMTensorEnv:
    env = {}
    for n in ("C1", "C2", "C3", "C4"):
        env[n] = torch.eye(chi, dtype=torch.float64, device=dev) * S.mask[n]
    m = min(min(chi, D), min(chi_I, D))
    idx = torch.arange(m, device=dev)
    for n in ("T1", "T2", "T3", "T4"):
        tk = torch.zeros(chi, D, chi_I, dtype=torch.float64, device=dev)
        tb = torch.zeros(chi_I, D, chi, dtype=torch.float64, device=dev)
        tk[idx, :, idx] = 1.0
        tb[idx, :, idx] = 1.0
        env[n + "_ket"] = tk * S.mask[n + "_ket"]
        env[n + "_bra"] = tb * S.mask[n + "_bra"]
    return SplitCTMTensorEnv(**env)


def _projector(g1, g2, chi):
    """Leading eigenvectors of g1 g1^T + g2 g2^T (_split_ctm_tensor.py:431-449), FP64."""
    with torch.no_grad():
        rho = einsum("ij,kj->ik", g1, g1) + einsum("ij,kj->ik", g2, g2)
        rho = 0.5 * (rho + rho.T)
        _, vecs = torch.linalg.eigh(rho)
        k = min(chi, vecs.shape[0])
        return vecs[:, -k:].flip(1).contiguous()


def _fuse_rows(x, axes, inv):
    """fuse_indices(x, *axes, IN).todense() of a 3-leg grown corner."""
    a, b = axes
    other = 3 - a - b
    nat = x.permute(a, b, other).reshape(x.shape[a] * x.shape[b], x.shape[other])
    return nat.index_select(0, inv)


SVD_BROADENING = 1e-12


class _SVD(torch.autograd.Function):
    """Reduced SVD A = U diag(s) V^T (FP64, the library's cuSOLVER polar or
    Jacobi SVD) with a reverse pass that stays finite on degenerate spectra.

    Reverse mode of the SVD (Townsend, "Differentiating the singular value
    decomposition", 2016), over all min(m, n) singular triplets:

        A_bar = U [ (F o (U^T U_bar - U_bar^T U)) S + diag(s_bar)
                    + S (F o (V^T V_bar - V_bar^T V)) ] V^T
                + (I - U U^T) U_bar S^+ V^T  (m > n)
                + U S^+ V_bar^T (I - V V^T)  (n > m)

    with F_ij = 1/(s_j^2 - s_i^2) replaced by the Lorentzian
    D/(D^2 + eps^2), D = s_j^2 - s_i^2 (Francuz et al., PRR 7, 013237), so
    exactly degenerate pairs contribute nothing instead of 0/0.  For a loss
    invariant under rotations inside a degenerate subspace those terms
    vanish anyway, so the gradient is exact there too.  Truncation is done
    by the caller slicing the outputs: discarded triplets are coupled
    exactly through F."""

    @staticmethod
    def forward(ctx, A, polar_min=POLAR_MIN):
        if int(torch.count_nonzero(A)) == 0:
            # the zero edge of a collapsed environment (the U(1) runs): any
            # orthonormal U, V; this one costs nothing (a polar decomposition
            # of a zero matrix is slow)
            m, n = A.shape
            r = min(m, n)
            U = torch.eye(m, r, dtype=A.dtype, device=A.device)
            s = torch.zeros(r, dtype=A.dtype, device=A.device)
            Vh = torch.eye(r, n, dtype=A.dtype, device=A.device)
        else:
            U, s, Vh = linalg_svd(A, polar_min)
        ctx.save_for_backward(U, s, Vh)
        ctx.shape = A.shape
        return U, s, Vh

    @staticmethod
    def backward(ctx, gU, gs, gVh):
        U, s, Vh = ctx.saved_tensors
        m, n = ctx.shape
        V = Vh.T
        k = s.shape[0]
        gU = torch.zeros_like(U) if gU is None else gU
        gs = torch.zeros_like(s) if gs is None else gs
        gV = torch.zeros_like(V) if gVh is None else gVh.T
        s2 = s * s
        Dm = s2[None, :] - s2[:, None]
        F = Dm / (Dm * Dm + SVD_BROADENING ** 2)
        F.fill_diagonal_(0.0)
        UtgU = einsum("mi,mj->ij", U.contiguous(), gU.contiguous())
        VtgV = einsum("ni,nj->ij", V.contiguous(), gV.contiguous())
        J = (F * (UtgU - UtgU.T)) * s[None, :] + torch.diag(gs) + s[:, None] * (F * (VtgV - VtgV.T))
        gA = einsum("mi,ij->mj", U.contiguous(), J.contiguous())
        gA = einsum("mj,nj->mn", gA, V.contiguous())
        sinv = torch.where(s > SVD_BROADENING, 1.0 / s, torch.zeros_like(s))
        if m > k:
            X = gU - einsum("mi,ij->mj", U.contiguous(), UtgU.contiguous())
            gA = gA + einsum("mj,nj->mn", (X * sinv[None, :]).contiguous(), V.contiguous())
        if n > k:
            Y = gV - einsum("ni,ij->nj", V.contiguous(), VtgV.contiguous())
            gA = gA + einsum("mj,nj->mn", (U * sinv[None, :]).contiguous(), Y.contiguous())
        return gA, None


class _SqrtSV(torch.autograd.Function):
    """sqrt of singular values whose derivative is 0 where s == 0: zero
    singular values of the split edges are structural (the identity-like
    initial environment has rank deficits that hold for every site tensor),
    so they do not move and contribute no gradient."""

    @staticmethod
    def forward(ctx, s):
        r = torch.sqrt(s)
        ctx.save_for_backward(r)
        return r

    @staticmethod
    def backward(ctx, g):
        (r,) = ctx.saved_tensors
        return torch.where(r > 0, g / (2.0 * torch.where(r > 0, r, torch.ones_like(r))), torch.zeros_like(g))


def _move(env: dict, S: _Structure, A, i, chi, chi_I, prec, P_in=None, svd_in=None, rec=None, probe=None,
          polar_min=POLAR_MIN):
    mv = _MOVES[i]
    D = A.shape[0]
    (c1n, e1n, s1, ax1), (c2n, e2n, s2, ax2) = mv["c1"], mv["c2"]
    inv1, inv2 = S.moves[i]
    g1 = _fuse_rows(contract(s1, env[c1n], env[e1n]), ax1, inv1)
    g2 = _fuse_rows(contract(s2, env[c2n], env[e2n]), ax2, inv2)
    P1 = P_in[0] if P_in is not None else _projector(g1.detach(), g2.detach(), chi)
    mid1 = contract("nA,nc->Ac", P1, g1)
    mid2 = contract("nA,nc->Ac", P1, g2)
    h1 = contract(mv["m1"][1], mid1, env[mv["m1"][0]]).reshape(-1, chi)
    h2 = contract(mv["m2"][1], mid2, env[mv["m2"][0]]).reshape(-1, chi)
    P2 = P_in[1] if P_in is not None else _projector(h1.detach(), h2.detach(), chi)
    if rec is not None:
        rec.extend([P1, P2])
    if probe is not None:
        probe(i, (g1, g2, P1), (h1, h2, P2))
    new = dict(env)
    for cn, h in zip(mv["new"], (h1, h2)):
        new[cn] = contract("nA,nc->Ac", P2, h) * S.mask[cn]
    # combined projector P[x, rowK, rowB, A] (rows of the grown edge)
    P1_3 = P1.reshape(chi, D, -1)
    Pf = einsum(mv["pf"], P1_3, P2.reshape(P1_3.shape[2], D, -1))
    e, leg = mv["edge"], mv["leg"]
    r, R = mv["rows"]
    m, M = mv["mid"]
    c, Cc = mv["cols"]
    free = "".join(x for x in _SITE if x != leg)
    ket = contract(f"x{leg}I,{_SITE}s->xI{free}s", env[e + "_ket"], A)
    FREE = free.upper()
    bra = contract(f"I{leg.upper()}y,{_SITE.upper()}s->Iy{FREE}s", env[e + "_bra"], A)
    Prow = f"x{r}{R}A"
    Pcol = f"y{c}{Cc}B"
    rest = "".join(x for x in free if x != r)
    z = contract(f"{Prow},xI{free}s->A{R}I{rest}s", Pf, ket, prec)
    w = contract(f"A{R}I{rest}s,Iy{FREE}s->A{rest}y{''.join(x for x in FREE if x != R)}", z, bra, prec)
    wsub = f"A{rest}y{''.join(x for x in FREE if x != R)}"
    Tn = contract(f"{wsub},{Pcol}->A{m}{M}B", w, Pf, prec)
    k = Tn.shape[0]
    Tmat = Tn.reshape(k * D, D * Tn.shape[3])
    if svd_in is not None:
        U, s, Vh = svd_in
    else:
        U, s, Vh = _SVD.apply(Tmat, polar_min)
    kk = min(chi_I, s.shape[0])
    rs = _SqrtSV.apply(s[:kk])
    tk = (U[:, :kk] * rs[None, :]).reshape(k, D, kk)
    tb = (rs[:, None] * Vh[:kk, :]).reshape(kk, D, Tn.shape[3])
    new[e + "_ket"] = tk * S.mask[e + "_ket"]
    new[e + "_bra"] = tb * S.mask[e + "_bra"]
    return new


def _renormalize(env: dict) -> dict:
    """Corners by max-abs (+LOG_EPS), ket/bra pairs by the geometric mean of
    their max-abs (+EPS) (_split_ctm_tensor.py:1209-1240)."""
    out = dict(env)
    for n in ("C1", "C2", "C3", "C4"):
        out[n] = env[n] * (1.0 / (env[n].abs().max() + LOG_EPS))
    for n in ("T1", "T2", "T3", "T4"):
        k, b = env[n + "_ket"], env[n + "_bra"]
        shared = torch.sqrt(k.abs().max() * b.abs().max()) + EPS
        out[n + "_ket"] = k * (1.0 / shared)
        out[n + "_bra"] = b * (1.0 / shared)
    return out


def _sweeps(env: dict, S, A, chi, chi_I, renormalize, prec, n, Ps, svds, rec, p0, probe=None, polar_min=POLAR_MIN):
    for it in range(n):
        for i in range(4):
            j = 4 * (p0 + it) + i
            pin = None if Ps is None else (Ps[2 * j], Ps[2 * j + 1])
            sin = None if svds is None else svds[j]
            env = _move(env, S, A, i, chi, chi_I, prec, pin, sin, rec, probe, polar_min)
        if renormalize:
            env = _renormalize(env)
    return env


def ctm_split_tensor(A, chi: int, max_iter: int = 100, conv_tol: float = 1e-8, chi_I: int | None = None,
                     renormalize: bool = True, precision: str = "fp64", projectors=None, svds=None, record=None,
                     checkpoint_every: int = 0, A_dense: torch.Tensor | None = None,
                     probe=None, svd_driver: str = "polar") -> SplitCTMTensorEnv:
    """Split CTM to convergence (_split_ctm_tensor.py:1243-1289).

    Stops when the normalised singular values of C1 change by less than
    ``conv_tol`` between sweeps (not evaluated when ``conv_tol <= 0``).
    ``precision`` selects the arithmetic of the grown-edge projection
    ("fp64", "bf16x3", "tf32"); projectors and the edge SVD are FP64.
    ``projectors`` (two per move) / ``svds`` ((U, s, Vh) per move) replay a
    run; ``record`` receives the projectors used.  ``checkpoint_every`` > 0
    recomputes groups of that many sweeps in the backward pass (then
    ``conv_tol`` must be <= 0).  ``A_dense`` overrides A's dense data (the
    differentiable input) while A supplies the leg charges.  ``probe``, if
    given, is called at every move (not under checkpointing) as
    probe(move, (g1, g2, P1), (h1, h2, P2)) with the two pairs of grown
    corners and the projectors made from them -- a diagnostic hook.
    ``svd_driver`` picks the edge split's SVD: "polar" (the library's
    polar-decomposition driver for edges of 128 and more, Jacobi below) or
    "jacobi" (Jacobi for every edge).  Both agree to rounding, but inside
    degenerate singular-value clusters they pick different bases, which the
    later projectors depend on: runs that replay projectors recorded by
    another run should use the recording run's driver."""
    if svd_driver not in ("polar", "jacobi"):
        raise ValueError(f"Unknown svd_driver {svd_driver!r}: expected 'polar' or 'jacobi'")
    polar_min = POLAR_MIN if svd_driver == "polar" else 1 << 62
    chi_I = chi if chi_I is None else chi_I
    a, q, f, mod = _site(A)
    if A_dense is not None:
        a = A_dense
    S = _Structure(q, f, mod, chi, chi_I, a.device)
    env = _init(S, a.shape[0], chi, chi_I, a.device)._asdict()
    if checkpoint_every > 0:
        if conv_tol > 0:
            raise ValueError("checkpointed split CTM runs a fixed number of sweeps: pass conv_tol <= 0")
        Ps = projectors
        if Ps is None:
            Ps = []
            with torch.no_grad():
                _sweeps(dict(env), S, a.detach(), chi, chi_I, renormalize, precision, max_iter, None, svds, Ps, 0,
                        polar_min=polar_min)
        if record is not None:
            record.extend(Ps)
        done = 0
        while done < max_iter:
            n = min(checkpoint_every, max_iter - done)

            def seg(*xs, _n=n, _p0=done):
                e = dict(zip(_FIELDS, xs[:12]))
                e = _sweeps(e, S, xs[12], chi, chi_I, renormalize, precision, _n, Ps, svds, None, _p0,
                            polar_min=polar_min)
                return tuple(e[k] for k in _FIELDS)

            out = torch.utils.checkpoint.checkpoint(seg, *[env[k] for k in _FIELDS], a, use_reentrant=False)
            env = dict(zip(_FIELDS, out))
            done += n
        return SplitCTMTensorEnv(**env)
    prev = None
    for it in range(max_iter):
        env = _sweeps(env, S, a, chi, chi_I, renormalize, precision, 1, projectors, svds, record, it, probe,
                      polar_min)
        if conv_tol > 0:
            with torch.no_grad():
                sv = torch.linalg.svdvals(env["C1"])
            if prev is not None:
                s1, s2 = sv / (sv.sum() + 1e-15), prev / (prev.sum() + 1e-15)
                n = min(len(s1), len(s2))
                if float((s1[:n] - s2[:n]).abs().max()) < conv_tol:
                    break
            prev = sv
    return SplitCTMTensorEnv(**env)


def split_env_to_standard(env: SplitCTMTensorEnv) -> CTMEnvironment:
    """Ket and bra edges merged over the interlayer bond (:1292-1313)."""
    chi = env.C1.shape[0]

    def merge(k, b):
        D = k.shape[1]
        return contract("auc,cUb->auUb", k.contiguous(), b.contiguous()).reshape(chi, D * D, chi)

    return CTMEnvironment(env.C1, env.C2, env.C3, env.C4, merge(env.T1_ket, env.T1_bra), merge(env.T2_ket, env.T2_bra),
                          merge(env.T3_ket, env.T3_bra), merge(env.T4_ket, env.T4_bra))


def compute_energy_split_ctm_tensor(A, env: SplitCTMTensorEnv, hamiltonian_gate, d: int | None = None,
                                    A_dense: torch.Tensor | None = None) -> torch.Tensor:
    """Energy per site from the split environment (:1316-1351), through the
    dense two-site RDMs of ``compute_energy_ctm``."""
    a = A_dense if A_dense is not None else _site(A)[0]
    if d is None:
        d = a.shape[-1]
    H = torch.as_tensor(hamiltonian_gate, dtype=torch.float64, device=a.device).reshape(d, d, d, d)
    return compute_energy_ctm(a, split_env_to_standard(env), H, d)
