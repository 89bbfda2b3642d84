"""Dense 1-site CTMRG on the GPU with a hand-written adjoint.

Same surface as tenax ``algorithms/ipeps.py``: ``CTMConfig`` (:38-57),
``CTMEnvironment`` (:91-121), ``ctm`` (:779-851) and ``compute_energy_ctm``
(:1519-1549), on float64 CUDA tensors.  Every contraction runs on the
library's engine (``tenax_b200.dense``: permute-pack, FP64 tensor-core
grouped GEMM, scatter); QR and the small symmetric eigenproblem of the
projector are cuSOLVER calls through torch.linalg.

Absorb + truncate (one move) is a ``torch.autograd.Function`` whose backward
is written out by hand.  With the projector P fixed -- the reference passes
it through ``jax.lax.stop_gradient`` (ipeps.py:958, :996) -- a move is

    Cg1 = X . E_x,  Cg2 = Y . E_y                (corner growth)
    C1' = P^T Cg1,  C2' = P^T Cg2
    T'[A,t,B] = sum P[p,s,A] E[p,x,q] a[s,w,x,t] P[q,w,B]

and the edge is evaluated as three pairwise contractions
U = E.P, V = U.a, T' = P^T.V (4x fewer FLOPs than growing the
(chi D^2, D^2, chi D^2) edge and projecting it, and no such buffer).
The backward runs the transposed chain: dV = P.dT', dU = dV.a,
da = U.dV, dE = dU.P (U recomputed), plus two contractions per grown corner.

The renormalisation x / (max|x| + EPS) (ipeps.py:1133-1149) is a second
Function over the library's batched max-abs kernels and their adjoint.

Projectors: every move takes an optional fixed projector and can record the
one it used, so a run can be replayed exactly (``projectors=`` /
``record=``); with them fixed the energy is a smooth function of A, and its
gradient is what the adjoint computes.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import NamedTuple

import numpy as np
import torch

from tenax_b200 import _capi
from tenax_b200.dense import contract, einsum

EPS = 1e-15  # tenax core/__init__.py:15


@dataclass
class CTMConfig:
    """CTM parameters (ipeps.py:38-57)."""

    chi: int = 20
    max_iter: int = 100
    conv_tol: float = 1e-8
    renormalize: bool = True
    projector_method: str = "eigh"
    qr_warmup_steps: int = 3
    chi_I: int | None = None


class CTMEnvironment(NamedTuple):
    """Corners C1..C4 (chi, chi) and edges T1..T4 (chi, D^2, chi)
    (ipeps.py:91-121)."""

    C1: torch.Tensor
    C2: torch.Tensor
    C3: torch.Tensor
    C4: torch.Tensor
    T1: torch.Tensor
    T2: torch.Tensor
    T3: torch.Tensor
    T4: torch.Tensor


# Per move: corner-1 growth, corner-2 growth, the double layer's subscripts in
# the edge growth (edge E[p,x,q], rows (p,s), middle t, columns (q,w)), the
# environment slots (C1..C4 = 0..3, T1..T4 = 4..7) of (X, E_x, Y, E_y, E)
# and the slots of the outputs (C1', C2', T').
_MOVE_SPECS = (
    ("ab,buc->auc", "gh,hdi->gdi", "swxt", (0, 4, 3, 6, 7), (0, 3, 7)),  # left   ipeps.py:1016-1045
    ("ce,buc->eub", "im,hdi->mdh", "swtx", (1, 4, 2, 6, 5), (1, 2, 5)),  # right  ipeps.py:1048-1071
    ("ab,alg->blg", "ce,erm->crm", "xtsw", (0, 7, 1, 5, 4), (0, 1, 4)),  # top    ipeps.py:1074-1097
    ("gh,alg->hla", "im,erm->ire", "txsw", (3, 7, 2, 5, 6), (3, 2, 6)),  # bottom ipeps.py:1100-1125
)


def _projector(Cg1: torch.Tensor, Cg2: torch.Tensor, chi: int, method: str) -> torch.Tensor:
    """Projector of one move, (n, k) with n = rows of the grown corners.

    "qr": QR of [Cg1, Cg2], eigh of R R^H, P = Q V (ipeps.py:965-1000);
    "eigh": leading eigenvectors of Cg1 Cg1^H + Cg2 Cg2^H (ipeps.py:921-962)."""
    n = Cg1.shape[0] * Cg1.shape[1]
    m1 = Cg1.reshape(n, -1)
    m2 = Cg2.reshape(n, -1)
    if method == "qr":
        Q, R = torch.linalg.qr(torch.cat([m1, m2], dim=1))
        Q = Q.contiguous()
        rho = einsum("ij,kj->ik", R.contiguous(), R.contiguous())
    elif method == "eigh":
        rho = einsum("ij,kj->ik", m1, m1) + einsum("ij,kj->ik", m2, m2)
    else:
        raise ValueError(f"unknown projector method {method!r}")
    rho = 0.5 * (rho + rho.T)
    _, vecs = torch.linalg.eigh(rho)
    k = min(chi, vecs.shape[0])
    V = vecs[:, -k:].flip(1).contiguous()
    return einsum("ij,jk->ik", Q, V) if method == "qr" else V


def _corner_adjoint(subs, x, e, g, need_x, need_e):
    lhs, so = subs.split("->")
    sx, se = lhs.split(",")
    gx = einsum(f"{so},{se}->{sx}", g, e) if need_x else None
    ge = einsum(f"{sx},{so}->{se}", x, g) if need_e else None
    return gx, ge


class _Move(torch.autograd.Function):
    """One absorb + truncate move with a fixed (or freshly computed,
    gradient-free) projector; returns (C1', C2', T', P)."""

    @staticmethod
    def forward(ctx, spec_idx, chi, method, P, X, Ex, Y, Ey, E, a):
        c1, c2, asub, _, _ = _MOVE_SPECS[spec_idx]
        Cg1 = einsum(c1, X, Ex)
        Cg2 = einsum(c2, Y, Ey)
        if P is None:
            P = _projector(Cg1, Cg2, chi, method)
        P = P.contiguous()
        P3 = P.view(Cg1.shape[0], Cg1.shape[1], P.shape[1])
        C1n = einsum("psA,psq->Aq", P3, Cg1)
        C2n = einsum("psA,psq->Aq", P3, Cg2)
        U = einsum("pxq,qwB->pxwB", E, P3)
        V = einsum(f"pxwB,{asub}->pBst", U, a)
        Tn = einsum("psA,pBst->AtB", P3, V)
        ctx.spec_idx = spec_idx
        ctx.save_for_backward(X, Ex, Y, Ey, E, a, P3)
        ctx.mark_non_differentiable(P)
        return C1n, C2n, Tn, P

    @staticmethod
    def backward(ctx, gC1, gC2, gT, _gP):
        X, Ex, Y, Ey, E, a, P3 = ctx.saved_tensors
        c1, c2, asub, _, _ = _MOVE_SPECS[ctx.spec_idx]
        need = ctx.needs_input_grad
        gX = gEx = gY = gEy = gE = ga = None
        if gC1 is not None and (need[4] or need[5]):
            g = einsum("psA,Aq->psq", P3, gC1.contiguous())
            gX, gEx = _corner_adjoint(c1, X, Ex, g, need[4], need[5])
        if gC2 is not None and (need[6] or need[7]):
            g = einsum("psA,Aq->psq", P3, gC2.contiguous())
            gY, gEy = _corner_adjoint(c2, Y, Ey, g, need[6], need[7])
        if gT is not None and (need[8] or need[9]):
            gV = einsum("psA,AtB->pBst", P3, gT.contiguous())
            if need[8]:
                gU = einsum(f"pBst,{asub}->pxwB", gV, a)
                gE = einsum("pxwB,qwB->pxq", gU, P3)
            if need[9]:
                U = einsum("pxq,qwB->pxwB", E, P3)
                ga = einsum(f"pxwB,pBst->{asub}", U, gV)
        return None, None, None, None, gX, gEx, gY, gEy, gE, ga


_SCRATCH: dict = {}


def _renorm_scratch(device) -> torch.Tensor:
    key = torch.device(device).index
    s = _SCRATCH.get(key)
    if s is None:
        s = torch.empty(int(_capi.LIB.tnx_renorm_scratch_len()), dtype=torch.float64, device=device)
        _SCRATCH[key] = s
    return s


def _ptrs(ts):
    return (C.c_void_p * len(ts))(*[t.data_ptr() for t in ts])


class _Renormalize(torch.autograd.Function):
    """x_t / (max|x_t| + EPS) for up to 8 tensors, forward and adjoint on
    the library's kernels (ipeps.py:1133-1149)."""

    @staticmethod
    def forward(ctx, *xs):
        xs = tuple(x.contiguous() for x in xs)
        dev = xs[0].device
        ys = tuple(torch.empty_like(x) for x in xs)
        stat = torch.empty(len(xs), dtype=torch.float64, device=dev)
        ns = (C.c_int64 * len(xs))(*[x.numel() for x in xs])
        st = torch.cuda.current_stream(dev).cuda_stream
        _capi.check(_capi.LIB.tnx_renorm_maxabs(len(xs), _ptrs(xs), _ptrs(ys), ns, EPS, stat.data_ptr(),
                                                _renorm_scratch(dev).data_ptr(), st))
        ctx.save_for_backward(*xs, stat)
        return ys

    @staticmethod
    def backward(ctx, *gys):
        *xs, stat = ctx.saved_tensors
        gs = tuple(torch.zeros_like(x) if g is None else g.contiguous() for x, g in zip(xs, gys))
        dev = xs[0].device
        gxs = tuple(torch.empty_like(x) for x in xs)
        ns = (C.c_int64 * len(xs))(*[x.numel() for x in xs])
        st = torch.cuda.current_stream(dev).cuda_stream
        _capi.check(_capi.LIB.tnx_renorm_maxabs_adjoint(len(xs), _ptrs(xs), _ptrs(gs), _ptrs(gxs), ns, EPS,
                                                        stat.data_ptr(), _renorm_scratch(dev).data_ptr(), st))
        return gxs


def renormalize_env(env: CTMEnvironment) -> CTMEnvironment:
    """Max-abs normalisation of all eight tensors (ipeps.py:1133-1149)."""
    return CTMEnvironment(*_Renormalize.apply(*env))


def _as_site_tensor(A) -> torch.Tensor:
    if not isinstance(A, torch.Tensor):
        A = torch.as_tensor(np.asarray(A, dtype=np.float64))
    if not A.is_cuda:
        A = A.to("cuda")
    if A.dtype != torch.float64:
        raise TypeError("CTM site tensors are float64")
    if A.ndim != 5:
        raise ValueError("the GPU CTM takes 5-leg site tensors A[u, d, l, r, s]")
    return A


def build_double_layer(A: torch.Tensor) -> torch.Tensor:
    """a[uU, dD, lL, rR] = sum_s A[u,d,l,r,s] A[U,D,L,R,s] (ipeps.py:854-876,
    reshaped as at :803-806); real site tensors."""
    D = A.shape[0]
    a = contract("udlrs,UDLRs->uUdDlLrR", A, A)
    return a.reshape(D * D, D * D, D * D, D * D)


def build_double_layer_open(A: torch.Tensor) -> torch.Tensor:
    """Double layer with the physical legs open (ipeps.py:1368-1381)."""
    D, d = A.shape[0], A.shape[4]
    ao = contract("udlrs,UDLRt->uUdDlLrRst", A, A)
    return ao.reshape(D * D, D * D, D * D, D * D, d, d)


def initialize_env(a: torch.Tensor, chi: int) -> CTMEnvironment:
    """Identity corners and identity-like edges (ipeps.py:879-918)."""
    D2 = a.shape[0]
    m = min(chi, D2)
    C = torch.zeros(chi, chi, dtype=torch.float64, device=a.device)
    C[:m, :m] = torch.eye(m, dtype=torch.float64, device=a.device)
    T = torch.zeros(chi, D2, chi, dtype=torch.float64, device=a.device)
    idx = torch.arange(m, device=a.device)
    T[idx, :, idx] = 1.0
    return CTMEnvironment(C, C, C, C, T, T, T, T)


def ctm_move(env: CTMEnvironment, a: torch.Tensor, direction: int, chi: int, method: str,
             P: torch.Tensor | None = None):
    """One move (0 left, 1 right, 2 top, 3 bottom).  Returns (env', P)."""
    _, _, _, slots, outs = _MOVE_SPECS[direction]
    ins = [env[s] for s in slots]
    C1n, C2n, Tn, P = _Move.apply(direction, chi, method, P, *ins, a)
    new = list(env)
    for s, x in zip(outs, (C1n, C2n, Tn)):
        new[s] = x
    return CTMEnvironment(*new), P


def ctm_sweep(env, a, chi, renormalize, method, projectors=None, record=None) -> CTMEnvironment:
    """Left, right, top, bottom moves, then renormalise (ipeps.py:755-769)."""
    for i in range(4):
        env, P = ctm_move(env, a, i, chi, method, None if projectors is None else projectors[i])
        if record is not None:
            record.append(P)
    if renormalize:
        env = renormalize_env(env)
    return env


def _sv_diff(sv_new, sv_old):
    """ipeps.py:772-776"""
    s1 = sv_new / (sv_new.sum() + 1e-15)
    s2 = sv_old / (sv_old.sum() + 1e-15)
    return float((s1 - s2).abs().max())


def ctm(A, config: CTMConfig, initial_env: CTMEnvironment | None = None, projectors=None, record=None,
        a: torch.Tensor | None = None) -> CTMEnvironment:
    """CTM environment of a 1x1-cell PEPS (ipeps.py:779-851).

    Eigh warm-up sweeps when ``projector_method == "qr"``, then sweeps until
    the normalised corner spectrum of C1 changes by less than ``conv_tol``
    or ``max_iter`` sweeps ran.  With ``conv_tol <= 0`` the spectrum is not
    computed (it can never fall below it).  ``projectors``: flat list, four
    per sweep, used instead of computing them; ``record``: list the used
    projectors are appended to.  Differentiable in A (projectors fixed)."""
    A = _as_site_tensor(A)
    chi = config.chi
    if a is None:
        a = build_double_layer(A)
    env = initial_env if initial_env is not None else initialize_env(a.detach(), chi)
    max_iter = config.max_iter
    method = config.projector_method
    it_total = 0

    def sweep(env, m):
        nonlocal it_total
        ps = None if projectors is None else projectors[4 * it_total: 4 * it_total + 4]
        it_total += 1
        return ctm_sweep(env, a, chi, config.renormalize, m, ps, record)

    if method == "qr" and config.qr_warmup_steps > 0:
        warm = min(config.qr_warmup_steps, max_iter)
        for _ in range(warm):
            env = sweep(env, "eigh")
        max_iter -= warm
    prev = torch.zeros(min(chi, env.C1.shape[0]), dtype=torch.float64, device=A.device)
    for _ in range(max_iter):
        env = sweep(env, method)
        if config.conv_tol > 0:
            with torch.no_grad():
                sv = torch.linalg.svdvals(env.C1)
            if _sv_diff(sv, prev) < config.conv_tol:
                break
            prev = sv
    return env


def _finish_rdm(rdm, d):
    """(s1,s1',s2,s2') -> (s1,s2,s1',s2'), symmetrise, trace-normalise
    (ipeps.py:1440-1448)."""
    m = rdm.permute(0, 2, 1, 3).reshape(d * d, d * d)
    m = 0.5 * (m + m.T)
    m = m / (torch.trace(m) + 1e-15)
    return m.reshape(d, d, d, d)


def rdm2x1(A, env: CTMEnvironment, d: int, ao=None):
    """Horizontal two-site RDM (ipeps.py:1384-1448): left and right halves
    each contracted with the open double layer, then joined."""
    C1, C2, C3, C4, T1, T2, T3, T4 = env
    if ao is None:
        ao = build_double_layer_open(A)
    UL = contract("ab,buc->auc", C1, T1)
    UR = contract("cuf,fg->cug", T1, C2)
    LL = contract("gi,idj->gdj", C4, T3)
    LR = contract("jdk,mk->jdm", T3, C3)
    X = contract("auc,axg->ucxg", UL, T4)
    X = contract("ucxg,udxrst->cgdrst", X, ao)
    L1 = contract("cgdrst,gdj->crjst", X, LL)
    Y = contract("cuf,frm->curm", UR, T2)
    Y = contract("curm,udlrtv->cmdltv", Y, ao)
    R2 = contract("cmdltv,jdm->cjltv", Y, LR)
    return _finish_rdm(contract("crjst,cjruv->stuv", L1, R2), d)


def rdm1x2(A, env: CTMEnvironment, d: int, ao=None):
    """Vertical two-site RDM (ipeps.py:1451-1516): upper and lower halves
    each contracted with the open double layer, then joined."""
    C1, C2, C3, C4, T1, T2, T3, T4 = env
    if ao is None:
        ao = build_double_layer_open(A)
    top = contract("auc,ce->aue", contract("ab,buc->auc", C1, T1), C2)
    Z = contract("aue,alf->uelf", top, T4)
    Z = contract("uelf,udlrst->efdrst", Z, ao)
    site1 = contract("efdrst,erg->dfgst", Z, T2)
    bot = contract("hqk,ik->hqi", contract("hj,jqk->hqk", C4, T3), C3)
    W = contract("fmh,hqi->fmqi", T4, bot)
    W = contract("fmqi,pqmnwx->fipnwx", W, ao)
    site2 = contract("fipnwx,gni->fgpwx", W, T2)
    return _finish_rdm(contract("dfgst,fgdwx->stwx", site1, site2), d)


def compute_energy_ctm(A, env: CTMEnvironment, hamiltonian_gate, d: int) -> torch.Tensor:
    """Energy per site E_h + E_v from the two-site RDMs (ipeps.py:1519-1549).
    Returns a 0-dim CUDA tensor (differentiable in A and env)."""
    A = _as_site_tensor(A)
    H = torch.as_tensor(hamiltonian_gate, dtype=torch.float64, device=A.device).reshape(d, d, d, d)
    ao = build_double_layer_open(A)
    eh = (rdm2x1(A, env, d, ao) * H).sum()
    ev = (rdm1x2(A, env, d, ao) * H).sum()
    return eh + ev


def rdm2x1_2site(A, B, env_A: CTMEnvironment, env_B: CTMEnvironment, d: int, ao_A=None, ao_B=None):
    """Horizontal RDM of a checkerboard cell, A left and B right
    (ipeps.py:1552-1594): the left half from A's corners and edges with A's
    open double layer, the right half from B's with B's."""
    C1, _, _, C4, T1, _, T3, T4 = env_A
    _, C2, C3, _, T1b, T2, T3b, _ = env_B
    ao_A = build_double_layer_open(A) if ao_A is None else ao_A
    ao_B = build_double_layer_open(B) if ao_B is None else ao_B
    UL = contract("ab,buc->auc", C1, T1)
    LL = contract("gi,idj->gdj", C4, T3)
    X = contract("auc,axg->ucxg", UL, T4)
    X = contract("ucxg,udxrst->cgdrst", X, ao_A)
    L1 = contract("cgdrst,gdj->crjst", X, LL)
    UR = contract("cuf,fg->cug", T1b, C2)
    LR = contract("jdk,mk->jdm", T3b, C3)
    Y = contract("cuf,frm->curm", UR, T2)
    Y = contract("curm,udlrtv->cmdltv", Y, ao_B)
    R2 = contract("cmdltv,jdm->cjltv", Y, LR)
    return _finish_rdm(contract("crjst,cjruv->stuv", L1, R2), d)


def rdm1x2_2site(A, B, env_A: CTMEnvironment, env_B: CTMEnvironment, d: int, ao_A=None, ao_B=None):
    """Vertical RDM of a checkerboard cell, A top and B bottom
    (ipeps.py:1597-1642)."""
    C1, C2, _, _, T1, T2, _, T4 = env_A
    _, _, C3b, C4b, _, T2b, T3b, T4b = env_B
    ao_A = build_double_layer_open(A) if ao_A is None else ao_A
    ao_B = build_double_layer_open(B) if ao_B is None else ao_B
    top = contract("auc,ce->aue", contract("ab,buc->auc", C1, T1), C2)
    Z = contract("aue,alf->uelf", top, T4)
    Z = contract("uelf,udlrst->efdrst", Z, ao_A)
    site1 = contract("efdrst,erg->dfgst", Z, T2)
    bot = contract("hqk,ik->hqi", contract("hj,jqk->hqk", C4b, T3b), C3b)
    W = contract("fmh,hqi->fmqi", T4b, bot)
    W = contract("fmqi,pqmnwx->fipnwx", W, ao_B)
    site2 = contract("fipnwx,gni->fgpwx", W, T2b)
    return _finish_rdm(contract("dfgst,fgdwx->stwx", site1, site2), d)


def compute_energy_ctm_2site(A, B, env_A: CTMEnvironment, env_B: CTMEnvironment, hamiltonian_gate,
                             d: int) -> torch.Tensor:
    """Energy per site of a checkerboard cell, one horizontal and one
    vertical bond (ipeps.py:1645-1662)."""
    A, B = _as_site_tensor(A), _as_site_tensor(B)
    H = torch.as_tensor(hamiltonian_gate, dtype=torch.float64, device=A.device).reshape(d, d, d, d)
    ao_A, ao_B = build_double_layer_open(A), build_double_layer_open(B)
    eh = (rdm2x1_2site(A, B, env_A, env_B, d, ao_A, ao_B) * H).sum()
    ev = (rdm1x2_2site(A, B, env_A, env_B, d, ao_A, ao_B) * H).sum()
    return eh + ev


def energy_and_grad(A, hamiltonian_gate, config: CTMConfig, projectors=None):
    """Energy after ``config`` CTM sweeps and its gradient in A through the
    hand-written adjoint, projectors held fixed (stop-gradient semantics).

    Returns ``(E, dE/dA, projectors)`` with E a float and dE/dA a CUDA tensor
    shaped like A; ``projectors`` are those used (pass them back to replay)."""
    A = _as_site_tensor(A).detach().clone().requires_grad_(True)
    rec: list = []
    env = ctm(A, config, projectors=projectors, record=rec)
    E = compute_energy_ctm(A, env, hamiltonian_gate, A.shape[4])
    (g,) = torch.autograd.grad(E, A)
    return float(E.detach()), g, rec


def heisenberg_gate(device="cuda") -> torch.Tensor:
    """S=1/2 Heisenberg bond operator S.S as (2, 2, 2, 2)."""
    sz = torch.tensor([[0.5, 0.0], [0.0, -0.5]], dtype=torch.float64)
    sp = torch.tensor([[0.0, 1.0], [0.0, 0.0]], dtype=torch.float64)
    sm = sp.T.contiguous()
    h = torch.kron(sz, sz) + 0.5 * torch.kron(sp, sm) + 0.5 * torch.kron(sm, sp)
    return h.reshape(2, 2, 2, 2).to(device)
