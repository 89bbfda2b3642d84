"""Float64 restatement of tenax's dense 1-site CTMRG and its NN energy.

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).

Written with torch CPU float64 operations so that the same code gives the
forward values and, through torch autograd, the reverse-mode gradient the
reference obtains from JAX AD.  Every einsum follows the reference's own
subscripts and order (tenax ``algorithms/ipeps.py``); the projectors are
detached exactly where the reference calls ``jax.lax.stop_gradient``
(``ipeps.py:958``, ``:996``).  ``jnp.max`` splits its cotangent evenly among
ties, and so does ``torch.Tensor.max``.

Environment tuples are ordered ``(C1, C2, C3, C4, T1, T2, T3, T4)`` like the
reference's ``CTMEnvironment`` (``ipeps.py:91-121``).

Every move accepts an optional projector ``P``; when given it is used in
place of the one computed from the grown corners.  Passing the projectors
recorded by another implementation makes two runs gauge-identical, which
lets gradients be compared element for element.
"""

from __future__ import annotations

import torch
import torch.utils.checkpoint

EPS = 1e-15  # tenax core/__init__.py:15


def heisenberg_gate(dtype=torch.float64):
    """S=1/2 Heisenberg bond operator S.S as a (d, d, d, d) tensor, the gate
    of the reference's CTM tests (tests/test_ctm_tensor.py:95-103)."""
    sz = torch.tensor([[0.5, 0.0], [0.0, -0.5]], dtype=dtype)
    sp = torch.tensor([[0.0, 1.0], [0.0, 0.0]], dtype=dtype)
    sm = sp.T.contiguous()
    h = torch.kron(sz, sz) + 0.5 * torch.kron(sp, sm) + 0.5 * torch.kron(sm, sp)
    return h.reshape(2, 2, 2, 2)


def build_double_layer(A):
    """a[uU,dD,lL,rR] = sum_s A[u,d,l,r,s] conj(A)[U,D,L,R,s]
    (ipeps.py:854-876, 5-leg branch; reshape at :803-806)."""
    D = A.shape[0]
    a = torch.einsum("udlrs,UDLRs->uUdDlLrR", A, A.conj())
    return a.reshape(D * D, D * D, D * D, D * D)


def build_double_layer_open(A):
    """Double layer with the physical legs left open (ipeps.py:1368-1381)."""
    D, d = A.shape[0], A.shape[4]
    ao = torch.einsum("udlrs,UDLRt->uUdDlLrRst", A, A.conj())
    return ao.reshape(D * D, D * D, D * D, D * D, d, d)


def initialize_env(a, chi):
    """Identity corners and identity-like edges (ipeps.py:879-918)."""
    D2 = a.shape[0]
    m = min(chi, D2)
    C = torch.zeros(chi, chi, dtype=a.dtype)
    C[:m, :m] = torch.eye(m, dtype=a.dtype)
    T = torch.zeros(chi, D2, chi, dtype=a.dtype)
    for i in range(m):
        T[i, :, i] += 1.0
    return (C, C, C, C, T, T, T, T)


def projector_qr(C1g, C2g, chi):
    """QR of [C1g, C2g] then eigh of R R^H (ipeps.py:965-993)."""
    M = torch.cat([C1g, C2g], dim=1)
    Q, R = torch.linalg.qr(M)
    rho = R @ R.conj().T
    rho = 0.5 * (rho + rho.conj().T)
    _, vecs = torch.linalg.eigh(rho)
    k = min(chi, vecs.shape[0])
    V = vecs[:, -k:].flip(1)
    return Q @ V


def projector_eigh(C1g, C2g, chi):
    """Leading eigenvectors of C1g C1g^H + C2g C2g^H (ipeps.py:921-950)."""
    rho = C1g @ C1g.conj().T + C2g @ C2g.conj().T
    rho = 0.5 * (rho + rho.conj().T)
    _, vecs = torch.linalg.eigh(rho)
    k = min(chi, vecs.shape[0])
    return vecs[:, -k:].flip(1)


def truncation_gap(C1g, C2g, chi, method):
    """Relative eigenvalue gap at the cut, (lam_k - lam_{k+1}) / lam_1, of the
    matrix whose leading eigenvectors the projector keeps (1.0 when nothing
    is cut).  Where it is small the kept subspace is ill-determined and two
    correct implementations may keep different ones."""
    with torch.no_grad():
        if method == "qr":
            _, R = torch.linalg.qr(torch.cat([C1g, C2g], dim=1))
            rho = R @ R.conj().T
        else:
            rho = C1g @ C1g.conj().T + C2g @ C2g.conj().T
        lam = torch.linalg.eigvalsh(0.5 * (rho + rho.conj().T)).flip(0)
        k = min(chi, lam.shape[0])
        if k >= lam.shape[0] or float(lam[0]) <= 0.0:
            return 1.0
        return float((lam[k - 1] - lam[k]) / lam[0])


def ctm_move(C1g, C2g, Tg, chi, method, P=None):
    """Truncate both grown corners and the grown edge with one projector
    (ipeps.py:921-1013).  Returns ``(C1', C2', T', P)``."""
    if P is None:
        with torch.no_grad():
            f = projector_qr if method == "qr" else projector_eigh
            P = f(C1g.detach(), C2g.detach(), chi)
    P = P.detach()
    C1n = P.conj().T @ C1g
    C2n = P.conj().T @ C2g
    Tn = torch.einsum("ia,idj,jb->adb", P, Tg, P)
    return C1n, C2n, Tn, P


def grow_left(env, a):
    """Grown C1, C4 and T4 of the left move (ipeps.py:1027-1033)."""
    C1, C2, C3, C4, T1, T2, T3, T4 = env
    D2 = a.shape[0]
    C1g = torch.einsum("ab,buc->auc", C1, T1).reshape(-1, T1.shape[2])
    C4g = torch.einsum("gh,hdi->gdi", C4, T3).reshape(-1, T3.shape[2])
    T4g = torch.einsum("alg,udlr->augdr", T4, a)
    T4g = T4g.permute(0, 1, 4, 2, 3).reshape(C1g.shape[0], D2, C4g.shape[0])
    return C1g, C4g, T4g


def grow_right(env, a):
    """Grown C2, C3 and T2 of the right move (ipeps.py:1056-1062)."""
    C1, C2, C3, C4, T1, T2, T3, T4 = env
    D2 = a.shape[0]
    C2g = torch.einsum("ce,buc->eub", C2, T1).reshape(-1, T1.shape[0])
    C3g = torch.einsum("im,hdi->mdh", C3, T3).reshape(-1, T3.shape[0])
    T2g = torch.einsum("erm,udlr->eumdl", T2, a)
    T2g = T2g.permute(0, 1, 4, 2, 3).reshape(C2g.shape[0], D2, C3g.shape[0])
    return C2g, C3g, T2g


def grow_top(env, a):
    """Grown C1, C2 and T1 of the top move (ipeps.py:1082-1088)."""
    C1, C2, C3, C4, T1, T2, T3, T4 = env
    D2 = a.shape[0]
    C1g = torch.einsum("ab,alg->blg", C1, T4).reshape(-1, T4.shape[2])
    C2g = torch.einsum("ce,erm->crm", C2, T2).reshape(-1, T2.shape[2])
    T1g = torch.einsum("buc,udlr->bcdlr", T1, a)
    T1g = T1g.permute(0, 3, 2, 1, 4).reshape(C1g.shape[0], D2, C2g.shape[0])
    return C1g, C2g, T1g


def grow_bottom(env, a):
    """Grown C4, C3 and T3 of the bottom move (ipeps.py:1108-1115)."""
    C1, C2, C3, C4, T1, T2, T3, T4 = env
    D2 = a.shape[0]
    C4g = torch.einsum("gh,alg->hal", C4, T4)
    C4g = C4g.permute(0, 2, 1).reshape(-1, T4.shape[0])
    C3g = torch.einsum("im,erm->ire", C3, T2).reshape(-1, T2.shape[0])
    T3g = torch.einsum("hdi,udlr->hiulr", T3, a)
    T3g = T3g.permute(0, 3, 2, 1, 4).reshape(C4g.shape[0], D2, C3g.shape[0])
    return C4g, C3g, T3g


GROW = (grow_left, grow_right, grow_top, grow_bottom)
# environment slots (C1..C4 = 0..3, T1..T4 = 4..7) each move's outputs replace
PLACE = ((0, 3, 7), (1, 2, 5), (0, 1, 4), (3, 2, 6))


def _make_move(i):
    def move(env, a, chi, method, P=None):
        Cg1, Cg2, Tg = GROW[i](env, a)
        C1n, C2n, Tn, P = ctm_move(Cg1, Cg2, Tg, chi, method, P)
        out = list(env)
        for slot, x in zip(PLACE[i], (C1n, C2n, Tn)):
            out[slot] = x
        return tuple(out), P

    return move


left_move, right_move, top_move, bottom_move = (_make_move(i) for i in range(4))
left_move.__doc__ = "ipeps.py:1016-1045 -> updates C1, C4, T4."
right_move.__doc__ = "ipeps.py:1048-1071 -> updates C2, C3, T2."
top_move.__doc__ = "ipeps.py:1074-1097 -> updates C1, C2, T1."
bottom_move.__doc__ = "ipeps.py:1100-1125 -> updates C4, C3, T3."


MOVES = (left_move, right_move, top_move, bottom_move)  # ipeps.py:763-766


def renormalize_env(env):
    """x / (max|x| + EPS) for all eight tensors (ipeps.py:1133-1149)."""
    return tuple(x / (x.abs().max() + EPS) for x in env)


def ctm_sweep(env, a, chi, renormalize, method, projectors=None, record=None):
    """One sweep: left, right, top, bottom, then renormalise (ipeps.py:755-769).

    ``projectors``: optional list of 4 projectors to use instead of computing
    them; ``record``: optional list the 4 projectors used are appended to.
    """
    for i, mv in enumerate(MOVES):
        env, P = mv(env, a, chi, method, None if projectors is None else projectors[i])
        if record is not None:
            record.append(P)
    if renormalize:
        env = renormalize_env(env)
    return env


def ctm(A, chi, iters, method="qr", warmup=0, renormalize=True, projectors=None, record=None,
        checkpoint=False):
    """Fixed-count CTM: ``warmup`` eigh sweeps then ``iters - warmup`` sweeps
    of ``method`` (ipeps.py:779-851 with ``conv_tol=0``, so the while-loop
    runs to ``max_iter``).  ``projectors`` / ``record``: flat lists, 4 per
    sweep.  ``checkpoint`` recomputes each sweep in the backward pass to keep
    host memory bounded at large chi."""
    a = build_double_layer(A)
    env = initialize_env(a, chi)
    warm = min(warmup, iters) if method == "qr" else 0
    for it in range(iters):
        m = "eigh" if it < warm else method
        Ps = None if projectors is None else projectors[4 * it: 4 * it + 4]
        if checkpoint and torch.is_grad_enabled():
            if Ps is None:
                rec: list = []
                with torch.no_grad():
                    ctm_sweep(tuple(x.detach() for x in env), a.detach(), chi, renormalize, m, None, rec)
                Ps = rec
            if record is not None:
                record.extend(Ps)

            def body(*xs, _Ps=Ps, _m=m):
                return ctm_sweep(tuple(xs[:8]), xs[8], chi, renormalize, _m, _Ps)

            env = torch.utils.checkpoint.checkpoint(body, *env, a, use_reentrant=False)
        else:
            env = ctm_sweep(env, a, chi, renormalize, m, Ps, record)
    return env


def rdm2x1(A, env, d):
    """Horizontal two-site RDM, the reference's contraction sequence
    (ipeps.py:1384-1448)."""
    C1, C2, C3, C4, T1, T2, T3, T4 = env
    ao = build_double_layer_open(A)
    UL = torch.einsum("ab,buc->auc", C1, T1)
    UR = torch.einsum("cuf,fg->cug", T1, C2)
    LL = torch.einsum("gi,idj->gdj", C4, T3)
    LR = torch.einsum("jdk,mk->jdm", T3, C3)
    Lenv = torch.einsum("auc,axg,gdj->ucxdj", UL, T4, LL)
    Renv = torch.einsum("cuf,frm,jdm->curjd", UR, T2, LR)
    L1 = torch.einsum("ucxdj,udxrst->crjst", Lenv, ao)
    R2 = torch.einsum("curjd,udlrtv->cjltv", Renv, ao)
    rdm = torch.einsum("crjst,cjruv->stuv", L1, R2).permute(0, 2, 1, 3)
    return _finish_rdm(rdm, d)


def rdm1x2(A, env, d):
    """Vertical two-site RDM, the reference's contraction sequence
    (ipeps.py:1451-1516)."""
    C1, C2, C3, C4, T1, T2, T3, T4 = env
    ao = build_double_layer_open(A)
    top = torch.einsum("ab,buc,ce->aue", C1, T1, C2)
    row1 = torch.einsum("aue,alf,erg->ulfrg", top, T4, T2)
    site1 = torch.einsum("ulfrg,udlrst->dfgst", row1, ao)
    T4ao = torch.einsum("fmh,pqmnwx->fhpqnwx", T4, ao)
    s12 = torch.einsum("abcst,bhaqnwx->chqnstwx", site1, T4ao)
    s12r = torch.einsum("chqnstwx,cni->hqistwx", s12, T2)
    bot = torch.einsum("hj,jqk,ik->hqi", C4, T3, C3)
    rdm = torch.einsum("hqistwx,hqi->stwx", s12r, bot).permute(0, 2, 1, 3)
    return _finish_rdm(rdm, d)


def _finish_rdm(rdm, d):
    """Symmetrise and trace-normalise (ipeps.py:1444-1448, :1512-1516)."""
    m = rdm.reshape(d * d, d * d)
    m = 0.5 * (m + m.conj().T)
    m = m / (torch.trace(m) + 1e-15)
    return m.reshape(d, d, d, d)


def energy(A, env, H, d):
    """E_h + E_v (ipeps.py:1519-1549)."""
    Hr = H.reshape(d, d, d, d)
    eh = torch.einsum("ijkl,ijkl->", rdm2x1(A, env, d), Hr)
    ev = torch.einsum("ijkl,ijkl->", rdm1x2(A, env, d), Hr)
    return eh + ev


def rdm2x1_2site(A, B, env_A, env_B, d):
    """Horizontal RDM of a checkerboard cell, A left and B right, left half
    from A's environment and right half from B's (ipeps.py:1552-1594)."""
    C1, _, _, C4, T1, _, T3, T4 = env_A
    _, C2, C3, _, T1b, T2, T3b, _ = env_B
    ao_A, ao_B = build_double_layer_open(A), build_double_layer_open(B)
    UL = torch.einsum("ab,buc->auc", C1, T1)
    LL = torch.einsum("gi,idj->gdj", C4, T3)
    Lenv = torch.einsum("auc,axg,gdj->ucxdj", UL, T4, LL)
    UR = torch.einsum("cuf,fg->cug", T1b, C2)
    LR = torch.einsum("jdk,mk->jdm", T3b, C3)
    Renv = torch.einsum("cuf,frm,jdm->curjd", UR, T2, LR)
    L1 = torch.einsum("ucxdj,udxrst->crjst", Lenv, ao_A)
    R2 = torch.einsum("curjd,udlrtv->cjltv", Renv, ao_B)
    rdm = torch.einsum("crjst,cjruv->stuv", L1, R2).permute(0, 2, 1, 3)
    return _finish_rdm(rdm, d)


def rdm1x2_2site(A, B, env_A, env_B, d):
    """Vertical RDM of a checkerboard cell, A top and B bottom
    (ipeps.py:1597-1642)."""
    C1, C2, _, _, T1, T2, _, T4 = env_A
    _, _, C3b, C4b, _, T2b, T3b, T4b = env_B
    ao_A, ao_B = build_double_layer_open(A), build_double_layer_open(B)
    top = torch.einsum("ab,buc,ce->aue", C1, T1, C2)
    row1 = torch.einsum("aue,alf,erg->ulfrg", top, T4, T2)
    site1 = torch.einsum("ulfrg,udlrst->dfgst", row1, ao_A)
    T4ao = torch.einsum("fmh,pqmnwx->fhpqnwx", T4b, ao_B)
    s12 = torch.einsum("abcst,bhaqnwx->chqnstwx", site1, T4ao)
    s12r = torch.einsum("chqnstwx,cni->hqistwx", s12, T2b)
    bot = torch.einsum("hj,jqk,ik->hqi", C4b, T3b, C3b)
    rdm = torch.einsum("hqistwx,hqi->stwx", s12r, bot).permute(0, 2, 1, 3)
    return _finish_rdm(rdm, d)


def energy_2site(A, B, env_A, env_B, H, d):
    """E_h + E_v of a checkerboard cell (ipeps.py:1645-1662)."""
    Hr = H.reshape(d, d, d, d)
    eh = torch.einsum("ijkl,ijkl->", rdm2x1_2site(A, B, env_A, env_B, d), Hr)
    ev = torch.einsum("ijkl,ijkl->", rdm1x2_2site(A, B, env_A, env_B, d), Hr)
    return eh + ev


def energy_and_grad(A, H, chi, iters, method="qr", warmup=0, projectors=None, checkpoint=False):
    """Energy after ``iters`` CTM sweeps and its gradient in A with the
    projectors held fixed (the stop-gradient semantics of the reference).
    Returns ``(E, dE/dA, projectors used)``."""
    A = A.detach().clone().requires_grad_(True)
    rec: list = []
    env = ctm(A, chi, iters, method, warmup, True, projectors, rec, checkpoint)
    E = energy(A, env, H, A.shape[4])
    (g,) = torch.autograd.grad(E, A)
    return float(E.detach()), g, rec


def energy_fixed(A, H, chi, iters, projectors, method="qr", warmup=0):
    """Energy with every projector given (no decomposition): the function
    whose derivative the stop-gradient adjoint computes."""
    with torch.no_grad():
        env = ctm(A, chi, iters, method, warmup, True, projectors)
        return float(energy(A, env, H, A.shape[4]))


def site_tensor(D, d, seed):
    """Site tensor A ~ N(0,1)/sqrt(2 D^4), float64, from numpy's seeded
    generator (shape (D, D, D, D, d))."""
    import numpy as np

    rng = np.random.default_rng(seed)
    return torch.from_numpy(rng.standard_normal((D, D, D, D, d)) / np.sqrt(2.0 * D ** 4))
