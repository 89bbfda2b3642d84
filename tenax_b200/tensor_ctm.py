"""Block-sparse standard CTMRG on the GPU (tenax ``algorithms/_ctm_tensor.py``).

The environment is eight block-sparse tensors (``CTMTensorEnv``: corners
``(chi, chi)``, edges ``(chi, D^2, chi)``) and the double layer is built and
absorbed block by block, never densified:

  * every absorb step is a label contraction on the library's planner and
    grouped-GEMM engine with the reference's filtered semantics (output
    blocks, key order and charge bookkeeping identical);
  * the grown corners and edges are re-indexed by ``fuse_indices`` (the
    planner's fuse tables and the strided-copy kernel);
  * the projector is the reference's per-sector one: for every charge q of
    the fused leg, rho_q = sum M M^T over the grown corners' blocks carrying
    q (one engine GEMM per sector over the blocks side by side), symmetrised
    and diagonalised (cuSOLVER through ``torch.linalg.eigh``); eigenpairs are
    ranked over all sectors by (-lambda, -index) and the first chi kept;
  * the max-abs renormalisation of all eight tensors is one launch pair of
    the library's batched reduction kernels; each tensor is then laid out
    over every valid block, as the reference's dense round trip does.

The new bond gets trivial charges (``_ctm_tensor.py:173-191``), so a
projector keeps only the fused rows of charge 0; with non-trivial charges
the reference's environment becomes exactly zero within the first sweep, and
so does this one, block for block.

Projectors can be supplied and recorded, as the dense P the reference
passes to ``jax.lax.stop_gradient`` (:185, :247, :282), so a run replays the
reference's choices inside degenerate eigenvalue clusters exactly.

A dense 5-leg site tensor (torch or numpy) stands for the reference's
``DenseTensor`` input: trivial charges, zero-padded identity corners and
the dense projector branch.
"""

from __future__ import annotations

from typing import NamedTuple

import ctypes as C
import numpy as np
import torch

from tenax_b200 import _capi
from tenax_b200.contraction import contract
from tenax_b200.core import FlowDirection, TensorIndex, U1Symmetry
from tenax_b200.dense import einsum
from tenax_b200.ipeps import CTMEnvironment, compute_energy_ctm, compute_energy_ctm_2site
from tenax_b200.tensor import SymmetricTensor, block_shape, compute_valid_blocks, embed_in_keys
from tenax_b200.tensor_utils import fuse_indices

IN, OUT = FlowDirection.IN, FlowDirection.OUT
EPS = 1e-15  # tenax core/__init__.py:15


class CTMTensorEnv(NamedTuple):
    """Standard CTM environment of block-sparse tensors (_ctm_tensor.py:38-58).

    Corners (C1: c1_d, c1_r), (C2: c2_l, c2_d), (C3: c3_u, c3_l),
    (C4: c4_r, c4_u); edges (T1: t1_l, u2, t1_r), (T2: t2_u, r2, t2_d),
    (T3: t3_r, d2, t3_l), (T4: t4_d, l2, t4_u)."""

    C1: SymmetricTensor
    C2: SymmetricTensor
    C3: SymmetricTensor
    C4: SymmetricTensor
    T1: SymmetricTensor
    T2: SymmetricTensor
    T3: SymmetricTensor
    T4: SymmetricTensor


# corner: labels, flows and the site-tensor axis its charges derive from
# (_split_ctm_tensor.py:262-267)
_CORNERS = {
    "C1": ("c1_d", "c1_r", IN, OUT, 1),
    "C2": ("c2_l", "c2_d", IN, OUT, 0),
    "C3": ("c3_u", "c3_l", OUT, IN, 1),
    "C4": ("c4_r", "c4_u", OUT, IN, 0),
}
# edge: labels, flows, the axis of the chi charges and the axis fused into D^2
# (_ctm_tensor.py:395-405)
_EDGES = {
    "T1": ("t1_l", "u2", "t1_r", IN, IN, OUT, 3, 0),
    "T2": ("t2_u", "r2", "t2_d", OUT, OUT, IN, 0, 3),
    "T3": ("t3_r", "d2", "t3_l", OUT, OUT, IN, 3, 1),
    "T4": ("t4_d", "l2", "t4_u", IN, IN, OUT, 1, 2),
}
# per direction (_ctm_tensor.py:586-759): two grown corners (corner, its leg
# renamed to the perpendicular edge's, that edge, the pair fused into
# "fused"), the parallel edge with its two fused pairs, and the renames that
# turn the projected tensors back into environment tensors
_MOVES = {
    "left": (("C1", "c1_r", "t1_l", "T1", "c1_d", "u2"), ("C4", "c4_u", "t3_r", "T3", "c4_r", "d2"),
             ("T4", "t4_d", "u2", "t4_u", "d2"),
             (("C1", {"chi_new": "c1_d", "t1_r": "c1_r"}), ("C4", {"chi_new": "c4_r", "t3_l": "c4_u"}),
              ("T4", {"chi_new": "t4_d", "chi_new_r": "t4_u", "r2": "l2"}))),
    "right": (("C2", "c2_l", "t1_r", "T1", "c2_d", "u2"), ("C3", "c3_u", "t3_l", "T3", "c3_l", "d2"),
              ("T2", "t2_u", "u2", "t2_d", "d2"),
              (("C2", {"chi_new": "c2_l", "t1_l": "c2_d"}), ("C3", {"chi_new": "c3_u", "t3_r": "c3_l"}),
               ("T2", {"chi_new": "t2_u", "chi_new_r": "t2_d", "l2": "r2"}))),
    "top": (("C1", "c1_d", "t4_d", "T4", "c1_r", "l2"), ("C2", "c2_d", "t2_u", "T2", "c2_l", "r2"),
            ("T1", "t1_l", "l2", "t1_r", "r2"),
            (("C1", {"chi_new": "c1_d", "t4_u": "c1_r"}), ("C2", {"chi_new": "c2_l", "t2_d": "c2_d"}),
             ("T1", {"chi_new": "t1_l", "chi_new_r": "t1_r", "d2": "u2"}))),
    "bottom": (("C4", "c4_r", "t4_u", "T4", "c4_u", "l2"), ("C3", "c3_l", "t2_d", "T2", "c3_u", "r2"),
               ("T3", "t3_r", "l2", "t3_l", "r2"),
               (("C4", {"chi_new": "c4_r", "t4_d": "c4_u"}), ("C3", {"chi_new": "c3_u", "t2_u": "c3_l"}),
                ("T3", {"chi_new": "t3_r", "chi_new_r": "t3_l", "u2": "d2"}))),
}
_DIRECTIONS = ("left", "right", "top", "bottom")

SINGLE_SITE_NEIGHBORS = {(0, 0): {d: (0, 0) for d in _DIRECTIONS}}
CHECKERBOARD_NEIGHBORS = {(0, 0): {d: (1, 0) for d in _DIRECTIONS}, (1, 0): {d: (0, 0) for d in _DIRECTIONS}}


# ---------------------------------------------------------------------------
# site tensor, double layer, initial environment
# ---------------------------------------------------------------------------

class _Site(NamedTuple):
    A: SymmetricTensor
    dense: bool  # the reference's DenseTensor branch


def _site(A) -> _Site:
    if isinstance(A, SymmetricTensor):
        if A.ndim != 5:
            raise ValueError("ctm_tensor takes 5-leg site tensors (u, d, l, r, phys)")
        return _Site(A, False)
    x = A if isinstance(A, torch.Tensor) else torch.as_tensor(np.asarray(A, dtype=np.float64))
    x = x.to(device="cuda", dtype=torch.float64)
    if x.ndim != 5:
        raise ValueError("ctm_tensor takes 5-leg site tensors (u, d, l, r, phys)")
    sym = U1Symmetry()
    idx = tuple(TensorIndex(sym, np.zeros(n, np.int32), f, label=l)
                for n, f, l in zip(x.shape, (OUT, IN, OUT, IN, IN), ("u", "d", "l", "r", "phys")))
    return _Site(SymmetricTensor.from_flat(idx, [(0, 0, 0, 0, 0)], x.reshape(-1).contiguous()), True)


def _fuse_pair(t: SymmetricTensor, la, lb, fused, flow) -> SymmetricTensor:
    """(_ctm_tensor.py:65-76)"""
    lab = t.labels()
    return fuse_indices(t, lab.index(la), lab.index(lb), fused, flow)


def build_double_layer_tensor(A, open_phys: bool = False, precision=None) -> SymmetricTensor:
    """a = sum_phys A bar(A) with the ket/bra pairs fused: (u,U)->u2 IN,
    (d,D)->d2 OUT, (l,L)->l2 IN, (r,R)->r2 OUT (_ctm_tensor.py:346-392);
    ``open_phys`` keeps (phys, phys_bra) as legs."""
    A = _site(A).A
    ren = {"u": "U", "d": "D", "l": "L", "r": "R"}
    if open_phys:
        ren["phys"] = "phys_bra"
    a = contract(A, A.bar().relabels(ren), precision=precision)
    a = _fuse_pair(a, "u", "U", "u2", IN)
    a = _fuse_pair(a, "d", "D", "d2", OUT)
    a = _fuse_pair(a, "l", "L", "l2", IN)
    return _fuse_pair(a, "r", "R", "r2", OUT)


def _pair_charges(idx: TensorIndex, fused_flow) -> np.ndarray:
    """Charges of idx fused with its flow-flipped copy, position i*d + j
    (_tensor_utils.py:169-203)."""
    q = idx.charges.astype(np.int64)
    raw = (int(idx.flow) * q[:, None] - int(idx.flow) * q[None, :]) * int(fused_flow)
    n = idx.symmetry.n_values()
    return (np.mod(raw, n) if n is not None else raw).reshape(-1).astype(np.int32)


def _derive(base, n: int) -> np.ndarray:
    """(_split_ctm_tensor.py:251-257)"""
    base = np.asarray(base, dtype=np.int32)
    return base[:n].copy() if n <= len(base) else np.tile(base, n // len(base) + 1)[:n].astype(np.int32)


def initialize_ctm_tensor_env(A, chi: int) -> CTMTensorEnv:
    """Identity corners and identity-like edges (_ctm_tensor.py:408-583)."""
    return _init(_site(A), chi)


def _init(site: _Site, chi: int) -> CTMTensorEnv:
    A = site.A
    D = A.indices[0].dim
    D2 = D * D
    sym = A.indices[0].symmetry
    dev = A.data.device
    out = {}
    for name, (la, lb, fa, fb, ref) in _CORNERS.items():
        if site.dense:
            q = np.zeros(chi, np.int32)
            m = min(chi, D2)
            Cm = torch.zeros(chi, chi, dtype=torch.float64, device=dev)
            Cm[:m, :m] = torch.eye(m, dtype=torch.float64, device=dev)
        else:
            q = _derive(_pair_charges(A.indices[ref], fa), chi)
            Cm = torch.eye(chi, dtype=torch.float64, device=dev)
        out[name] = SymmetricTensor.from_dense(Cm, (TensorIndex(sym, q, fa, label=la),
                                                    TensorIndex(sym, q.copy(), fb, label=lb)))
    m = min(chi, D2)
    T = torch.zeros(chi, D2, chi, dtype=torch.float64, device=dev)
    ar = torch.arange(m, device=dev)
    T[ar, :, ar] = 1.0
    for name, (l1, l2, l3, f1, f2, f3, rc, rd) in _EDGES.items():
        if site.dense:
            qc, qd = np.zeros(chi, np.int32), np.zeros(D2, np.int32)
        else:
            qc, qd = _derive(A.indices[rc].charges, chi), _pair_charges(A.indices[rd], f2)
        idx = (TensorIndex(sym, qc, f1, label=l1), TensorIndex(sym, qd, f2, label=l2),
               TensorIndex(sym, qc.copy(), f3, label=l3))
        out[name] = SymmetricTensor.from_dense(T, idx, tol=float("inf"))
    return CTMTensorEnv(**out)


# ---------------------------------------------------------------------------
# projector
# ---------------------------------------------------------------------------

def _top_k(rho: torch.Tensor, chi: int):
    w, v = torch.linalg.eigh(0.5 * (rho + rho.T))
    k = min(chi, w.shape[0])
    return v[:, w.shape[0] - k:].flip(1)


def _eigh_projector_symmetric(C1g: SymmetricTensor, C4g: SymmetricTensor, chi: int) -> torch.Tensor:
    """Dense projector from per-sector density matrices (_ctm_tensor.py:79-192).

    For each fused charge q (sorted) the blocks of C1g and then C4g carrying
    q are reshaped to (d_q, -1), d_q counted on C1g's fused leg (a C4g block
    whose size is not a multiple of d_q raises ValueError, as the
    reference's reshape does), and rho_q accumulates M M^T block by block
    (one FP64 engine GEMM each, in the reference's order).  With a single
    sector this is the dense branch's arithmetic exactly, so trivial-charge
    symmetric and dense inputs give identical runs, as in the reference."""
    fpos = C1g.labels().index("fused")
    fidx = C1g.indices[fpos]
    by_q: dict = {}
    for t in (C1g, C4g):
        for k, blk in t.blocks.items():
            by_q.setdefault(int(k[fpos]), []).append(blk)
    rows = {q: np.flatnonzero(fidx.charges == q) for q in sorted(by_q)}
    sectors = []
    for q in sorted(by_q):
        dq = len(rows[q])
        if dq == 0:
            continue
        rho = None
        for blk in by_q[q]:
            n = blk.numel()
            if n % dq:
                shape = f"({dq},newaxis)" if fpos == 0 else f"(newaxis,{dq})"
                raise ValueError(f"cannot reshape array of size {n} into shape {shape}")
            M = (blk.reshape(dq, -1) if fpos == 0 else blk.reshape(-1, dq).T).contiguous()
            r = einsum("ik,jk->ij", M, M)
            rho = r if rho is None else rho + r
        w, v = torch.linalg.eigh(0.5 * (rho + rho.T))
        sectors.append((q, w, v))
    dev = C1g.data.device
    if sectors:
        ws = torch.cat([w for _, w, _ in sectors]).cpu().numpy()
    else:
        ws = np.zeros(0)
    ranked, off = [], 0
    for q, w, _ in sectors:
        ranked.extend((float(ws[off + i]), q, i) for i in range(w.shape[0]))
        off += w.shape[0]
    ranked.sort(key=lambda e: (-e[0], -e[2]))
    n_keep = min(chi, len(ranked))
    keep: dict = {}
    for _, q, i in ranked[:n_keep]:
        keep.setdefault(q, []).append(i)
    vecs = {q: v for q, _, v in sectors}
    P = torch.zeros(fidx.dim, n_keep, dtype=torch.float64, device=dev)
    col = 0
    for q in sorted(keep):
        sel = sorted(keep[q], reverse=True)
        r = torch.as_tensor(rows[q], device=dev)
        P[r[:, None], torch.arange(col, col + len(sel), device=dev)[None, :]] = \
            vecs[q][:, torch.as_tensor(sel, device=dev)]
        col += len(sel)
    return P


def _dense_projector(C1g: SymmetricTensor, C4g: SymmetricTensor, chi: int, method: str) -> torch.Tensor:
    """Projector of the densified grown corners (_ctm_tensor.py:231-289)."""
    a, b = C1g.todense(), C4g.todense()
    if method == "qr":
        Q, R = torch.linalg.qr(torch.cat([a, b], dim=1))
        V = _top_k(einsum("ik,jk->ij", R, R), chi)
        return einsum("ij,jk->ik", Q, V.contiguous())
    return _top_k(einsum("ik,jk->ij", a, a) + einsum("ik,jk->ij", b, b), chi)


def _projector(C1g, C4g, chi: int, method: str, dense: bool) -> torch.Tensor:
    """(_ctm_tensor.py:195-296)"""
    if method not in ("eigh", "qr"):
        raise ValueError(f"Unknown projector_method={method!r}; expected 'eigh' or 'qr'.")
    if method == "eigh" and not dense and C1g.n_blocks and C4g.n_blocks:
        return _eigh_projector_symmetric(C1g, C4g, chi)
    return _dense_projector(C1g, C4g, chi, method)


def _wrap_projector(P: torch.Tensor, fidx: TensorIndex) -> SymmetricTensor:
    """P (fused, chi_new), trivial chi_new charges flowing OUT, kept on its
    valid blocks only (_ctm_tensor.py:187-191, :253-264, :284-296)."""
    chi_new = TensorIndex(fidx.symmetry, np.zeros(P.shape[1], np.int32), OUT, label="chi_new")
    return SymmetricTensor.from_dense(P, (fidx, chi_new), tol=float("inf"))


# ---------------------------------------------------------------------------
# moves and renormalisation
# ---------------------------------------------------------------------------

def _move(env: dict, env_nb: dict, a: SymmetricTensor, chi: int, method: str, direction: str, dense: bool,
          precision=None, P_in=None, record=None) -> dict:
    """One directional move (_ctm_tensor.py:586-759 with :299-338)."""
    g1, g2, (ename, la, lb, ra, rb), outs = _MOVES[direction]
    grown = []
    for cname, old, new, pname, fa, fb in (g1, g2):
        g = contract(env[cname].relabel(old, new), env_nb[pname], precision=precision)
        grown.append(_fuse_pair(g, fa, fb, "fused", IN))
    Tg = _fuse_pair(contract(env[ename], a, precision=precision), la, lb, "fl", IN)
    Tg = _fuse_pair(Tg, ra, rb, "fr", OUT)
    Pd = P_in if P_in is not None else _projector(grown[0], grown[1], chi, method, dense)
    if not isinstance(Pd, torch.Tensor) or not Pd.is_cuda:
        Pd = torch.as_tensor(np.asarray(Pd, dtype=np.float64)).to(a.data.device)
    if record is not None:
        record.append(Pd.detach().clone())
    P = _wrap_projector(Pd, grown[0].indices[grown[0].labels().index("fused")])
    Pb = P.bar()
    new = (contract(Pb, grown[0], precision=precision), contract(Pb, grown[1], precision=precision),
           contract(contract(Pb.relabel("fused", "fl"), Tg, precision=precision),
                    P.relabels({"fused": "fr", "chi_new": "chi_new_r"}), precision=precision))
    out = dict(env)
    for (name, ren), t in zip(outs, new):
        out[name] = t.relabels(ren)
    return out


_KEYS: dict = {}


def _all_keys(indices) -> list:
    """Every valid key whose legs all have basis states, sorted (the block
    set of from_dense)."""
    sig = tuple((i.charges.tobytes(), int(i.flow), i.symmetry.n_values()) for i in indices)
    keys = _KEYS.get(sig)
    if keys is None:
        keys = sorted(tuple(int(q) for q in k) for k in compute_valid_blocks(tuple(indices))
                      if all(s > 0 for s in block_shape(indices, k)))
        _KEYS[sig] = keys
    return keys


_SCRATCH: dict = {}


def _renormalize(env: dict) -> dict:
    """x / (max|x| + EPS) for all eight tensors in one launch pair, each then
    laid out over all its valid blocks (_ctm_tensor.py:767-793)."""
    names = list(env)
    xs = [env[n].data.contiguous() for n in names]
    dev = xs[0].device
    ys = [torch.empty_like(x) for x in xs]
    stat = torch.empty(len(xs), dtype=torch.float64, device=dev)
    s = _SCRATCH.get(dev.index)
    if s is None:
        s = torch.empty(int(_capi.LIB.tnx_renorm_scratch_len()), dtype=torch.float64, device=dev)
        _SCRATCH[dev.index] = s
    ptr = lambda ts: (C.c_void_p * len(ts))(*[t.data_ptr() for t in ts])  # noqa: E731
    ns = (C.c_int64 * len(xs))(*[x.numel() for x in xs])
    _capi.check(_capi.LIB.tnx_renorm_maxabs(len(xs), ptr(xs), ptr(ys), ns, EPS, stat.data_ptr(), s.data_ptr(),
                                            torch.cuda.current_stream(dev).cuda_stream))
    out = {}
    for n, y in zip(names, ys):
        t = SymmetricTensor.from_flat(env[n].indices, env[n].keys, y)
        out[n] = embed_in_keys(t, _all_keys(t.indices))
    return out


def _sweep(env: dict, a, chi, renormalize, method, dense, precision, Ps, record) -> dict:
    """Left, right, top, bottom, then renormalise (_ctm_tensor.py:796-808)."""
    for dr in _DIRECTIONS:
        env = _move(env, env, a, chi, method, dr, dense, precision, None if Ps is None else next(Ps), record)
    return _renormalize(env) if renormalize else env


def _sv_diff(s_new: torch.Tensor, s_old: torch.Tensor) -> float:
    """(_ctm_tensor.py:861-865)"""
    s1 = s_new / (s_new.sum() + 1e-15)
    s2 = s_old / (s_old.sum() + 1e-15)
    return float((s1 - s2).abs().max())


def ctm_tensor(A, chi: int, max_iter: int = 100, conv_tol: float = 1e-8, renormalize: bool = True,
               projector_method: str = "eigh", qr_warmup_steps: int = 3, *, projectors=None, record=None,
               precision=None) -> CTMTensorEnv:
    """Standard CTM to convergence of the corner spectrum (_ctm_tensor.py:868-917).

    ``projectors``: the dense projectors to use, in call order (four per
    sweep), instead of computing them; ``record``: a list the used ones are
    appended to.  ``precision``: the absorb contractions' arithmetic (FP64
    by default; the projector GEMMs and eigh are always FP64).  With
    ``conv_tol <= 0`` the corner spectrum is not computed (it can never fall
    below it)."""
    site = _site(A)
    a = build_double_layer_tensor(site.A, precision=precision)
    env = _init(site, chi)._asdict()
    Ps = iter(projectors) if projectors is not None else None
    if projector_method == "qr" and qr_warmup_steps > 0:
        warm = min(qr_warmup_steps, max_iter)
        for _ in range(warm):
            env = _sweep(env, a, chi, renormalize, "eigh", site.dense, precision, Ps, record)
        max_iter -= warm
    prev = None
    for _ in range(max_iter):
        env = _sweep(env, a, chi, renormalize, projector_method, site.dense, precision, Ps, record)
        if conv_tol > 0:
            sv = torch.linalg.svdvals(env["C1"].todense())
            if prev is not None and _sv_diff(sv, prev) < conv_tol:
                break
            prev = sv
    return CTMTensorEnv(**env)


def _ctm_tensor_multisite(sites: dict, neighbors: dict, chi: int, max_iter: int = 100, conv_tol: float = 1e-8,
                          renormalize: bool = True, projector_method: str = "eigh", qr_warmup_steps: int = 3,
                          projectors=None, record=None, precision=None) -> dict:
    """Multisite CTM (_ctm_tensor.py:836-858, :920-974): per direction every
    site (sorted coordinates) moves with its neighbour's environment and
    double layer; converged when every site's corner spectrum is."""
    info = {c: _site(A) for c, A in sites.items()}
    dls = {c: build_double_layer_tensor(s.A, precision=precision) for c, s in info.items()}
    envs = {c: _init(s, chi)._asdict() for c, s in info.items()}
    dense = any(s.dense for s in info.values())
    Ps = iter(projectors) if projectors is not None else None

    def run(envs, method):
        for dr in _DIRECTIONS:
            for c in sorted(envs):
                nb = neighbors[c][dr]
                envs[c] = _move(envs[c], envs[nb], dls[nb], chi, method, dr, dense, precision,
                                None if Ps is None else next(Ps), record)
        if renormalize:
            envs = {c: _renormalize(e) for c, e in envs.items()}
        return envs

    if projector_method == "qr" and qr_warmup_steps > 0:
        warm = min(qr_warmup_steps, max_iter)
        for _ in range(warm):
            envs = run(envs, "eigh")
        max_iter -= warm
    prev: dict = {}
    for _ in range(max_iter):
        envs = run(envs, projector_method)
        if conv_tol > 0:
            done = True
            for c in sorted(envs):
                sv = torch.linalg.svdvals(envs[c]["C1"].todense())
                if c not in prev or _sv_diff(sv, prev[c]) >= conv_tol:
                    done = False
                prev[c] = sv
            if done:
                break
    return {c: CTMTensorEnv(**e) for c, e in envs.items()}


def ctm_tensor_2site(A, B, chi: int, max_iter: int = 100, conv_tol: float = 1e-8, renormalize: bool = True,
                     projector_method: str = "eigh", qr_warmup_steps: int = 3, *, projectors=None, record=None,
                     precision=None):
    """Checkerboard CTM of sublattices A (0,0) and B (1,0) (_ctm_tensor.py:977-1018)."""
    envs = _ctm_tensor_multisite({(0, 0): A, (1, 0): B}, CHECKERBOARD_NEIGHBORS, chi, max_iter, conv_tol,
                                 renormalize, projector_method, qr_warmup_steps, projectors, record, precision)
    return envs[(0, 0)], envs[(1, 0)]


# ---------------------------------------------------------------------------
# energy
# ---------------------------------------------------------------------------

def _dense_env(env: CTMTensorEnv) -> CTMEnvironment:
    """(_ctm_tensor.py:1021-1034)"""
    return CTMEnvironment(*[t.todense() for t in env])


def _dense_site(A) -> torch.Tensor:
    if isinstance(A, SymmetricTensor):
        return A.todense()
    return (A if isinstance(A, torch.Tensor) else torch.as_tensor(np.asarray(A, dtype=np.float64))).to(
        device="cuda", dtype=torch.float64)


def _gate(H, d: int) -> torch.Tensor:
    if isinstance(H, SymmetricTensor):
        H = H.todense()
    return torch.as_tensor(np.asarray(H) if not isinstance(H, torch.Tensor) else H,
                           dtype=torch.float64).reshape(d, d, d, d)


def compute_energy_ctm_tensor(A, env: CTMTensorEnv, hamiltonian_gate, d: int | None = None) -> torch.Tensor:
    """Energy per site through the dense RDMs (_ctm_tensor.py:1037-1069)."""
    Ad = _dense_site(A)
    d = Ad.shape[-1] if d is None else d
    return compute_energy_ctm(Ad, _dense_env(env), _gate(hamiltonian_gate, d).to(Ad.device), d)


def compute_energy_ctm_tensor_2site(A, B, env_A: CTMTensorEnv, env_B: CTMTensorEnv, hamiltonian_gate,
                                    d: int | None = None) -> torch.Tensor:
    """Energy per site of a checkerboard cell (_ctm_tensor.py:1072-1109)."""
    Ad, Bd = _dense_site(A), _dense_site(B)
    d = Ad.shape[-1] if d is None else d
    return compute_energy_ctm_2site(Ad, Bd, _dense_env(env_A), _dense_env(env_B),
                                    _gate(hamiltonian_gate, d).to(Ad.device), d)
