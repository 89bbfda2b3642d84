"""Two-site symmetric DMRG on the GPU.

Same driver, configuration and result as tenax's symmetric back-end
(algorithms/dmrg.py:44-305, 890-1365): environment updates via the
unfiltered block contraction, theta via ``contract``, the two-site H_eff
matvec via the fused ``HeffOperator``, a device-side Lanczos (FP64 scalars
and vectors, one host read-back per solve), and the block-diagonal truncated
SVD (linalg.py:75-333) with cuSOLVER per charge sector.
"""

from __future__ import annotations

import time
from dataclasses import dataclass, field
from typing import NamedTuple

import numpy as np
import torch

from tenax_b200 import _capi, vector
from tenax_b200.contraction import blockwise_contract, contract
from tenax_b200.core import FlowDirection, TensorIndex, U1Symmetry
from tenax_b200.heff import HeffBatch, HeffOperator
from tenax_b200.linalg import POLAR_MIN, svd_batch
from tenax_b200.network import TensorNetwork
from tenax_b200.tensor import SymmetricTensor, _device, block_shape, embed_in_keys, restrict_to_keys


@dataclass
class DMRGConfig:
    """(algorithms/dmrg.py:44-77); ``precision`` selects the H_eff sector GEMMs:
    "fp64" (DMMA), "bf16x3" or "tf32" (tcgen05).  With a mixed precision the
    Lanczos recurrence stays FP64 and the reported energy is the FP64 Rayleigh
    quotient of the Ritz vector when ``fp64_energy`` is set."""

    max_bond_dim: int = 100
    num_sweeps: int = 10
    convergence_tol: float = 1e-10
    num_states: int = 1
    two_site: bool = True
    lanczos_max_iter: int = 50
    lanczos_tol: float = 1e-12
    noise: float = 0.0
    svd_trunc_err: float | None = None
    target_charge: int | None = None
    verbose: bool = False
    precision: str = "fp64"
    fp64_energy: bool = True
    # relative Lanczos stop level beta < tol_rel*|alpha|; None = 0 for FP64
    # (the reference's absolute test only) and the matvec noise level otherwise
    lanczos_tol_rel: float | None = None
    check_matvec_residual: bool = False
    # with a mixed precision: FP64 Lanczos steps started from the mixed Ritz
    # vector (0 = report the FP64 Rayleigh quotient only)
    fp64_polish_steps: int = 3
    # cuSOLVER driver of the per-sector SVD and the number of CUDA streams the
    # sectors of one bond are decomposed on concurrently: "native" is the
    # library's batch (tnx_svd_batch: polar decomposition for large sectors,
    # Jacobi for small ones), anything else is torch.linalg.svd's driver.
    # chi=2048 cylinder, 4 sweeps, mixed: SVD phase 9.8 s (gesvd, 1 stream),
    # 4.7 s (gesvd, 8 streams), 2.9 s (Jacobi gesvdj, 8 streams), 2.1 s
    # (polar decomposition for every sector, 8 workers).
    svd_driver: str | None = "native"
    svd_streams: int = 8
    # run each Krylov loop of a fused H_eff as one captured CUDA graph
    cuda_graph: bool = False
    # schedule of the mixed-precision H_eff stages 1-3 (HeffOperator's
    # ``schedule``).  A sweep builds one operator per site and applies it a
    # few dozen times, so the three-kernel schedule, whose tables are the
    # cheapest to build on the host, is the default; None takes the
    # operator's automatic choice (routed from 5e9 stage FLOPs on).
    heff_schedule: dict | None = field(default_factory=lambda: {"fuse_mpo": 0, "c_per_tile": 0})


NOISE_REL = {"fp64": 0.0, "bf16x3": 1e-5, "tf32": 2e-3}


class DMRGResult(NamedTuple):
    energy: float
    energies_per_sweep: list
    mps: TensorNetwork
    truncation_errors: list
    converged: bool


# ---------------------------------------------------------------------------
# padding and environments
# ---------------------------------------------------------------------------

def _pad(t: SymmetricTensor, pad_left: bool) -> SymmetricTensor:
    """Add a trivial charge-0 leg (dmrg.py:924-952); the flat data is unchanged."""
    u1 = U1Symmetry()
    z = np.zeros(1, np.int32)
    if pad_left:
        idx = (TensorIndex(u1, z, FlowDirection.IN, "_pad_l"),) + t.indices
        keys = [(0,) + k for k in t.keys]
    else:
        idx = t.indices + (TensorIndex(u1, z, FlowDirection.OUT, "_pad_r"),)
        keys = [k + (0,) for k in t.keys]
    return SymmetricTensor.from_flat(idx, keys, t.data)


def _unpad(t: SymmetricTensor, pad_left: bool) -> SymmetricTensor:
    """(dmrg.py:955-975)"""
    if pad_left:
        return SymmetricTensor.from_flat(t.indices[1:], [k[1:] for k in t.keys], t.data)
    return SymmetricTensor.from_flat(t.indices[:-1], [k[:-1] for k in t.keys], t.data)


def _trivial_env(left: bool) -> SymmetricTensor:
    """(dmrg.py:890-921)"""
    u1 = U1Symmetry()
    z = np.zeros(1, np.int32)
    if left:
        idx = (TensorIndex(u1, z, FlowDirection.IN, "env_mps_l"), TensorIndex(u1, z, FlowDirection.IN, "env_mpo_l"),
               TensorIndex(u1, z, FlowDirection.OUT, "env_mps_conj_l"))
    else:
        idx = (TensorIndex(u1, z, FlowDirection.OUT, "env_mps_r"), TensorIndex(u1, z, FlowDirection.OUT, "env_mpo_r"),
               TensorIndex(u1, z, FlowDirection.IN, "env_mps_conj_r"))
    return SymmetricTensor.from_flat(idx, [(0, 0, 0)], torch.ones(1, dtype=torch.float64, device=_device()))


def _pad_site(A: SymmetricTensor) -> SymmetricTensor:
    if A.ndim == 2:
        lab0 = A.labels()[0]
        return _pad(A, pad_left=isinstance(lab0, str) and lab0.startswith("p"))
    return A


def update_left_env(env, A, W, precision="fp64"):
    """new_L[d,e,f] = L[a,b,c] A[a,p,d] W[b,p,x,e] A*[c,x,f] (dmrg.py:1165-1198)."""
    A = _pad_site(A)
    out_idx = (A.indices[2], W.indices[3], A.indices[2])
    return blockwise_contract([env, A, W, A], "abc,apd,bpxe,cxf->def", out_idx, precision)


def update_right_env(env, B, W, precision="fp64"):
    """new_R[d,e,f] = R[a,b,c] B[d,p,a] W[e,p,x,b] B*[f,x,c] (dmrg.py:1201-1232)."""
    B = _pad_site(B)
    out_idx = (B.indices[0], W.indices[0], B.indices[0])
    return blockwise_contract([env, B, W, B], "abc,dpa,epxb,fxc->def", out_idx, precision)


# ---------------------------------------------------------------------------
# Lanczos on the device
# ---------------------------------------------------------------------------

class LanczosStats(NamedTuple):
    steps: int
    alphas: np.ndarray
    betas: np.ndarray
    seconds: float


def lanczos(op: HeffOperator, theta: SymmetricTensor, num_steps: int, tol: float, fp64_op: HeffOperator | None = None,
            tol_rel: float = 0.0, polish_steps: int = 0, graph: bool = False):
    """Plain three-term Lanczos without reorthogonalisation (dmrg.py:978-1045).

    Krylov vectors live on the operator's closed key layout; alpha/beta and
    the early-exit flag stay on the device until the single read-back after
    the loop.  ``fp64_op`` may also be a zero-argument callable returning
    the FP64 operator: it is then called after the first loop is queued on
    the device and before its read-back, so that the operator's host-side
    planning overlaps the device work.  ``graph``: each Krylov loop of a
    fused operator runs as one captured CUDA graph (see ``_krylov``).
    Returns (eigenvalue, eigenvector SymmetricTensor with the reference's key
    set, LanczosStats).
    """
    t0 = time.perf_counter()
    x0 = embed_in_keys(theta, op.keys).data
    built = {}

    def build():
        if fp64_op is not None and not isinstance(fp64_op, HeffOperator):
            built["op"] = fp64_op()

    energy, vec, m, a, b = _krylov(op, x0, num_steps, tol, tol_rel, between=build, graph=graph)
    fp64_op = built.get("op", fp64_op)
    key_seq = op.key_seq
    keys = key_seq[0] if m <= 1 else key_seq[min(m - 1, len(key_seq) - 1)]
    if fp64_op is not None and polish_steps > 0:
        # FP64 polish: a short FP64 Lanczos started from the mixed Ritz vector
        energy, vec, m2, _, _ = _krylov(fp64_op, vec, polish_steps, tol, 0.0, graph=graph)
        keys = op.keys
    elif fp64_op is not None:
        # Rayleigh quotient of the Ritz vector with the FP64 operator
        hv = fp64_op.apply(vec)
        energy = float(vector.dot(vec, hv)) / float(vector.dot(vec, vec))
    full = SymmetricTensor.from_flat(theta.indices, op.keys, vec)
    result = restrict_to_keys(full, keys)
    return energy, result, LanczosStats(m, a[:m], b[1:m + 1], time.perf_counter() - t0)


_GENERAL_DONE_POLL = 4  # steps between early-exit checks of a general-path operator
_CAPTURE_STREAMS: dict = {}
_GRAPH_KEEP: list = [None]


def _capture_stream(dev: torch.device) -> torch.cuda.Stream:
    """One side stream per device for graph capture (its reduction scratch is
    created before capture, so nothing is allocated inside a graph)."""
    s = _CAPTURE_STREAMS.get(dev.index)
    if s is None:
        with torch.cuda.device(dev):
            s = torch.cuda.Stream()
        _CAPTURE_STREAMS[dev.index] = s
    return s


def _krylov(op: HeffOperator, x0: torch.Tensor, num_steps: int, tol: float, tol_rel: float, between=None,
            graph: bool = False):
    """Device Lanczos loop from x0 on op's key layout: returns
    (Ritz value, normalised Ritz vector, steps used, alphas, betas).
    ``between`` (if given) runs on the host once the loop is queued, before
    the read-back waits for it.  ``graph`` (fused operators only) captures the
    whole loop -- start vector, every matvec and orthogonalisation step with
    its early-exit flag -- in one CUDA graph and launches that instead of the
    individual kernels."""
    dev = x0.device
    n = op.size
    basis = torch.empty((num_steps + 1, max(n, 1)), dtype=torch.float64, device=dev)
    alpha = torch.zeros(num_steps + 1, dtype=torch.float64, device=dev)
    beta = torch.zeros(num_steps + 2, dtype=torch.float64, device=dev)
    done = torch.zeros(1, dtype=torch.int32, device=dev)
    w = torch.empty(max(n, 1), dtype=torch.float64, device=dev)
    # fused operators skip their kernels once the early-exit flag is set; a
    # general-path operator (planning and allocating per apply) reads the flag
    # back every few steps and stops issuing applies once it is set
    batch = HeffBatch([op], skip_flag=done) if op.fused else None
    graph = graph and batch is not None

    def issue(x_in, scr, nrm):
        st = torch.cuda.current_stream().cuda_stream
        _capi.check(_capi.LIB.tnx_nrm2(x0.data_ptr(), n, nrm.data_ptr(), scr.data_ptr(), st))
        _capi.check(_capi.LIB.tnx_scale(x0.data_ptr(), basis[0].data_ptr(), n, nrm.data_ptr(), 2, st))
        for k in range(num_steps):
            if batch is not None:
                if x_in is not None:
                    # fixed matvec input: the batch's pointer tables never change inside a graph
                    x_in[:n].copy_(basis[k, :n])
                    batch.apply([x_in[:n]], [w[:n]])
                else:
                    batch.apply([basis[k, :n]], [w[:n]])
            else:
                if k > 0 and k % _GENERAL_DONE_POLL == 0 and int(done.item()) != 0:
                    break
                op.apply(basis[k, :n], w[:n])
            _capi.check(_capi.LIB.tnx_lanczos_step(
                w.data_ptr(), basis[k].data_ptr(), basis[k - 1].data_ptr() if k > 0 else 0,
                basis[k + 1].data_ptr(), n, alpha.data_ptr(), beta.data_ptr(), k, float(tol), float(tol_rel),
                done.data_ptr(), scr.data_ptr(), st))

    if graph:
        cap = _capture_stream(dev)
        cap.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(cap):
            scr = vector.scratch(dev)
            nrm = torch.empty((), dtype=torch.float64, device=dev)
            x_in = torch.empty(max(n, 1), dtype=torch.float64, device=dev)
            # bind the batch's pointer tables to (x_in, w) before capture
            batch.apply([x_in[:n]], [w[:n]])
            done.zero_()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=cap):
            issue(x_in, scr, nrm)
        g.replay()
        torch.cuda.current_stream().wait_stream(cap)
        _GRAPH_KEEP[0] = (g, x_in, nrm)  # alive until the read-back below completes
    else:
        issue(None, vector.scratch(dev), torch.empty((), dtype=torch.float64, device=dev))
    st = torch.cuda.current_stream().cuda_stream
    if between is not None:
        between()
    a = alpha.cpu().numpy()
    b = beta.cpu().numpy()
    if batch is not None and batch.device_error():
        raise RuntimeError("tcgen05 GEMM reported a device-side timeout")
    m = num_steps
    for k in range(num_steps):
        if b[k + 1] < tol or b[k + 1] < tol_rel * abs(a[k]):
            m = k + 1
            break
    if m == 1 or num_steps == 0:
        vec = basis[0, :n]
        energy = float(a[0]) if m == 1 else 0.0
    else:
        T = np.diag(a[:m]) + np.diag(b[1:m], 1) + np.diag(b[1:m], -1)
        ev, evecs = np.linalg.eigh(T)
        idx = int(np.argmin(ev))
        energy = float(ev[idx])
        coefs = torch.from_numpy(np.ascontiguousarray(evecs[:, idx])).to(dev)
        table = torch.tensor([basis[k].data_ptr() for k in range(m)], dtype=torch.int64, device=dev)
        out = torch.empty(max(n, 1), dtype=torch.float64, device=dev)
        _capi.check(_capi.LIB.tnx_combine(table.data_ptr(), coefs.data_ptr(), m, n, out.data_ptr(), st))
        nn = vector.nrm2(out[:n])
        vec = vector.scale(out[:n], nn, 2)
    return energy, vec, m, a, b


# ---------------------------------------------------------------------------
# truncated block SVD and bond scaling
# ---------------------------------------------------------------------------

_SVD_WORKERS: dict = {}


def _svd_workers(device: torch.device, n: int):
    """A thread pool with one CUDA stream per worker on ``device``."""
    from concurrent.futures import ThreadPoolExecutor

    key = (device.index, n)
    w = _SVD_WORKERS.get(key)
    if w is None:
        with torch.cuda.device(device):
            streams = [torch.cuda.Stream() for _ in range(n)]
        w = (ThreadPoolExecutor(max_workers=n, thread_name_prefix="tnx-svd"), streams)
        _SVD_WORKERS[key] = w
    return w


def native_sector_svds(mats, n_workers: int = 8, polar_min: int = POLAR_MIN):
    """The library's sector SVD batch (``tenax_b200.linalg.svd_batch``)."""
    return svd_batch(mats, n_workers, polar_min)


def sector_svds(mats, driver: str | None = None, n_streams: int = 1):
    """``torch.linalg.svd(M, full_matrices=False)`` of every sector matrix.

    ``driver="native"`` runs the library's own batch (``native_sector_svds``,
    ``n_streams`` workers).  Otherwise ``driver`` is torch's cuSOLVER driver
    and with ``n_streams > 1`` the sectors are split into ``n_streams`` lists
    (longest-first, greedy by m*n*min(m,n)) and each list is decomposed on its
    own CUDA stream by its own host thread: cuSOLVER's per-call latency and
    its host synchronisation then overlap across sectors.  The results are
    identical to the sequential calls (same routine, same inputs); the
    current stream waits for all of them before this returns."""
    if driver == "native":
        return native_sector_svds(mats, max(1, n_streams))
    if n_streams <= 1 or len(mats) <= 1:
        return [torch.linalg.svd(M, full_matrices=False, driver=driver) for M in mats]
    dev = mats[0].device
    pool, streams = _svd_workers(dev, n_streams)
    main = torch.cuda.current_stream(dev)
    ready = torch.cuda.Event()
    ready.record(main)
    cost = [M.shape[0] * M.shape[1] * min(M.shape) for M in mats]
    parts: list = [[] for _ in range(n_streams)]
    load = [0] * n_streams
    for i in sorted(range(len(mats)), key=lambda j: -cost[j]):
        k = load.index(min(load))
        parts[k].append(i)
        load[k] += cost[i]
    out: list = [None] * len(mats)
    done = [torch.cuda.Event() for _ in range(n_streams)]

    def run(k):
        s = streams[k]
        with torch.cuda.device(dev), torch.cuda.stream(s):
            s.wait_event(ready)
            for i in parts[k]:
                mats[i].record_stream(s)
                out[i] = torch.linalg.svd(mats[i], full_matrices=False, driver=driver)
            done[k].record(s)

    for f in [pool.submit(run, k) for k in range(n_streams) if parts[k]]:
        f.result()
    for k in range(n_streams):
        if parts[k]:
            main.wait_event(done[k])
    for r in out:
        for x in r:
            x.record_stream(main)
    return out


def truncated_svd(t: SymmetricTensor, left_labels, right_labels, new_bond_label, max_singular_values=None,
                  max_truncation_err=None, normalize=False, driver: str | None = None, n_streams: int = 1):
    """Block-diagonal SVD with global truncation (linalg.py:75-333).

    Sectors = fused flow-weighted charge of the left legs; each sector matrix
    is assembled on the device from the blocks reshaped in their stored leg
    order (linalg.py:186), decomposed with torch.linalg.svd (cuSOLVER), and
    the singular values are merged and stably sorted by -s on the host.
    Returns (U, s_kept (numpy), Vh, s_full (numpy)).
    """
    labels = t.labels()
    l2a = {l: i for i, l in enumerate(labels)}
    la = [l2a[l] for l in left_labels]
    ra = [l2a[l] for l in right_labels]
    sym = t.indices[0].symmetry
    mod = sym.n_values()
    blocks = t.blocks
    grouped: dict = {}
    for key in t.keys:
        q = sum(int(t.indices[i].flow) * int(key[i]) for i in la)
        if mod is not None:
            q %= mod
        grouped.setdefault(q, []).append((tuple(key[i] for i in la), tuple(key[i] for i in ra), key))
    results = {}
    mats = []
    for q, entries in grouped.items():
        lseen, rseen = {}, {}
        for lk, rk, _ in entries:
            lseen.setdefault(lk, len(lseen))
            rseen.setdefault(rk, len(rseen))
        lsz = [int(np.prod([np.count_nonzero(t.indices[a].charges == c) for a, c in zip(la, lk)])) for lk in lseen]
        rsz = [int(np.prod([np.count_nonzero(t.indices[a].charges == c) for a, c in zip(ra, rk)])) for rk in rseen]
        if sum(lsz) == 0 or sum(rsz) == 0:
            continue
        loff = np.concatenate([[0], np.cumsum(lsz)])
        roff = np.concatenate([[0], np.cumsum(rsz)])
        M = torch.zeros((int(loff[-1]), int(roff[-1])), dtype=torch.float64, device=t.data.device)
        for lk, rk, key in entries:
            li, ri = lseen[lk], rseen[rk]
            M[loff[li]:loff[li + 1], roff[ri]:roff[ri + 1]] = blocks[key].reshape(lsz[li], rsz[ri])
        mats.append(M)
        results[q] = [None, None, None, list(lseen), list(rseen), lsz, rsz, loff, roff]
    for r, usv in zip(results.values(), sector_svds(mats, driver, n_streams)):
        r[0:3] = usv
    del mats
    s_all = torch.cat([r[1] for r in results.values()]).cpu().numpy() if results else np.zeros(0)
    s_host, o = {}, 0
    for q, r in results.items():
        s_host[q] = s_all[o:o + r[1].shape[0]]
        o += r[1].shape[0]
    pairs = [(float(v), q, i) for q in results for i, v in enumerate(s_host[q])]
    pairs.sort(key=lambda x: -x[0])
    s_full = np.array([v for v, _, _ in pairs])
    n_total = len(pairs)
    n_keep = n_total
    if max_truncation_err is not None and n_total > 0:
        tot = sum(x[0] ** 2 for x in pairs)
        if tot > 0:
            tr = 0.0
            for i in range(n_total - 1, 0, -1):
                tr += pairs[i][0] ** 2
                if tr / tot > max_truncation_err ** 2:
                    n_keep = i + 1
                    break
            else:
                n_keep = n_total
    if max_singular_values is not None:
        n_keep = min(n_keep, max_singular_values)
    n_keep = max(1, min(n_keep, n_total))
    kept = pairs[:n_keep]
    bond_charges = np.array([q for _, q, _ in kept], dtype=np.int32)
    s_final = np.array([v for v, _, _ in kept])
    if normalize and s_final.sum() > 0:
        s_final = s_final / s_final.sum()
    cols: dict = {}
    for g, (_, q, i) in enumerate(kept):
        cols.setdefault(q, []).append(i)
    left_idx = tuple(t.indices[i] for i in la)
    right_idx = tuple(t.indices[i] for i in ra)
    U_idx = left_idx + (TensorIndex(sym, bond_charges, FlowDirection.OUT, new_bond_label),)
    V_idx = (TensorIndex(sym, bond_charges, FlowDirection.IN, new_bond_label),) + right_idx
    Ub, Vb = {}, {}
    for q, sv in cols.items():
        U, _, Vh, lks, rks, lsz, rsz, loff, roff = results[q]
        sel = torch.as_tensor(sv, device=U.device)
        Ut = U.index_select(1, sel)
        Vt = Vh.index_select(0, sel)
        for li, lk in enumerate(lks):
            shp = tuple(int(np.count_nonzero(t.indices[a].charges == c)) for a, c in zip(la, lk))
            Ub[lk + (q,)] = Ut[loff[li]:loff[li + 1]].reshape(shp + (len(sv),))
        for ri, rk in enumerate(rks):
            shp = tuple(int(np.count_nonzero(t.indices[a].charges == c)) for a, c in zip(ra, rk))
            Vb[(q,) + rk] = Vt[:, roff[ri]:roff[ri + 1]].reshape((len(sv),) + shp)
    validate = not any(int(sum(int(i.flow) * int(q) for i, q in zip(t.indices, k))) != 0 for k in t.keys[:1])
    return (SymmetricTensor(Ub, U_idx, _validate=validate), s_final, SymmetricTensor(Vb, V_idx, _validate=validate),
            s_full)


def scale_bond_axis(t: SymmetricTensor, label, scale) -> SymmetricTensor:
    """Scale along a labelled axis at the positions of each block's charge
    (algorithms/_tensor_utils.py:17-62)."""
    axis = t.labels().index(label)
    idx = t.indices[axis]
    s = torch.as_tensor(np.asarray(scale, dtype=np.float64), device=t.data.device)
    out = torch.empty_like(t.data)
    for i, k in enumerate(t.keys):
        pos = np.nonzero(idx.charges == k[axis])[0]
        shp = t._shapes[i]
        view = [1] * t.ndim
        view[axis] = shp[axis]
        sel = s[torch.as_tensor(pos[: shp[axis]], device=s.device)].view(view)
        out[t.offsets[i]:t.offsets[i + 1]] = (t.data[t.offsets[i]:t.offsets[i + 1]].view(shp) * sel).reshape(-1)
    return SymmetricTensor.from_flat(t.indices, t.keys, out)


def svd_and_truncate_site(theta, site, config, sweep_right=True):
    """(dmrg.py:808-882)"""
    labels = theta.labels()
    left_virt = f"v{site - 1}_{site}" if site > 0 else None
    right_virt = f"v{site + 1}_{site + 2}"
    ll = [l for l in labels if l in (left_virt, f"p{site}") and l is not None]
    rl = [l for l in labels if l in (right_virt, f"p{site + 1}") and l is not None]
    if not ll or not rl:
        n = len(labels)
        ll, rl = list(labels[: n // 2]), list(labels[n // 2:])
    bond = f"v{site}_{site + 1}"
    A, s, B, s_full = truncated_svd(theta, ll, rl, bond, config.max_bond_dim, config.svd_trunc_err,
                                    driver=config.svd_driver, n_streams=config.svd_streams)
    if len(s_full) > len(s):
        err = float(np.sqrt(np.sum(s_full[len(s):] ** 2) / (np.sum(s_full ** 2) + 1e-15)))
    else:
        err = 0.0
    if sweep_right:
        B = scale_bond_axis(B, bond, s)
    else:
        A = scale_bond_axis(A, bond, s)
    return A, s, B, err


# ---------------------------------------------------------------------------
# sweep driver
# ---------------------------------------------------------------------------

class SiteStats(NamedTuple):
    site: int
    chi_theta: int
    lanczos_steps: int
    seconds: float
    flops_per_matvec: float
    matvec_rel_err: float | None  # mixed vs FP64 H_eff on this site's theta (None for FP64 runs)
    diag_seconds: float           # time spent on that residual diagnostic


class SweepStats(NamedTuple):
    sweep: int
    seconds: float
    energy: float
    max_bond: int
    matvecs: int


def two_site_update(site_l, site_r, L, Wl, Wr, R, config, stats: list | None = None, phases: dict | None = None):
    """(dmrg.py:1235-1299)"""
    if phases is not None:
        torch.cuda.synchronize()
    t0 = time.perf_counter()
    shared = set(site_l.labels()) & set(site_r.labels())
    theta = contract(site_l, site_r) if shared else site_l
    ndim0 = theta.ndim
    pad_left = False
    if ndim0 == 3:
        lab0 = theta.labels()[0]
        if not (isinstance(lab0, str) and lab0.startswith("v")):
            pad_left = True
            theta = _pad(theta, True)
        else:
            theta = _pad(theta, False)
    t1 = _tick(phases, "theta", t0)
    op = HeffOperator(L, Wl, Wr, R, theta.indices, theta.keys, config.precision,
                      schedule=None if config.precision == "fp64" else config.heff_schedule)
    fp64 = {}

    def make_fp64():
        # built while the mixed Krylov loop runs (the polish and the FP64
        # energy need it only after that loop's read-back)
        fp64["op"] = HeffOperator(L, Wl, Wr, R, theta.indices, theta.keys, "fp64")
        return fp64["op"]

    need_fp64 = config.precision != "fp64" and config.fp64_energy
    t1 = _tick(phases, "operators", t1)
    tol_rel = NOISE_REL.get(config.precision, 0.0) if config.lanczos_tol_rel is None else config.lanczos_tol_rel
    energy, th, ls = lanczos(op, theta, config.lanczos_max_iter, config.lanczos_tol,
                             make_fp64 if need_fp64 else None, tol_rel,
                             config.fp64_polish_steps if need_fp64 else 0, graph=config.cuda_graph)
    t1 = _tick(phases, "lanczos", t1)
    rel = None
    diag_s = 0.0
    fp64_op = fp64.get("op")
    if fp64_op is not None and config.check_matvec_residual:
        # diagnostic, excluded from the sweep time: mixed vs FP64 matvec of
        # the initial theta (unchanged by the solve)
        t_diag = time.perf_counter()
        x = embed_in_keys(theta, op.keys).data
        ym, yd = op.apply(x), fp64_op.apply(x)
        torch.cuda.synchronize()
        if op.device_error() or fp64_op.device_error():
            raise RuntimeError("tcgen05 GEMM reported a device-side timeout")
        rel = float(vector.nrm2(ym - yd)) / max(float(vector.nrm2(yd)), 1e-300)
        diag_s = time.perf_counter() - t_diag
        _tick(phases, "residual_check", t1)
    if ndim0 == 3:
        th = _unpad(th, pad_left)
    if stats is not None:
        stats.append(SiteStats(-1, int(max(i.dim for i in theta.indices)), ls.steps, time.perf_counter() - t0,
                               op.flops, rel, diag_s))
    return th, energy


def _tick(phases: dict | None, name: str, t_prev: float) -> float:
    """Accumulate device-synchronised wall time of one driver phase."""
    if phases is None:
        return t_prev
    torch.cuda.synchronize()
    t = time.perf_counter()
    phases[name] = phases.get(name, 0.0) + (t - t_prev)
    return t


def dmrg(hamiltonian: TensorNetwork, initial_mps: TensorNetwork, config: DMRGConfig, stats: list | None = None,
         phases: dict | None = None):
    """Two-site symmetric DMRG (dmrg.py:125-305) with every contraction on the GPU."""
    Ln = hamiltonian.n_nodes()
    mps = [initial_mps.get_tensor(i) for i in range(Ln)]
    mpo = [hamiltonian.get_tensor(i) for i in range(Ln)]
    if not all(isinstance(t, SymmetricTensor) for t in mps + mpo):
        raise TypeError("dmrg() requires uniform tensor types: all SymmetricTensor for the GPU back-end.")
    if not config.two_site:
        raise _capi.TnxUnsupported("only two-site DMRG is implemented on the GPU path")
    prec = "fp64"

    def build_right():
        envs = [None] * (Ln + 1)
        envs[Ln] = _trivial_env(False)
        for i in range(Ln - 1, 0, -1):
            envs[i] = update_right_env(envs[i + 1], mps[i], mpo[i], prec)
        return envs

    # The reference builds every left environment up front and rebuilds all
    # left environments before each left-to-right pass and all right
    # environments before each right-to-left pass (dmrg.py:170-172, :182-184,
    # :225).  In the two-site sweep each pass reads left_envs[i] (resp.
    # right_envs[i + 2]) only after its previous step has overwritten it, the
    # boundary entries excepted, so none of those values is ever read: only
    # the boundary left environment and the initial right environments (read
    # by the first left-to-right pass) are computed here, and the sweep's
    # results are the same.
    left = [None] * (Ln + 1)
    left[0] = _trivial_env(True)
    right = build_right()
    energies, terrs = [], []
    energy, converged = 0.0, False
    for sweep in range(config.num_sweeps):
        torch.cuda.synchronize()
        t_sweep = time.perf_counter()
        n_site_stats = len(stats) if stats is not None else 0
        prev = energy
        for i in range(Ln - 1):
            r = right[i + 2] if right[i + 2] is not None else _trivial_env(False)
            th, e = two_site_update(mps[i], mps[i + 1], left[i], mpo[i], mpo[i + 1], r, config, stats, phases)
            energy = float(e)
            t1 = time.perf_counter()
            A, s, B, err = svd_and_truncate_site(th, i, config)
            t1 = _tick(phases, "svd", t1)
            mps[i], mps[i + 1] = A, B
            terrs.append(err)
            left[i + 1] = update_left_env(left[i], A, mpo[i], prec)
            _tick(phases, "env", t1)
        for i in range(Ln - 2, -1, -1):
            r2 = right[i + 2] if right[i + 2] is not None else _trivial_env(False)
            th, e = two_site_update(mps[i], mps[i + 1], left[i], mpo[i], mpo[i + 1], r2, config, stats, phases)
            energy = float(e)
            t1 = time.perf_counter()
            A, s, B, err = svd_and_truncate_site(th, i, config, sweep_right=False)
            t1 = _tick(phases, "svd", t1)
            mps[i], mps[i + 1] = A, B
            terrs.append(err)
            right[i + 1] = update_right_env(r2, B, mpo[i + 1], prec)
            _tick(phases, "env", t1)
        energies.append(energy)
        if stats is not None:
            torch.cuda.synchronize()
            site_stats = [s for s in stats[n_site_stats:] if isinstance(s, SiteStats)]
            stats.append(SweepStats(sweep, time.perf_counter() - t_sweep, energy,
                                    max(max(i.dim for i in t.indices) for t in mps),
                                    sum(s.lanczos_steps for s in site_stats)))
        if config.verbose:
            print(f"Sweep {sweep + 1}/{config.num_sweeps}: E = {energy:.10f}")
        if sweep > 0 and abs(energy - prev) < config.convergence_tol:
            converged = True
            break
    net = TensorNetwork(name="DMRG_MPS")
    for i, t in enumerate(mps):
        net.add_node(i, t)
    for i in range(Ln - 1):
        for lab in sorted(set(mps[i].labels()) & set(mps[i + 1].labels()), key=str):
            net.connect(i, lab, i + 1, lab)
    return DMRGResult(energy, energies, net, terrs, converged)
