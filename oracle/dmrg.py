"""Float64 NumPy restatement of tenax's symmetric two-site DMRG.

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).

Covers the H_eff matvec, the Lanczos solver, the block-sparse truncated
SVD, bond scaling, environment updates and the sweep driver of the
reference's symmetric back-end.
"""

from __future__ import annotations

import numpy as np

from oracle.blocksparse import (
    Leg,
    OTensor,
    blockwise_contract,
    contract_symmetric,
    inner,
    labels_to_subscripts,
    norm,
    t_add,
    t_scale,
)

HEFF_SUBSCRIPTS = "abc,apqd,bpse,eqtf,dfg->cstg"
LEFT_ENV_SUBSCRIPTS = "abc,apd,bpxe,cxf->def"
RIGHT_ENV_SUBSCRIPTS = "abc,dpa,epxb,fxc->def"


def heff_matvec(L, theta, Wl, Wr, R):
    """Two-site H_eff application (algorithms/dmrg.py:1282-1289)."""
    return blockwise_contract([L, theta, Wl, Wr, R], HEFF_SUBSCRIPTS, out_legs=theta.legs)


def heff_flops(L, theta, Wl, Wr, R) -> float:
    """Algorithmic FLOPs of one two-site H_eff application, counted from the
    stored block dims of the operands (the reference's sector structure,
    ``algorithms/dmrg.py:1282-1289``) over the canonical four pairwise stages:
    L.theta over a; .W_l over (b, p); .W_r over (e, q); .R over (d, f).
    Each stage sums 2*m*n*k over its matching block pairs; blocks of zero
    size are skipped; the stage-3 inputs are the distinct stage-2 result
    blocks.  No padding and no dense equivalent."""
    def shapes(t):
        return {k: tuple(int(x) for x in np.shape(v)) for k, v in t.blocks.items() if np.size(v) > 0}

    sL, sT, sWl, sWr, sR = map(shapes, (L, theta, Wl, Wr, R))
    # stage 1: X1[b,c,p,q,d] = L[a,b,c] theta[a,p,q,d]
    rows, cols, ka = {}, {}, {}
    for (qa, qb, qc), (ma, mb, mc) in sL.items():
        rows[qa] = rows.get(qa, 0) + mb * mc
        ka[qa] = ma
    for (qa, qp, qq, qd), (ma, mp, mq, md) in sT.items():
        cols[qa] = cols.get(qa, 0) + mp * mq * md
    flops = sum(2.0 * rows[q] * cols[q] * ka[q] for q in rows if q in cols)
    x1 = {}
    for (qa, qb, qc), (ma, mb, mc) in sL.items():
        for (qa2, qp, qq, qd), (_, mp, mq, md) in sT.items():
            if qa2 == qa:
                x1[(qb, qc, qp, qq, qd)] = (mb, mc, mp, mq, md)
    # stage 2: X2[c,s,e,q,d] = X1[b,c,p,q,d] W_l[b,p,s,e]
    wl_by = {}
    for (qb, qp, qs, qe), d in sWl.items():
        wl_by.setdefault((qb, qp), []).append(((qs, qe), d))
    x2 = {}
    for (qb, qc, qp, qq, qd), (mb, mc, mp, mq, md) in x1.items():
        for (qs, qe), (_, _, ms, me) in wl_by.get((qb, qp), []):
            x2[(qc, qs, qe, qq, qd)] = (mc, ms, me, mq, md)
            flops += 2.0 * (mc * mq * md) * (ms * me) * (mb * mp)
    # stage 3: X3[c,s,t,f,d] = X2[c,s,e,q,d] W_r[e,q,t,f]
    wr_by = {}
    for (qe, qq, qt, qf), d in sWr.items():
        wr_by.setdefault((qe, qq), []).append(((qt, qf), d))
    x3 = {}
    for (qc, qs, qe, qq, qd), (mc, ms, me, mq, md) in x2.items():
        for (qt, qf), (_, _, mt, mf) in wr_by.get((qe, qq), []):
            x3[(qc, qs, qt, qf, qd)] = (mc, ms, mt, mf, md)
            flops += 2.0 * (mc * ms * md) * (mt * mf) * (me * mq)
    # stage 4: Y[c,s,t,g] = X3[c,s,t,f,d] R[d,f,g]
    r_by = {}
    for (qd, qf, qg), (md, mf, mg) in sR.items():
        r_by.setdefault((qf, qd), []).append(mg)
    for (qc, qs, qt, qf, qd), (mc, ms, mt, mf, md) in x3.items():
        for mg in r_by.get((qf, qd), []):
            flops += 2.0 * (mc * ms * mt) * mg * (mf * md)
    return float(flops)


def lanczos(matvec, initial, num_steps, tol):
    """Plain 3-term Lanczos (algorithms/dmrg.py:978-1045).

    No reorthogonalisation; stops when beta < tol.  Returns
    ``(eigenvalue, eigenvector, alphas, betas)``.
    """
    v = t_scale(initial, 1.0 / (norm(initial) + 1e-15))
    basis = [v]
    alphas: list = []
    betas: list = [0.0]
    for step in range(num_steps):
        w = matvec(basis[-1])
        a = float(np.real(inner(basis[-1], w)))
        alphas.append(a)
        w = t_add(w, t_scale(basis[-1], -a))
        if step > 0:
            w = t_add(w, t_scale(basis[-2], -betas[-1]))
        b = float(norm(w))
        betas.append(b)
        if b < tol:
            break
        basis.append(t_scale(w, 1.0 / b))
    n = len(alphas)
    if n == 0:
        return 0.0, v, alphas, betas
    if n == 1:
        return alphas[0], basis[0], alphas, betas
    T = np.diag(alphas) + np.diag(betas[1:n], 1) + np.diag(betas[1:n], -1)
    ev, evec = np.linalg.eigh(T)
    idx = int(np.argmin(ev))
    coefs = evec[:, idx]
    out = t_scale(basis[0], float(coefs[0]))
    for k in range(1, n):
        out = t_add(out, t_scale(basis[k], float(coefs[k])))
    out = t_scale(out, 1.0 / (norm(out) + 1e-15))
    return float(ev[idx]), out, alphas, betas


def pad_boundary(t: OTensor, pad_left: bool) -> OTensor:
    """Add a trivial charge-0 leg (algorithms/dmrg.py:924-952)."""
    if pad_left:
        leg = Leg(np.zeros(1, np.int32), 1, "_pad_l")
        return OTensor((leg,) + t.legs, {(0,) + k: v[np.newaxis] for k, v in t.blocks.items()}, t.modulus)
    leg = Leg(np.zeros(1, np.int32), -1, "_pad_r")
    return OTensor(t.legs + (leg,), {k + (0,): v[..., np.newaxis] for k, v in t.blocks.items()}, t.modulus)


def unpad_boundary(t: OTensor, pad_left: bool) -> OTensor:
    """Remove the trivial leg (algorithms/dmrg.py:955-975)."""
    if pad_left:
        return OTensor(t.legs[1:], {k[1:]: v[0] for k, v in t.blocks.items()}, t.modulus)
    return OTensor(t.legs[:-1], {k[:-1]: v[..., 0] for k, v in t.blocks.items()}, t.modulus)


def trivial_left_env():
    """(algorithms/dmrg.py:890-904)"""
    z = np.zeros(1, np.int32)
    legs = (Leg(z, 1, "env_mps_l"), Leg(z, 1, "env_mpo_l"), Leg(z, -1, "env_mps_conj_l"))
    return OTensor(legs, {(0, 0, 0): np.ones((1, 1, 1))})


def trivial_right_env():
    """(algorithms/dmrg.py:907-921)"""
    z = np.zeros(1, np.int32)
    legs = (Leg(z, -1, "env_mps_r"), Leg(z, -1, "env_mpo_r"), Leg(z, 1, "env_mps_conj_r"))
    return OTensor(legs, {(0, 0, 0): np.ones((1, 1, 1))})


def _pad_site(A: OTensor) -> OTensor:
    if len(A.legs) == 2:
        lab0 = A.legs[0].label
        is_left = isinstance(lab0, str) and lab0.startswith("p")
        return pad_boundary(A, pad_left=is_left)
    return A


def update_left_env(env, A, W):
    """new_L[d,e,f] = L[a,b,c] A[a,p,d] W[b,p,x,e] A*[c,x,f] (algorithms/dmrg.py:1165-1198)."""
    A = _pad_site(A)
    Ac = OTensor(A.legs, {k: np.conj(v) for k, v in A.blocks.items()}, A.modulus)
    out_legs = (A.legs[2], W.legs[3], Ac.legs[2])
    return blockwise_contract([env, A, W, Ac], LEFT_ENV_SUBSCRIPTS, out_legs=out_legs)


def update_right_env(env, B, W):
    """new_R[d,e,f] = R[a,b,c] B[d,p,a] W[e,p,x,b] B*[f,x,c] (algorithms/dmrg.py:1201-1232)."""
    B = _pad_site(B)
    Bc = OTensor(B.legs, {k: np.conj(v) for k, v in B.blocks.items()}, B.modulus)
    out_legs = (B.legs[0], W.legs[0], Bc.legs[0])
    return blockwise_contract([env, B, W, Bc], RIGHT_ENV_SUBSCRIPTS, out_legs=out_legs)


def contract_labels(*tensors, output_labels=None):
    """``tenax.contract`` for symmetric operands (contraction/contractor.py:490-531)."""
    subs, _ = labels_to_subscripts(tensors, output_labels)
    out, _target = contract_symmetric(list(tensors), subs)
    return out


def two_site_update(site_l, site_r, L, Wl, Wr, R, lanczos_max_iter, lanczos_tol):
    """(algorithms/dmrg.py:1235-1299)"""
    shared = set(site_l.labels()) & set(site_r.labels())
    theta = contract_labels(site_l, site_r) if shared else site_l
    original_ndim = len(theta.legs)
    pad_left = False
    if original_ndim == 3:
        lab0 = theta.legs[0].label
        has_left_virt = isinstance(lab0, str) and lab0.startswith("v")
        if not has_left_virt:
            pad_left = True
            theta = pad_boundary(theta, True)
        else:
            theta = pad_boundary(theta, False)
    e, th, _, _ = lanczos(lambda v: heff_matvec(L, v, Wl, Wr, R), theta, lanczos_max_iter, lanczos_tol)
    if original_ndim == 3:
        th = unpad_boundary(th, pad_left)
    return th, e


def truncated_svd(t: OTensor, left_labels, right_labels, new_bond_label, max_sv=None, max_err=None,
                  normalize=False):
    """Block-diagonal SVD with global truncation (linalg.py:75-333).

    Blocks are grouped by the fused flow-weighted charge of the left legs
    (linalg.py:34-69); rows/cols are unique sub-keys in first-seen order;
    singular values are merged and stably sorted by -s (:211), the kept
    bond charges follow that global order (:242).
    Returns ``(U, s_kept, Vh, s_full)``.
    """
    labels = t.labels()
    l2a = {l: i for i, l in enumerate(labels)}
    la = [l2a[l] for l in left_labels]
    ra = [l2a[l] for l in right_labels]
    grouped: dict = {}
    for key, blk in t.blocks.items():
        q = sum(int(t.legs[i].flow) * int(key[i]) for i in la)
        if t.modulus is not None:
            q %= t.modulus
        grouped.setdefault(q, []).append((tuple(key[i] for i in la), tuple(key[i] for i in ra), blk))
    results = {}
    for q, entries in grouped.items():
        lseen: dict = {}
        rseen: dict = {}
        for lk, rk, _ in entries:
            lseen.setdefault(lk, len(lseen))
            rseen.setdefault(rk, len(rseen))
        lks = list(lseen)
        rks = list(rseen)
        lsz = [int(np.prod([np.sum(t.legs[a].charges == c) for a, c in zip(la, lk)])) for lk in lks]
        rsz = [int(np.prod([np.sum(t.legs[a].charges == c) for a, c in zip(ra, rk)])) for rk in rks]
        if sum(lsz) == 0 or sum(rsz) == 0:
            continue
        M = np.zeros((sum(lsz), sum(rsz)))
        for lk, rk, blk in entries:
            li, ri = lseen[lk], rseen[rk]
            r0, c0 = sum(lsz[:li]), sum(rsz[:ri])
            # the reference reshapes the block in its stored leg order, without a
            # transpose to (left, right) (linalg.py:186)
            M[r0:r0 + lsz[li], c0:c0 + rsz[ri]] = blk.reshape(lsz[li], rsz[ri])
        U, s, Vh = np.linalg.svd(M, full_matrices=False)
        results[q] = (U, s, Vh, lks, rks, lsz, rsz)
    pairs = []
    for q, (_, s, _, _, _, _, _) in results.items():
        for i, v in enumerate(s):
            pairs.append((float(v), q, i))
    pairs.sort(key=lambda x: -x[0])
    s_full = np.array([v for v, _, _ in pairs])
    n_total = len(pairs)
    n_keep = n_total
    if max_err is not None and n_total > 0:
        tot = sum(x[0] ** 2 for x in pairs)
        if tot > 0:
            tr = 0.0
            for i in range(n_total - 1, 0, -1):
                tr += pairs[i][0] ** 2
                if tr / tot > max_err ** 2:
                    n_keep = i + 1
                    break
            else:
                n_keep = n_total
    if max_sv is not None:
        n_keep = min(n_keep, max_sv)
    n_keep = max(1, min(n_keep, n_total))
    kept = pairs[:n_keep]
    bond_charges = np.array([q for _, q, _ in kept], dtype=np.int32)
    s_kept = np.array([v for v, _, _ in kept])
    if normalize and s_kept.sum() > 0:  # linalg.py:251-252
        s_kept = s_kept / s_kept.sum()
    cols: dict = {}
    for g, (_, q, i) in enumerate(kept):
        cols.setdefault(q, []).append((g, i))
    left_legs = tuple(t.legs[i] for i in la)
    right_legs = tuple(t.legs[i] for i in ra)
    bond_out = Leg(bond_charges, -1, new_bond_label)
    bond_in = Leg(bond_charges, 1, new_bond_label)
    Ub, Vb = {}, {}
    for q, cl in cols.items():
        U, _, Vh, lks, rks, lsz, rsz = results[q]
        sv = [i for _, i in cl]
        Ut = U[:, sv]
        Vt = Vh[sv, :]
        off = 0
        for li, lk in enumerate(lks):
            shp = tuple(int(np.sum(t.legs[a].charges == c)) for a, c in zip(la, lk))
            Ub[lk + (q,)] = Ut[off:off + lsz[li]].reshape(shp + (len(sv),))
            off += lsz[li]
        off = 0
        for ri, rk in enumerate(rks):
            shp = tuple(int(np.sum(t.legs[a].charges == c)) for a, c in zip(ra, rk))
            Vb[(q,) + rk] = Vt[:, off:off + rsz[ri]].reshape((len(sv),) + shp)
            off += rsz[ri]
    U_t = OTensor(left_legs + (bond_out,), Ub, t.modulus)
    V_t = OTensor((bond_in,) + right_legs, Vb, t.modulus)
    return U_t, s_kept, V_t, s_full


def scale_bond_axis(t: OTensor, label, scale) -> OTensor:
    """Scale along a labelled axis at the positions of each block's charge
    (algorithms/_tensor_utils.py:17-62)."""
    axis = t.labels().index(label)
    leg = t.legs[axis]
    out = {}
    for key, blk in t.blocks.items():
        pos = np.where(leg.charges == key[axis])[0]
        n = blk.shape[axis]
        shp = [1] * len(t.legs)
        shp[axis] = n
        out[key] = blk * np.asarray(scale)[pos[:n]].reshape(shp)
    return OTensor(t.legs, out, t.modulus)


def svd_and_truncate_site(theta, site, max_bond_dim, svd_trunc_err=None, sweep_right=True):
    """(algorithms/dmrg.py:808-882)"""
    labels = theta.labels()
    left_virt = f"v{site - 1}_{site}" if site > 0 else None
    right_virt = f"v{site + 1}_{site + 2}"
    left_phys = f"p{site}"
    right_phys = f"p{site + 1}"
    ll = [l for l in labels if l in (left_virt, left_phys) and l is not None]
    rl = [l for l in labels if l in (right_virt, right_phys) and l is not None]
    if not ll or not rl:
        n = len(labels)
        ll, rl = list(labels[: n // 2]), list(labels[n // 2:])
    bond = f"v{site}_{site + 1}"
    A, s, B, s_full = truncated_svd(theta, ll, rl, bond, max_sv=max_bond_dim, max_err=svd_trunc_err)
    n_keep = len(s)
    if len(s_full) > n_keep:
        tot = np.sum(s_full ** 2)
        tr = np.sum(s_full[n_keep:] ** 2)
        err = float(np.sqrt(tr / (tot + 1e-15)))
    else:
        err = 0.0
    if sweep_right:
        B = scale_bond_axis(B, bond, s)
    else:
        A = scale_bond_axis(A, bond, s)
    return A, s, B, err


def dmrg(mpo, mps, max_bond_dim, num_sweeps, lanczos_max_iter=50, lanczos_tol=1e-12,
         convergence_tol=1e-10, svd_trunc_err=None):
    """Two-site symmetric DMRG sweep driver (algorithms/dmrg.py:125-305).

    ``mpo`` and ``mps`` are lists of OTensor.  Returns
    ``(energy, energies_per_sweep, mps, truncation_errors)``.
    """
    L = len(mpo)
    mps = list(mps)

    def build_left():
        envs = [None] * (L + 1)
        envs[0] = trivial_left_env()
        for i in range(L - 1):
            envs[i + 1] = update_left_env(envs[i], mps[i], mpo[i])
        return envs

    def build_right():
        envs = [None] * (L + 1)
        envs[L] = trivial_right_env()
        for i in range(L - 1, 0, -1):
            envs[i] = update_right_env(envs[i + 1], mps[i], mpo[i])
        return envs

    left = build_left()
    right = build_right()
    energies, terrs = [], []
    energy = 0.0
    for sweep in range(num_sweeps):
        prev = energy
        if sweep > 0:
            left = build_left()
        for i in range(L - 1):
            r = right[i + 2] if right[i + 2] is not None else trivial_right_env()
            th, e = two_site_update(mps[i], mps[i + 1], left[i], mpo[i], mpo[i + 1], r,
                                    lanczos_max_iter, lanczos_tol)
            energy = float(e)
            A, s, B, err = svd_and_truncate_site(th, i, max_bond_dim, svd_trunc_err)
            mps[i], mps[i + 1] = A, B
            terrs.append(err)
            left[i + 1] = update_left_env(left[i], A, mpo[i])
        right = build_right()
        for i in range(L - 2, -1, -1):
            r2 = right[i + 2] if right[i + 2] is not None else trivial_right_env()
            th, e = two_site_update(mps[i], mps[i + 1], left[i], mpo[i], mpo[i + 1], r2,
                                    lanczos_max_iter, lanczos_tol)
            energy = float(e)
            A, s, B, err = svd_and_truncate_site(th, i, max_bond_dim, svd_trunc_err, sweep_right=False)
            mps[i], mps[i + 1] = A, B
            terrs.append(err)
            right[i + 1] = update_right_env(r2, B, mpo[i + 1])
        energies.append(energy)
        if sweep > 0 and abs(energy - prev) < convergence_tol:
            break
    return energy, energies, mps, terrs
