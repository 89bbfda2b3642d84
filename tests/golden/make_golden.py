"""Generate the golden fixtures by executing the reference's own tenax source.

Run in the development container only (it needs the read-only reference
checkout; nothing at test or bench time reads it):

    python tests/golden/make_golden.py --ref <reference checkout>/src

The reference modules are loaded by file path under the NumPy stand-in for
jax (``_jax_standin.py``); their outputs -- plus the inputs that produced
them -- are written as small ``.npz``/``.json`` files next to this script.
Inputs are drawn from seeded ``numpy.random.default_rng`` generators so the
same inputs can be rebuilt anywhere.
"""

from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import _jax_standin  # noqa: E402
from fixture_io import pack_tensor  # noqa: E402


def ref_tensor_to_legs(t):
    return [(np.asarray(i.charges), int(i.flow), i.label) for i in t.indices]


def ref_blocks(t):
    return {tuple(int(q) for q in k): np.asarray(v, dtype=np.float64) for k, v in t.blocks.items()}


def dump_tensor(prefix, t, modulus=None):
    return pack_tensor(prefix, ref_tensor_to_legs(t), ref_blocks(t), modulus)


def make_sym_tensor(M, legs, rng, modulus=None, target=None):
    """Build a reference SymmetricTensor with N(0,1) blocks from ``rng``
    over the reference's own valid-block set (sorted-key order)."""
    core = M["tenax.core.tensor"]
    idx = M["tenax.core.index"]
    sym_mod = M["tenax.core.symmetry"]
    sym = sym_mod.U1Symmetry() if modulus is None else sym_mod.ZnSymmetry(modulus)
    indices = tuple(
        idx.TensorIndex(sym, np.asarray(c, np.int32), idx.FlowDirection(f), label=lab) for c, f, lab in legs
    )
    keys = core._compute_valid_blocks(indices, target=target)
    blocks = {}
    for k in sorted(keys):
        _, shp = core._block_slices(indices, k)
        if all(s > 0 for s in shp):
            blocks[k] = rng.standard_normal(shp)
    if target not in (None, 0):
        obj = object.__new__(core.SymmetricTensor)
        obj._indices = indices
        obj._blocks = blocks
        return obj
    return core.SymmetricTensor(blocks, indices)


def c1_virtual_charges():
    """Virtual charges -4..4 with multiplicities proportional to C(8,k),
    total 64: floor with a minimum of 1, then the largest sector absorbs
    the difference.  Result: [1, 2, 7, 14, 16, 14, 7, 2, 1]."""
    from math import comb

    x = np.array([comb(8, k) / 256 * 64 for k in range(9)])
    m = np.maximum(1, np.floor(x)).astype(int)
    diff = 64 - int(m.sum())
    if diff < 0:
        m[int(np.argmax(m))] += diff
    elif diff > 0:
        rem = x - np.floor(x)
        for i in np.argsort(-rem, kind="stable")[:diff]:
            m[i] += 1
    charges = np.concatenate([np.full(mk, q, np.int32) for q, mk in zip(range(-4, 5), m)])
    return charges, m


def gen_valid_blocks(M):
    core = M["tenax.core.tensor"]
    idx = M["tenax.core.index"]
    sm = M["tenax.core.symmetry"]
    cases = [
        ("u1_3leg", None, [[-1, 0, 1, 0], [1, -1], [0, 1, 1, -1, 2]], [1, 1, -1], None),
        ("u1_4leg_target", None, [[-2, 0, 2], [1, -1], [1, -1], [-3, -1, 1, 3]], [1, 1, 1, -1], 2),
        ("u1_env_out", None, [[-3, -1, 1, 3], [0, 2, -2, 0], [-3, -1, 1, 3]], [-1, -1, -1], None),
        ("z3_3leg", 3, [[0, 1, 2, 1], [0, 2], [0, 1, 2]], [1, 1, -1], None),
        ("z3_4leg", 3, [[0, 1, 2], [1, 2], [0, 0, 1], [2, 1, 0]], [1, -1, 1, -1], 1),
        ("z2_2leg", 2, [[0, 1, 1], [1, 0]], [1, -1], None),
        ("u1_1leg", None, [[0, 1, -1]], [1], None),
        ("u1_5leg", None, [[-1, 1], [0, 2, -2], [1, -1], [1, -1], [-2, 0, 2, 4]], [1, 1, -1, 1, -1], None),
    ]
    out = []
    for name, mod, charges, flows, target in cases:
        sym = sm.U1Symmetry() if mod is None else sm.ZnSymmetry(mod)
        inds = tuple(
            idx.TensorIndex(sym, np.array(c, np.int32), idx.FlowDirection(f), label=f"l{i}")
            for i, (c, f) in enumerate(zip(charges, flows))
        )
        keys = core._compute_valid_blocks(inds, target=target)
        out.append(
            {"name": name, "modulus": mod, "charges": charges, "flows": flows, "target": target,
             "keys": [list(map(int, k)) for k in keys]}
        )
    with open(os.path.join(HERE, "valid_blocks.json"), "w") as f:
        json.dump(out, f, indent=1)


def gen_contract(M):
    contractor = M["tenax.contraction.contractor"]
    rng = np.random.default_rng(7)
    arrays = {}
    cases = []

    def add(name, tensors, output_labels=None, modulus=None):
        res = contractor.contract(*tensors, output_labels=output_labels)
        subs, _ = contractor._labels_to_subscripts(tensors, output_labels)
        d = {}
        for i, t in enumerate(tensors):
            d.update(dump_tensor(f"{name}.in{i}", t, modulus))
        d.update(dump_tensor(f"{name}.out", res, modulus))
        arrays.update(d)
        cases.append({"name": name, "n_in": len(tensors), "subscripts": subs,
                      "output_labels": output_labels, "modulus": modulus, "n_out_blocks": len(res.blocks)})

    phys = [-1, 1]
    bond = [-1, 0, 1]
    A = make_sym_tensor(M, [(phys, 1, "p0"), (bond, 1, "bond_left"), (bond, -1, "bond")], rng)
    B = make_sym_tensor(M, [(phys, 1, "p1"), (bond, 1, "bond"), (bond, -1, "bond_right")], rng)
    add("pair_u1", [A, B])
    add("pair_u1_perm", [A, B], output_labels=["bond_right", "p0", "p1", "bond_left"])
    # MPS-like pair with degenerate sectors
    v = [-2, -2, 0, 0, 0, 2, 1, -1, 1]
    A2 = make_sym_tensor(M, [(v, 1, "vl"), ([1, -1], 1, "p"), (v, -1, "m")], rng)
    B2 = make_sym_tensor(M, [(v, 1, "m"), ([1, -1], 1, "q"), (v, -1, "vr")], rng)
    add("mps_pair", [A2, B2])
    # two contracted legs
    C = make_sym_tensor(M, [([0, 1, -1, 1], 1, "x"), ([1, -1], 1, "y"), ([0, 2, 1, -1, 0], -1, "z")], rng)
    D = make_sym_tensor(M, [([0, 2, 1, -1, 0], 1, "z"), ([1, -1], -1, "y"), ([0, 0, 1], -1, "w")], rng)
    add("two_legs", [C, D])
    # Z3
    E = make_sym_tensor(M, [([0, 1, 2, 1], 1, "a"), ([0, 2, 1], -1, "b")], rng, modulus=3)
    F = make_sym_tensor(M, [([0, 2, 1], 1, "b"), ([1, 1, 0, 2], -1, "c"), ([0, 1], 1, "d")], rng, modulus=3)
    add("z3_pair", [E, F], modulus=3)
    # non-zero target on one operand (boundary-site style)
    G = make_sym_tensor(M, [([1, -1, 3], 1, "u"), ([1, -1], 1, "s")], rng, target=2)
    H = make_sym_tensor(M, [([1, -1], -1, "s"), ([1, -1, 3], -1, "t")], rng)
    add("target_pair", [G, H])
    # three operands with differing contracted sets (reference returns no blocks)
    P = make_sym_tensor(M, [(bond, 1, "i"), (bond, -1, "j")], rng)
    Q = make_sym_tensor(M, [(bond, 1, "j"), (bond, -1, "k")], rng)
    R = make_sym_tensor(M, [(bond, 1, "k"), (bond, -1, "l")], rng)
    add("three_chain", [P, Q, R])
    # three operands all contracting the same set
    S1 = make_sym_tensor(M, [(bond, 1, "i"), (bond, -1, "j"), (phys, 1, "p")], rng)
    S2 = make_sym_tensor(M, [(bond, 1, "j"), (phys, -1, "q"), (bond, -1, "k")], rng)
    add("outer_free", [S1, S2])

    np.savez_compressed(os.path.join(HERE, "contract.npz"), **arrays)
    with open(os.path.join(HERE, "contract.json"), "w") as f:
        json.dump(cases, f, indent=1)


def chain_mps_site_legs(i, L, v):
    if i == 0:
        return [([1, -1], 1, f"p{i}"), (v, -1, f"v{i}_{i+1}")]
    if i == L - 1:
        return [(v, 1, f"v{i-1}_{i}"), ([1, -1], 1, f"p{i}")]
    return [(v, 1, f"v{i-1}_{i}"), ([1, -1], 1, f"p{i}"), (v, -1, f"v{i}_{i+1}")]


def build_c1_mps(M, L, seed):
    v, _ = c1_virtual_charges()
    rng = np.random.default_rng(seed)
    core = M["tenax.core.tensor"]
    sites = []
    for i in range(L):
        t = make_sym_tensor(M, chain_mps_site_legs(i, L, v), rng, target=0 if i == L - 1 else None)
        nrm = np.sqrt(sum(np.sum(b ** 2) for b in t.blocks.values()))
        t._blocks = {k: b / nrm for k, b in t.blocks.items()}
        sites.append(t)
    return sites


def gen_dmrg_pieces(M):
    """Small H_eff matvec, env updates, Lanczos and SVD with the reference."""
    dm = M["tenax.algorithms.dmrg"]
    arrays = {}
    L = 6
    mpo = dm.build_mpo_heisenberg(L)
    Ws = [mpo.get_tensor(i) for i in range(L)]
    v = [-2, -1, -1, 0, 0, 0, 1, 1, 2, -1, 0, 1, 3, -3]
    rng = np.random.default_rng(11)
    sites = [make_sym_tensor(M, chain_mps_site_legs(i, L, v), rng, target=0 if i == L - 1 else None)
             for i in range(L)]
    # left env at site 2 and right env at site 4 built by the reference
    envL = dm._build_trivial_left_env_symmetric()
    for i in range(2):
        envL = dm._update_left_env_symmetric(envL, sites[i], Ws[i])
    envR = dm._build_trivial_right_env_symmetric()
    for i in range(L - 1, 3, -1):
        envR = dm._update_right_env_symmetric(envR, sites[i], Ws[i])
    contractor = M["tenax.contraction.contractor"]
    theta = contractor.contract(sites[2], sites[3])
    cache = {}
    hv = dm._blockwise_contract([envL, theta, Ws[2], Ws[3], envR], "abc,apqd,bpse,eqtf,dfg->cstg",
                                output_indices=theta.indices, expr_cache=cache)
    arrays.update(dump_tensor("heff.L", envL))
    arrays.update(dump_tensor("heff.theta", theta))
    arrays.update(dump_tensor("heff.Wl", Ws[2]))
    arrays.update(dump_tensor("heff.Wr", Ws[3]))
    arrays.update(dump_tensor("heff.R", envR))
    arrays.update(dump_tensor("heff.out", hv))
    # env update step outputs
    newL = dm._update_left_env_symmetric(envL, sites[2], Ws[2])
    newR = dm._update_right_env_symmetric(envR, sites[3], Ws[3])
    arrays.update(dump_tensor("envl.A", sites[2]))
    arrays.update(dump_tensor("envl.out", newL))
    arrays.update(dump_tensor("envr.B", sites[3]))
    arrays.update(dump_tensor("envr.out", newR))
    # Lanczos on this H_eff
    matvec = lambda x: dm._blockwise_contract([envL, x, Ws[2], Ws[3], envR], "abc,apqd,bpse,eqtf,dfg->cstg",
                                             output_indices=x.indices, expr_cache=cache)
    e, vec = dm._lanczos_solve_tensor(matvec, theta, 8, 1e-12)
    arrays["lanczos.energy"] = np.array(e)
    arrays.update(dump_tensor("lanczos.vec", vec))
    # truncated SVD of the Lanczos vector (two-site update style)
    U, s, Vh, err = dm._svd_and_truncate_site(vec, 2, M["cfg"](max_bond_dim=5))
    arrays.update(dump_tensor("svd.U", U))
    arrays.update(dump_tensor("svd.Vh", Vh))
    arrays["svd.s"] = np.asarray(s)
    arrays["svd.err"] = np.array(err)
    np.savez_compressed(os.path.join(HERE, "dmrg_pieces.npz"), **arrays)


def gen_dmrg_c1(M, L=20, sweeps=2, lanczos=10, seed=1234):
    dm = M["tenax.algorithms.dmrg"]
    net = M["tenax.network.network"]
    mpo = dm.build_mpo_heisenberg(L)
    sites = build_c1_mps(M, L, seed)
    mps = net.TensorNetwork(name="c1")
    for i, t in enumerate(sites):
        mps.add_node(i, t)
    for i in range(L - 1):
        mps.connect(i, f"v{i}_{i+1}", i + 1, f"v{i}_{i+1}")
    arrays = {}
    for i, t in enumerate(sites):
        arrays.update(dump_tensor(f"mps{i}", t))
    for i in range(L):
        arrays.update(dump_tensor(f"mpo{i}", mpo.get_tensor(i)))
    t0 = time.time()
    cfg = dm.DMRGConfig(max_bond_dim=64, num_sweeps=sweeps, lanczos_max_iter=lanczos, two_site=True)
    res = dm.dmrg(mpo, mps, cfg)
    wall = time.time() - t0
    arrays["energy"] = np.array(res.energy)
    arrays["energies_per_sweep"] = np.array(res.energies_per_sweep)
    arrays["truncation_errors"] = np.array(res.truncation_errors)
    for i in range(L):
        t = res.mps.get_tensor(i)
        arrays.update(dump_tensor(f"final{i}", t))
    np.savez_compressed(os.path.join(HERE, f"dmrg_c1_L{L}.npz"), **arrays)
    v, m = c1_virtual_charges()
    with open(os.path.join(HERE, f"dmrg_c1_L{L}.json"), "w") as f:
        json.dump({"L": L, "sweeps": sweeps, "lanczos": lanczos, "seed": seed, "multiplicities": m.tolist(),
                   "energy": float(res.energy), "energies_per_sweep": [float(x) for x in res.energies_per_sweep],
                   "reference_wall_s_standin": wall}, f, indent=1)
    print(f"C1 L={L}: E={res.energy:.15f} in {wall:.1f}s")


def gen_mpo(M):
    am = M["tenax.algorithms.auto_mpo"]
    arrays = {}
    Lx, Ly = 3, 6
    terms = []
    for (i, j) in cylinder_bonds(Lx, Ly):
        terms += [(1.0, "Sz", i, "Sz", j), (0.5, "Sp", i, "Sm", j), (0.5, "Sm", i, "Sp", j)]
    mpo = am.build_auto_mpo(terms, L=Lx * Ly, symmetric=True, compress=False)
    for i in range(Lx * Ly):
        arrays.update(dump_tensor(f"cyl{i}", mpo.get_tensor(i)))
    dm = M["tenax.algorithms.dmrg"]
    chain = dm.build_mpo_heisenberg(7)
    for i in range(7):
        arrays.update(dump_tensor(f"chain{i}", chain.get_tensor(i)))
    np.savez_compressed(os.path.join(HERE, "mpo.npz"), **arrays)


def cylinder_bonds(Lx, Ly):
    """Nearest-neighbour bonds of an Lx x Ly cylinder, each bond once,
    column-major site order i = x*Ly + y (examples/heisenberg_cylinder.py:43-66)."""
    bonds = []
    for x in range(Lx):
        for y in range(Ly):
            i, j = x * Ly + y, x * Ly + (y + 1) % Ly
            bonds.append((min(i, j), max(i, j)))
            if x < Lx - 1:
                bonds.append((x * Ly + y, (x + 1) * Ly + y))
    return bonds


def gen_fuse(M):
    """fuse_indices (algorithms/_tensor_utils.py:106-325) on symmetric
    tensors: the fused leg's charges, the output blocks (pair-grouped in-sector
    order) and the reference's todense() of the result."""
    tu = M["tenax.algorithms._tensor_utils"]
    idx = M["tenax.core.index"]
    rng = np.random.default_rng(31)
    cases = [
        # name, modulus, legs (charges, flow, label), axis_a, axis_b, fused flow
        ("u1_adjacent", None, [([-1, 0, 1, 0, 1], 1, "a"), ([1, -1, 0], 1, "b"), ([0, 1, -1, 2, 1, 0], -1, "c")],
         0, 1, 1),
        ("u1_interleaved", None, [([-2, -1, 0, 1, 2], -1, "c1_d"), ([2, 1, 0, -1, -2, 0], -1, "u"),
                                  ([0, 1, 2, -1, -2, 0, 1], 1, "I")], 0, 1, 1),
        ("u1_flow_out", None, [([0, 1, -1], 1, "x"), ([1, 1, -1, 0], -1, "y"), ([1, 0, 2, -1], 1, "z")], 1, 2, -1),
        ("u1_nonadjacent", None, [([0, 1, -1, 1], 1, "p"), ([1, -1], 1, "q"), ([0, 2, -2, 0, 1], -1, "r"),
                                  ([1, 0, -1], -1, "s")], 0, 2, 1),
        ("u1_reversed_axes", None, [([1, -1, 0], 1, "p"), ([0, 1, 2], -1, "q"), ([1, 0, -1, 2], -1, "r")], 2, 1, 1),
        ("z3", 3, [([0, 1, 2, 1], 1, "a"), ([0, 2, 1], 1, "b"), ([1, 2, 0, 0], -1, "c")], 0, 1, -1),
    ]
    arrays, meta = {}, []
    for name, mod, legs, a, b, ff in cases:
        T = make_sym_tensor(M, legs, rng, modulus=mod)
        out = tu.fuse_indices(T, a, b, "fused", idx.FlowDirection(ff))
        arrays.update(dump_tensor(f"{name}.in", T, mod))
        arrays.update(dump_tensor(f"{name}.out", out, mod))
        arrays[f"{name}.out_dense"] = np.asarray(out.todense(), dtype=np.float64)
        arrays[f"{name}.in_dense"] = np.asarray(T.todense(), dtype=np.float64)
        meta.append({"name": name, "modulus": mod, "axis_a": a, "axis_b": b, "fused_flow": ff,
                     "n_out_blocks": len(out.blocks), "out_key_order": [list(map(int, k)) for k in out.blocks]})
    np.savez_compressed(os.path.join(HERE, "fuse.npz"), **arrays)
    with open(os.path.join(HERE, "fuse.json"), "w") as fh:
        json.dump(meta, fh, indent=1)


def gen_split_ctm(M):
    """U(1) split-CTMRG (algorithms/_split_ctm_tensor.py) on small symmetric
    site tensors: every projector (recorded at stop_gradient, ket/bra per
    move in call order) and every edge-split SVD (U, s, Vh) the reference
    computed, the final environments (dense) and the energy from
    compute_energy_split_ctm_tensor.  Site legs (u, d, l, r, phys) with flows
    (OUT, IN, OUT, IN, IN), N(0,1) blocks in sorted-key order.

    Trivial-charge cases (all charges 0, the only setting in which the
    reference's own tests check values) and U(1) cases with bond charges
    -k..k of multiplicity 1 and physical charges {-1, +1}.  On the U(1) cases
    the reference's environment becomes exactly zero within the first sweep
    (its charge-tiled re-wrapping of the rotated corners and edges keeps no
    entry), and the fixture records that."""
    sc = M["tenax.algorithms._split_ctm_tensor"]
    sz = np.array([[0.5, 0.0], [0.0, -0.5]])
    sp = np.array([[0.0, 1.0], [0.0, 0.0]])
    H = (np.kron(sz, sz) + 0.5 * np.kron(sp, sp.T) + 0.5 * np.kron(sp.T, sp)).reshape(2, 2, 2, 2)
    # (name, D, bond charges (None: -k..k), chi, sweeps, seed)
    cases = [("triv_d2_chi6", 2, [0, 0], 6, 3, 44), ("triv_d3_chi8", 3, [0, 0, 0], 8, 3, 45),
             ("u1_d3_chi6", 3, None, 6, 2, 41), ("u1_d3_chi9", 3, None, 9, 2, 42)]
    arrays, meta = {"H": H}, {}
    names = ("C1", "C2", "C3", "C4", "T1_ket", "T1_bra", "T2_ket", "T2_bra", "T3_ket", "T3_bra", "T4_ket",
             "T4_bra")
    for name, D, bond, chi, iters, seed in cases:
        rng = np.random.default_rng(seed)
        trivial = bond is not None
        if bond is None:
            bond = list(range(-(D // 2), D // 2 + 1))
        phys = [0, 0] if trivial else [-1, 1]
        legs = [(bond, -1, "u"), (bond, 1, "d"), (bond, -1, "l"), (bond, 1, "r"), (phys, 1, "phys")]
        A = make_sym_tensor(M, legs, rng)
        sg, sv = [], []
        _jax_standin.record_stop_gradient(sg)
        _jax_standin.record_svd(sv)
        t0 = time.time()
        env = sc.ctm_split_tensor(A, chi, max_iter=iters, conv_tol=0.0)
        _jax_standin.record_stop_gradient(None)
        _jax_standin.record_svd(None)
        E = float(sc.compute_energy_split_ctm_tensor(A, env, H, 2))
        assert len(sg) == 8 * iters and len(sv) == 4 * iters, (name, len(sg), len(sv))
        arrays.update(dump_tensor(f"{name}.A", A))
        for i, P in enumerate(sg):
            arrays[f"{name}.P{i}"] = P
        for i, (U, s, Vh) in enumerate(sv):
            arrays[f"{name}.svdU{i}"] = U
            arrays[f"{name}.svds{i}"] = s
            arrays[f"{name}.svdVh{i}"] = Vh
        for nm, x in zip(names, env):
            arrays[f"{name}.{nm}"] = np.asarray(x.todense(), dtype=np.float64)
        meta[name] = {"D": D, "bond_charges": [int(q) for q in bond], "phys_charges": phys, "chi": chi,
                      "chi_I": chi, "iters": iters, "seed": seed, "energy": E}
        print(f"split ctm {name}: E={E:.15f} ({time.time() - t0:.1f} s)", flush=True)
    np.savez_compressed(os.path.join(HERE, "split_ctm.npz"), **arrays)
    with open(os.path.join(HERE, "split_ctm.json"), "w") as fh:
        json.dump(meta, fh, indent=1)


def gen_ctm_tensor(M):
    """Block-sparse standard CTMRG (algorithms/_ctm_tensor.py): every
    projector the reference computed (the dense P recorded at its
    stop_gradient call, in call order), the final environments as
    block-sparse tensors (keys + data) and the energy from
    compute_energy_ctm_tensor; one checkerboard (2-site) case with
    compute_energy_ctm_tensor_2site.

    Site legs (u, d, l, r, phys) with flows (OUT, IN, OUT, IN, IN), N(0,1)
    blocks in sorted-key order.  Trivial-charge cases carry values; on the
    U(1) and Z2 cases the reference's trivial chi_new charges keep only the
    fused charge-0 rows of each projector and the environment is exactly
    zero after the first sweep (the fixture records its block structure).
    Charges whose grown corners differ in sector height make the
    reference's per-sector reshape fail; that case records the error."""
    ct = M["tenax.algorithms._ctm_tensor"]
    core = M["tenax.core.tensor"]
    sz = np.array([[0.5, 0.0], [0.0, -0.5]])
    sp = np.array([[0.0, 1.0], [0.0, 0.0]])
    H = (np.kron(sz, sz) + 0.5 * np.kron(sp, sp.T) + 0.5 * np.kron(sp.T, sp)).reshape(2, 2, 2, 2)
    # (name, bond charges, phys charges, modulus, chi, sweeps, method, warm-up, seed, DenseTensor input)
    cases = [("triv_d2_chi6", [0, 0], [0, 0], None, 6, 3, "eigh", 0, 44, False),
             ("triv_d3_chi10", [0, 0, 0], [0, 0], None, 10, 2, "eigh", 0, 45, False),
             ("triv_d2_chi5_qr", [0, 0], [0, 0], None, 5, 4, "qr", 2, 46, False),
             ("dense_d2_chi6", [0, 0], [0, 0], None, 6, 3, "eigh", 0, 47, True),
             ("dense_d2_chi4_qr", [0, 0], [0, 0], None, 4, 3, "qr", 1, 48, True),
             ("u1_d3_chi8", [-1, 0, 1], [-1, 1], None, 8, 2, "eigh", 0, 41, False),
             ("z2_d3_chi6", [0, 0, 1], [0, 1], 2, 6, 2, "eigh", 0, 7, False),
             ("u1_d2_chi6_err", [0, 1], [0, 1], None, 6, 1, "eigh", 0, 7, False)]
    arrays, meta = {"H": H}, {}
    for name, bond, phys, mod, chi, iters, method, warm, seed, dense in cases:
        rng = np.random.default_rng(seed)
        legs = [(bond, -1, "u"), (bond, 1, "d"), (bond, -1, "l"), (bond, 1, "r"), (phys, 1, "phys")]
        A = make_sym_tensor(M, legs, rng, modulus=mod)
        arrays.update(dump_tensor(f"{name}.A", A, mod))
        A_in = core.DenseTensor(A.todense(), A.indices) if dense else A
        sg = []
        _jax_standin.record_stop_gradient(sg)
        t0 = time.time()
        entry = {"bond_charges": bond, "phys_charges": phys, "modulus": mod, "chi": chi, "iters": iters,
                 "method": method, "warmup": warm, "seed": seed, "dense": dense}
        try:
            env = ct.ctm_tensor(A_in, chi, max_iter=iters, conv_tol=0.0, projector_method=method,
                                qr_warmup_steps=warm)
        except ValueError as e:
            _jax_standin.record_stop_gradient(None)
            entry["error"] = str(e)
            entry["n_projectors_before_error"] = len(sg)
            meta[name] = entry
            print(f"ctm_tensor {name}: ValueError {e}", flush=True)
            continue
        _jax_standin.record_stop_gradient(None)
        E = float(ct.compute_energy_ctm_tensor(A_in, env, H, 2))
        assert len(sg) == 4 * iters, (name, len(sg))
        for i, P in enumerate(sg):
            arrays[f"{name}.P{i}"] = np.asarray(P, dtype=np.float64)
        for f in env._fields:
            x = getattr(env, f)
            if dense:
                arrays[f"{name}.{f}"] = np.asarray(x.todense(), dtype=np.float64)
            else:
                arrays.update(dump_tensor(f"{name}.{f}", x, mod))
        entry["energy"] = E
        meta[name] = entry
        print(f"ctm_tensor {name}: E={E:.15f} ({time.time() - t0:.1f} s)", flush=True)

    # checkerboard cell, trivial charges
    name, chi, iters = "cb_d2_chi6", 6, 2
    sites = []
    for s, seed in (("A", 99), ("B", 200)):
        rng = np.random.default_rng(seed)
        legs = [([0, 0], -1, "u"), ([0, 0], 1, "d"), ([0, 0], -1, "l"), ([0, 0], 1, "r"), ([0, 0], 1, "phys")]
        sites.append(make_sym_tensor(M, legs, rng))
        arrays.update(dump_tensor(f"{name}.{s}", sites[-1]))
    sg = []
    _jax_standin.record_stop_gradient(sg)
    env_A, env_B = ct.ctm_tensor_2site(sites[0], sites[1], chi, max_iter=iters, conv_tol=0.0)
    _jax_standin.record_stop_gradient(None)
    E = float(ct.compute_energy_ctm_tensor_2site(sites[0], sites[1], env_A, env_B, H, 2))
    assert len(sg) == 8 * iters, len(sg)
    for i, P in enumerate(sg):
        arrays[f"{name}.P{i}"] = np.asarray(P, dtype=np.float64)
    for s, env in (("A", env_A), ("B", env_B)):
        for f in env._fields:
            arrays.update(dump_tensor(f"{name}.env{s}.{f}", getattr(env, f)))
    meta[name] = {"chi": chi, "iters": iters, "seeds": [99, 200], "energy": E}
    print(f"ctm_tensor {name}: E={E:.15f}", flush=True)
    np.savez_compressed(os.path.join(HERE, "ctm_tensor.npz"), **arrays)
    with open(os.path.join(HERE, "ctm_tensor.json"), "w") as fh:
        json.dump(meta, fh, indent=1)


NETFILE_SOURCES = [
    ("pair", "# a pair\nA: i, j\nB: j, k\nTOUT: k, i\n"),
    ("chain3", "A: i, j\nB: j, k\nC: k, l\n"),
    ("chain3_order", "A: i, j\nB: j, k\nC: k, l\nTOUT: l, i\nORDER: ((A, B), C)\n"),
    ("chain3_order_right", "A: i, j\nB: j, k\nC: k, l\nORDER: (A,(B,C))\n"),
    ("ring_scalar", "A: i, j\nB: j, i\nTOUT:\n"),
    ("no_tout", "X: a, b, c\nY: c, d\n"),
    ("err_no_colon", "A i j\n"),
    ("err_dup_tout", "A: i\nTOUT: i\nTOUT: i\n"),
    ("err_dup_order", "A: i, j\nB: j\nORDER: (A,B)\nORDER: (A,B)\n"),
    ("err_dup_name", "A: i\nA: j\n"),
    ("err_no_labels", "A:\n"),
    ("err_empty", "# nothing\n\n"),
    ("err_label3", "A: i\nB: i\nC: i\n"),
    ("err_order_unknown", "A: i, j\nB: j\nORDER: (A, Z)\n"),
    ("err_order_syntax", "A: i, j\nB: j\nORDER: (A B)\n"),
    ("err_order_trailing", "A: i, j\nB: j\nORDER: (A,B) C\n"),
    ("err_order_close", "A: i, j\nB: j\nORDER: (A,B\n"),
    ("err_tout_not_free", "A: i, j\nB: j, k\nTOUT: j\n"),
]


def gen_netfile(M):
    """Network files (network/netfile.py): the reference's parse result,
    pairwise ORDER steps, precomputed subscripts or its error text for each
    source above, and NetworkBlueprint.launch() on U(1) tensors: a pair with
    a TOUT permutation, a 3-chain without ORDER (the reference's filtered
    N-operand contraction returns no blocks), the same chain with ORDER
    left and right nested, a closed ring contracted to a scalar, and slots
    filled through label_order and through a transpose."""
    nf = M["tenax.network.netfile"]
    out = {"parse": {}, "launch": {}}
    for name, src in NETFILE_SOURCES:
        try:
            bp = nf.NetworkBlueprint(src)
            spec = nf.parse_netfile(src)
            steps = nf._parse_order(spec["order"], set(spec["tensors"])) if spec["order"] is not None else None
            out["parse"][name] = {"source": src, "tensors": spec["tensors"], "tout": spec["tout"],
                                  "order": spec["order"], "steps": steps, "subscripts": bp.subscripts,
                                  "tensor_names": bp.tensor_names, "output_labels": bp.output_labels}
        except ValueError as e:
            out["parse"][name] = {"source": src, "error": str(e)}
    rng = np.random.default_rng(31)
    bond = [-1, 0, 1, 0]
    arrays = {}

    def t(labels, flows):
        return make_sym_tensor(M, [(bond, f, lab) for lab, f in zip(labels, flows)], rng)

    A = t("ij", (1, -1))
    B = t("jk", (1, -1))
    Cc = t("kl", (1, -1))
    Bring = t("ji", (1, -1))
    for nm, x in (("A", A), ("B", B), ("C", Cc), ("Bring", Bring)):
        arrays.update(dump_tensor(f"in.{nm}", x))
    runs = [("pair", {"A": A, "B": B}), ("chain3", {"A": A, "B": B, "C": Cc}),
            ("chain3_order", {"A": A, "B": B, "C": Cc}), ("chain3_order_right", {"A": A, "B": B, "C": Cc}),
            ("ring_scalar", {"A": A, "B": Bring})]
    for name, slots in runs:
        bp = nf.NetworkBlueprint(dict(NETFILE_SOURCES)[name])
        bp.put_tensors(slots)
        res = bp.launch()
        arrays.update(dump_tensor(f"out.{name}", res))
        out["launch"][name] = {"n_blocks": len(res.blocks), "labels": [str(x) for x in res.labels()]}
    # slots filled through label_order (relabel) and through a transpose
    bp = nf.NetworkBlueprint(dict(NETFILE_SOURCES)["pair"])
    bp.put_tensor("A", A.relabels({"i": "x", "j": "y"}), label_order=["x", "y"])
    bp.put_tensor("B", B.transpose((1, 0)))
    res = bp.launch()
    arrays.update(dump_tensor("out.pair_label_order", res))
    out["launch"]["pair_label_order"] = {"n_blocks": len(res.blocks), "labels": [str(x) for x in res.labels()]}
    np.savez_compressed(os.path.join(HERE, "netfile.npz"), **arrays)
    with open(os.path.join(HERE, "netfile.json"), "w") as fh:
        json.dump(out, fh, indent=1)
    print(f"netfile: {len(out['parse'])} parse cases, {len(out['launch'])} launches", flush=True)


def gen_ctm(M):
    """Dense 1-site CTMRG (algorithms/ipeps.py): environments, corner
    singular values and NN Heisenberg energies from the reference's own
    ``ctm`` / ``compute_energy_ctm``.

    The reference's CTM on random site tensors does not converge: its
    truncation keeps a subspace whose edge is re-chosen every sweep, and a
    1e-14 change of A moves the 30-sweep energy by ~1e-2.  So the small cases
    also store every projector the reference computed (recorded at its
    ``jax.lax.stop_gradient`` call); replaying them makes the rest of the
    computation a smooth function that other implementations must match to
    rounding.  The D=4, chi=80, 30-sweep QR case stores the free-running
    energy and corner spectra only (a statistical reference)."""
    ip = M["tenax.algorithms.ipeps"]
    sz = np.array([[0.5, 0.0], [0.0, -0.5]])
    sp = np.array([[0.0, 1.0], [0.0, 0.0]])
    H = (np.kron(sz, sz) + 0.5 * np.kron(sp, sp.T) + 0.5 * np.kron(sp.T, sp)).reshape(2, 2, 2, 2)
    cases = [
        ("qr_small", 2, 6, 6, "qr", 0, 11),
        ("eigh_small", 2, 5, 4, "eigh", 0, 12),
        ("qr_mid", 3, 16, 6, "qr", 0, 13),
        ("qr_warm", 2, 6, 5, "qr", 2, 14),
        ("c4", 4, 80, 30, "qr", 0, 2024),
    ]
    arrays = {"H": H}
    meta = {}
    for name, D, chi, iters, method, warm, seed in cases:
        rng = np.random.default_rng(seed)
        A = rng.standard_normal((D, D, D, D, 2)) / np.sqrt(2.0 * D ** 4)
        cfg = ip.CTMConfig(chi=chi, max_iter=iters, conv_tol=0.0, renormalize=True,
                           projector_method=method, qr_warmup_steps=warm)
        t0 = time.time()
        log: list = []
        _jax_standin.record_stop_gradient(log)
        env = ip.ctm(A, cfg)
        _jax_standin.record_stop_gradient(None)
        E = float(ip.compute_energy_ctm(A, env, H, 2))
        assert len(log) == 4 * iters, (name, len(log))
        arrays[f"{name}.A"] = A
        if name != "c4":
            for i, P in enumerate(log):
                arrays[f"{name}.P{i}"] = P
        for nm, x in zip(("C1", "C2", "C3", "C4", "T1", "T2", "T3", "T4"), env):
            x = np.asarray(x, dtype=np.float64)
            if name != "c4":
                arrays[f"{name}.{nm}"] = x
            if nm.startswith("C"):
                arrays[f"{name}.sv_{nm}"] = np.linalg.svd(x, compute_uv=False)
        meta[name] = {"D": D, "chi": chi, "iters": iters, "method": method, "warmup": warm, "seed": seed,
                      "energy": E}
        print(f"ctm {name}: E={E:.15f} ({time.time() - t0:.1f} s)", flush=True)
    np.savez_compressed(os.path.join(HERE, "ctm.npz"), **arrays)
    with open(os.path.join(HERE, "ctm.json"), "w") as fh:
        json.dump(meta, fh, indent=1)


def make_fermion_tensor(M, sym, legs, rng):
    """A reference SymmetricTensor over a fermionic symmetry with N(0,1)
    blocks on its valid-block set (sorted-key order)."""
    core = M["tenax.core.tensor"]
    idx = M["tenax.core.index"]
    indices = tuple(
        idx.TensorIndex(sym, np.asarray(c, np.int32), idx.FlowDirection(f), label=lab) for c, f, lab in legs
    )
    blocks = {}
    for k in sorted(core._compute_valid_blocks(indices)):
        _, shp = core._block_slices(indices, k)
        if all(s > 0 for s in shp):
            blocks[k] = rng.standard_normal(shp)
    return core.SymmetricTensor(blocks, indices)


def gen_fermion(M):
    """Fermionic symmetries (FermionParity, FermionicU1): label contractions
    whose leg reordering exchanges odd charges (contractor.py:206-285,
    :460-470), transposes with the Koszul sign (core/tensor.py:32-50,
    :836-862) and daggers with the twist phase (core/tensor.py:795-820)."""
    contractor = M["tenax.contraction.contractor"]
    symm = M["tenax.core.symmetry"]
    rng = np.random.default_rng(29)
    arrays, cases = {}, []
    syms = {"fermion_parity": (symm.FermionParity(), 2), "fermionic_u1": (symm.FermionicU1(), None)}
    for sname, (sym, mod) in syms.items():
        if mod == 2:
            a = [0, 1, 1, 0, 1]
            b = [1, 0, 0, 1]
            p = [0, 1]
        else:
            a = [-1, 0, 0, 1, 2, 1]
            b = [0, 1, -1, 1]
            p = [0, 1]
        A = make_fermion_tensor(M, sym, [(a, 1, "i"), (p, 1, "s"), (b, -1, "k"), (p, -1, "t")], rng)
        B = make_fermion_tensor(M, sym, [(b, 1, "k"), (p, 1, "u"), (a, -1, "j")], rng)
        C = make_fermion_tensor(M, sym, [(p, 1, "t"), (b, -1, "m"), (a, 1, "j")], rng)
        for name, ts, ol in (
            ("pair", [A, B], None),
            ("pair_perm", [A, B], ["j", "u", "t", "s", "i"]),
            ("pair_rev", [B, A], None),
            ("two_legs", [A, C], None),
            ("two_legs_perm", [A, C], ["m", "s", "j", "k", "i"]),
        ):
            res = contractor.contract(*ts, output_labels=ol)
            subs, _ = contractor._labels_to_subscripts(ts, ol)
            cname = f"{sname}.{name}"
            for i, t in enumerate(ts):
                arrays.update(dump_tensor(f"{cname}.in{i}", t, mod))
            arrays.update(dump_tensor(f"{cname}.out", res, mod))
            cases.append({"name": cname, "kind": "contract", "symmetry": sname, "modulus": mod,
                          "subscripts": subs, "output_labels": ol, "n_in": len(ts), "n_out_blocks": len(res.blocks)})
        for axes in ((1, 0, 3, 2), (3, 2, 1, 0), (2, 0, 3, 1)):
            res = A.transpose(axes)
            cname = f"{sname}.transpose_{''.join(map(str, axes))}"
            arrays.update(dump_tensor(f"{cname}.in0", A, mod))
            arrays.update(dump_tensor(f"{cname}.out", res, mod))
            cases.append({"name": cname, "kind": "transpose", "symmetry": sname, "modulus": mod, "axes": list(axes)})
        res = A.dagger()
        cname = f"{sname}.dagger"
        arrays.update(dump_tensor(f"{cname}.in0", A, mod))
        arrays.update(dump_tensor(f"{cname}.out", res, mod))
        cases.append({"name": cname, "kind": "dagger", "symmetry": sname, "modulus": mod})
    np.savez_compressed(os.path.join(HERE, "fermion.npz"), **arrays)
    with open(os.path.join(HERE, "fermion.json"), "w") as f:
        json.dump(cases, f, indent=1)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", required=True, help="the reference checkout's src directory")
    ap.add_argument("--only", default="")
    args = ap.parse_args()
    mods = _jax_standin.load_reference(args.ref, [
        "tenax.core.symmetry", "tenax.core.index", "tenax.core.tensor", "tenax.linalg",
        "tenax.contraction.contractor", "tenax.network.network", "tenax.algorithms._tensor_utils",
        "tenax.algorithms.auto_mpo", "tenax.algorithms.dmrg", "tenax.algorithms.ipeps",
        "tenax.algorithms._split_ctm_tensor", "tenax.algorithms._ctm_tensor", "tenax.network.netfile",
    ])
    mods["cfg"] = mods["tenax.algorithms.dmrg"].DMRGConfig
    todo = args.only.split(",") if args.only else ["valid", "contract", "pieces", "mpo", "c1", "ctm", "fuse", "split",
                                                       "ctm_tensor", "netfile", "fermion"]
    if "valid" in todo:
        gen_valid_blocks(mods)
    if "contract" in todo:
        gen_contract(mods)
    if "pieces" in todo:
        gen_dmrg_pieces(mods)
    if "mpo" in todo:
        gen_mpo(mods)
    if "c1" in todo:
        gen_dmrg_c1(mods)
    if "ctm" in todo:
        gen_ctm(mods)
    if "fuse" in todo:
        gen_fuse(mods)
    if "split" in todo:
        gen_split_ctm(mods)
    if "ctm_tensor" in todo:
        gen_ctm_tensor(mods)
    if "netfile" in todo:
        gen_netfile(mods)
    if "fermion" in todo:
        gen_fermion(mods)


if __name__ == "__main__":
    main()
