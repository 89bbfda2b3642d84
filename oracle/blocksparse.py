"""Float64 NumPy restatement of tenax's block-sparse storage and contraction.

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).

A tensor here is an ``OTensor``: a tuple of legs (int32 charges per basis
state, flow +1/-1, label) plus ``dict[key -> ndarray]`` of dense blocks, the
same storage model as tenax ``SymmetricTensor`` (core/tensor.py:505-548).
``modulus`` is ``None`` for U(1) and ``n`` for Z_n
(core/symmetry.py:182-255).
"""

from __future__ import annotations

import itertools
from collections import Counter
from dataclasses import dataclass, field

import numpy as np


@dataclass(frozen=True)
class Leg:
    """One tensor leg: charges per basis state, flow, label (core/index.py:43-82)."""

    charges: np.ndarray
    flow: int
    label: object = ""

    @property
    def dim(self) -> int:
        return int(len(self.charges))


@dataclass
class OTensor:
    legs: tuple
    blocks: dict = field(default_factory=dict)
    modulus: int | None = None
    # fermionic grading (FermionParity: Z2; FermionicU1: U(1)), parity q mod 2
    # for the built-in gradings (core/symmetry.py:311-440)
    fermionic: bool = False

    def labels(self):
        return tuple(l.label for l in self.legs)

    def sorted_keys(self):
        # pytree leaf order (core/tensor.py:572-578)
        return sorted(self.blocks.keys())


def fuse(a: int, b: int, modulus: int | None) -> int:
    """U1: a+b; Z_n: (a+b) mod n (core/symmetry.py:194-195, 236-237)."""
    return a + b if modulus is None else (a + b) % modulus


def valid_blocks(charges_list, flows, modulus=None, target=None):
    """All keys with sum(flow*q) == target, in the reference's order.

    Restates ``_compute_valid_blocks`` (core/tensor.py:53-165): unique
    charges sorted per leg (:83), partial sums propagated leg by leg in
    dict-insertion order (:99-128), U1 last leg solved directly (:134-149),
    Z_n last leg enumerated (:150-163).
    """
    n_legs = len(charges_list)
    if n_legs == 0:
        return [()]
    eff_target = 0 if target is None else int(target)
    uniq = [sorted(set(int(q) for q in np.asarray(c).tolist())) for c in charges_list]
    if n_legs == 1:
        return [(q,) for q in uniq[0] if int(flows[0]) * q == eff_target]
    partial: dict = {}
    f0 = int(flows[0])
    for q in uniq[0]:
        partial.setdefault(f0 * q, []).append((q,))
    last = n_legs - 1
    for li in range(1, last):
        fi = int(flows[li])
        nxt: dict = {}
        for q in uniq[li]:
            eq = fi * q
            for prev, combos in partial.items():
                nf = fuse(prev, eq, modulus)
                ext = [c + (q,) for c in combos]
                if nf in nxt:
                    nxt[nf].extend(ext)
                else:
                    nxt[nf] = ext
        partial = nxt
    fl = int(flows[last])
    out = []
    if modulus is None:
        lastset = set(uniq[last])
        for prev, combos in partial.items():
            if fl == 0:
                continue
            ql = (eff_target - prev) * fl
            if ql in lastset:
                for c in combos:
                    out.append(c + (ql,))
    else:
        for q in uniq[last]:
            eq = fl * q
            for prev, combos in partial.items():
                if fuse(prev, eq, modulus) == eff_target:
                    for c in combos:
                        out.append(c + (q,))
    return out


def block_shape(charges_list, key):
    """Block shape = per-leg count of charge == key (core/tensor.py:168-188)."""
    return tuple(int(np.sum(np.asarray(c) == q)) for c, q in zip(charges_list, key))


def random_tensor(legs, rng, modulus=None, target=None, dtype=np.float64):
    """All valid non-empty blocks filled with N(0,1) in sorted-key order.

    Same block selection as ``SymmetricTensor.random_normal``
    (core/tensor.py:653-668); values come from the given numpy Generator.
    """
    charges = [l.charges for l in legs]
    flows = [l.flow for l in legs]
    keys = valid_blocks(charges, flows, modulus, target)
    blocks = {}
    for k in sorted(keys):
        shp = block_shape(charges, k)
        if all(s > 0 for s in shp):
            blocks[k] = rng.standard_normal(shp).astype(dtype)
    return OTensor(tuple(legs), blocks, modulus)


def todense(t: OTensor) -> np.ndarray:
    """Scatter blocks into a dense array (core/tensor.py:760-781)."""
    shape = tuple(l.dim for l in t.legs)
    dtype = next(iter(t.blocks.values())).dtype if t.blocks else np.float64
    out = np.zeros(shape, dtype=dtype)
    for key, blk in t.blocks.items():
        idx = [np.where(l.charges == q)[0] for l, q in zip(t.legs, key)]
        out[np.ix_(*idx)] = blk
    return out


def inner(a: OTensor, b: OTensor) -> float:
    """Sum over common keys of sum(conj(a)*b) (core/tensor.py:311-317)."""
    total = 0.0
    for k, blk in a.blocks.items():
        if k in b.blocks:
            total = total + np.sum(np.conj(blk) * b.blocks[k])
    return total


def norm(t: OTensor) -> float:
    """sqrt(sum |b|^2) over blocks (core/tensor.py:863-868)."""
    if not t.blocks:
        return 0.0
    return float(np.sqrt(sum(np.sum(np.abs(v) ** 2) for v in t.blocks.values())))


def t_scale(t: OTensor, s: float) -> OTensor:
    """Scalar multiply (core/tensor.py:923-928)."""
    return OTensor(t.legs, {k: v * s for k, v in t.blocks.items()}, t.modulus)


def t_add(a: OTensor, b: OTensor) -> OTensor:
    """Key-union addition (core/tensor.py:933-952)."""
    out = {}
    for k in set(a.blocks) | set(b.blocks):
        if k in a.blocks and k in b.blocks:
            out[k] = a.blocks[k] + b.blocks[k]
        elif k in a.blocks:
            out[k] = a.blocks[k]
        else:
            out[k] = b.blocks[k]
    return OTensor(a.legs, out, a.modulus)


def labels_to_subscripts(tensors, output_labels=None):
    """Label -> einsum subscripts (contraction/contractor.py:48-144).

    Returns (subscripts, output_legs).  Raises ValueError for a label used
    more than twice, more than 52 labels, or a bad ``output_labels`` entry.
    """
    counts: Counter = Counter()
    first: dict = {}
    for t in tensors:
        for leg in t.legs:
            counts[leg.label] += 1
            first.setdefault(leg.label, leg)
    for lbl, c in counts.items():
        if c > 2:
            raise ValueError(f"Label {lbl!r} appears {c} times across tensors.")
    free = [l for l, c in counts.items() if c == 1]
    all_labels = sorted(counts.keys(), key=str)
    if len(all_labels) > 52:
        raise ValueError("Too many unique labels")
    chars = "abcdefghijklmnopqrstuvwxyzABCDEFGHIJKLMNOPQRSTUVWXYZ"
    l2c = {l: chars[i] for i, l in enumerate(all_labels)}
    subs = ["".join(l2c[leg.label] for leg in t.legs) for t in tensors]
    if output_labels is None:
        seen = set()
        output_labels = []
        for t in tensors:
            for leg in t.legs:
                if leg.label in free and leg.label not in seen:
                    output_labels.append(leg.label)
                    seen.add(leg.label)
    else:
        fs = set(free)
        for lbl in output_labels:
            if lbl not in fs:
                raise ValueError(f"output_labels contains {lbl!r} which is not a free label.")
    out = "".join(l2c[l] for l in output_labels)
    return ",".join(subs) + "->" + out, tuple(first[l] for l in output_labels)


def parity(q) -> int:
    """Z2 grading of a charge: FermionParity ``q % 2`` and FermionicU1's
    built-in gradings ``|q| % 2`` / ``q % 2`` (core/symmetry.py:345-346,
    367-371) all equal q mod 2 on integers."""
    return int(q) % 2


def inversion_pairs(in_subs, outp):
    """Character pairs whose exchange can flip a fermionic contraction's sign
    (contraction/contractor.py:206-285): all input characters in order, each
    mapped to its target slot (the output characters, then the contracted
    characters by first appearance; the two occurrences of a contracted
    character take consecutive half-slots), and every inverted pair kept."""
    all_chars = [c for s in in_subs for c in s]
    counts = Counter(all_chars)
    contracted = {c for c, n in counts.items() if n >= 2}
    target = list(outp)
    seen = set()
    for c in all_chars:
        if c in contracted and c not in seen:
            target.append(c)
            seen.add(c)
    slot = {}
    for i, c in enumerate(target):
        slot.setdefault(c, i)
    used: Counter = Counter()
    perm = []
    for c in all_chars:
        perm.append(slot[c] * 2 + (used[c] if c in contracted else 0))
        used[c] += 1
    return [(all_chars[i], all_chars[j]) for i in range(len(all_chars)) for j in range(i + 1, len(all_chars))
            if perm[i] > perm[j]]


def koszul_sign(parities, perm) -> int:
    """(-1) per inverted pair of odd elements (core/tensor.py:32-50)."""
    sign = 1
    for i in range(len(perm)):
        for j in range(i + 1, len(perm)):
            if perm[i] > perm[j] and parities[perm[i]] and parities[perm[j]]:
                sign = -sign
    return sign


def transpose(t: OTensor, axes) -> OTensor:
    """Leg permutation with the Koszul sign of fermionic blocks
    (core/tensor.py:836-862)."""
    axes = tuple(axes)
    out = {}
    for key, blk in t.blocks.items():
        v = np.transpose(blk, axes)
        if t.fermionic and koszul_sign([parity(q) for q in key], axes) < 0:
            v = -v
        out[tuple(key[i] for i in axes)] = v
    return OTensor(tuple(t.legs[i] for i in axes), out, t.modulus, t.fermionic)


def dagger(t: OTensor) -> OTensor:
    """Conjugate with dual charges and flows; fermionic blocks take the twist
    phase (-1)^(sum of parities) (core/tensor.py:795-820)."""
    legs = tuple(Leg(np.asarray(dual_charges(l.charges, t.modulus), np.int32), -int(l.flow), l.label)
                 for l in t.legs)
    out = {}
    for key, blk in t.blocks.items():
        v = np.conj(blk)
        if t.fermionic and sum(parity(q) for q in key) % 2:
            v = -v
        out[tuple(int(q) for q in dual_charges(np.asarray(key), t.modulus))] = v
    return OTensor(legs, out, t.modulus, t.fermionic)


def dual_charges(q, modulus):
    """-q (U1) or (-q) mod n (Z_n) (core/symmetry.py:197-204, 239-246)."""
    q = np.asarray(q, dtype=np.int64)
    return (-q) if modulus is None else np.mod(-q, modulus)


def contract_symmetric(tensors, subscripts):
    """Block-sparse contraction with the reference's filtered semantics.

    Restates ``_contract_symmetric`` (contraction/contractor.py:291-484):
    output-target inference (:344-355), valid-output filter (:358-360,
    :439-441), per-tensor contracted-charge signature index sorted by
    contracted char (:373-395), signature intersection (:398-403; with >=3
    operands whose contracted sets differ this yields nothing), product of
    matching blocks with char->charge consistency (:410-436), einsum per
    combination with shape errors skipped (:443-459), summed into the output
    block (:472-476).  Returns ``(OTensor, output_target)``.
    """
    inp, outp = subscripts.split("->")
    in_subs = inp.split(",")
    modulus = tensors[0].modulus
    c2leg = {}
    for t, s in zip(tensors, in_subs):
        for ch, leg in zip(s, t.legs):
            c2leg[ch] = leg
    out_legs = tuple(c2leg[c] for c in outp)
    counts = Counter(inp.replace(",", ""))
    contracted = {c for c, n in counts.items() if n >= 2}

    output_target = None
    total = 0
    for t in tensors:
        if t.blocks:
            tg = set()
            for key in t.blocks:
                tg.add(sum(int(l.flow) * int(q) for l, q in zip(t.legs, key)))
            if len(tg) == 1:
                total += tg.pop()
    if total != 0:
        output_target = total
    valid_out = set(
        valid_blocks([l.charges for l in out_legs], [l.flow for l in out_legs], modulus, output_target)
    )

    csorted = sorted(contracted)
    cpos = {c: i for i, c in enumerate(csorted)}
    sig_maps = []
    for t, s in zip(tensors, in_subs):
        positions = sorted(((cpos[s[p]], p) for p in range(len(s)) if s[p] in contracted))
        m: dict = {}
        for key, arr in t.blocks.items():
            sig = tuple(int(key[p]) for _, p in positions)
            m.setdefault(sig, []).append((key, arr))
        sig_maps.append(m)
    common = set(sig_maps[0].keys()) if sig_maps else set()
    for m in sig_maps[1:]:
        common &= set(m.keys())

    fermionic = any(t.fermionic for t in tensors)
    pairs = inversion_pairs(in_subs, outp) if fermionic else []
    out_blocks: dict = {}
    for sig in common:
        for combo in itertools.product(*[m[sig] for m in sig_maps]):
            c2q: dict = {}
            ok = True
            for (key, _), s in zip(combo, in_subs):
                for ch, q in zip(s, key):
                    if ch in c2q:
                        if c2q[ch] != int(q):
                            ok = False
                            break
                    else:
                        c2q[ch] = int(q)
                if not ok:
                    break
            if not ok:
                continue
            okey = tuple(c2q.get(c, 0) for c in outp)
            if okey not in valid_out:
                continue
            try:
                res = np.einsum(subscripts, *[a for _, a in combo])
            except ValueError:
                continue
            # exchange sign of the leg reordering (contractor.py:460-470)
            sign = 1
            for ci, cj in pairs:
                if parity(c2q[ci]) and parity(c2q[cj]):
                    sign = -sign
            if sign < 0:
                res = -res
            if okey in out_blocks:
                out_blocks[okey] = out_blocks[okey] + res
            else:
                out_blocks[okey] = res
    return OTensor(out_legs, out_blocks, modulus, fermionic), output_target


def blockwise_contract(tensors, subscripts, out_legs=None):
    """Multi-operand block contraction without output filtering.

    Restates ``_blockwise_contract`` (algorithms/dmrg.py:1048-1151):
    backtracking over operands in order and blocks in dict order
    (:1094-1136), char->charge consistency by value equality, output key =
    charges of the output chars (:1097), all combinations contracted and
    summed per output key (:1139-1144), no conservation filter.
    """
    inp, outp = subscripts.split("->")
    in_subs = inp.split(",")
    accum: dict = {}
    arrays: list = []
    c2q: dict = {}

    def rec(ti):
        if ti == len(tensors):
            okey = tuple(c2q.get(c, 0) for c in outp)
            accum.setdefault(okey, []).append(np.einsum(subscripts, *arrays, optimize=True))
            return
        s = in_subs[ti]
        for key, arr in tensors[ti].blocks.items():
            added = []
            ok = True
            for ch, q in zip(s, key):
                q = int(q)
                if ch in c2q:
                    if c2q[ch] != q:
                        ok = False
                        break
                else:
                    c2q[ch] = q
                    added.append(ch)
            if ok:
                arrays.append(arr)
                rec(ti + 1)
                arrays.pop()
            for ch in added:
                del c2q[ch]

    rec(0)
    out = {}
    for k, lst in accum.items():
        tot = lst[0]
        for a in lst[1:]:
            tot = tot + a
        out[k] = tot
    if out_legs is None:
        c2leg = {}
        for t, s in zip(tensors, in_subs):
            for ch, leg in zip(s, t.legs):
                c2leg.setdefault(ch, leg)
        out_legs = tuple(c2leg[c] for c in outp)
    return OTensor(tuple(out_legs), out, tensors[0].modulus)


def blockwise_keys(tensors, subscripts):
    """Output key set of ``blockwise_contract`` (structure only, no arithmetic)."""
    inp, outp = subscripts.split("->")
    in_subs = inp.split(",")
    keys = set()
    c2q: dict = {}

    def rec(ti):
        if ti == len(tensors):
            keys.add(tuple(c2q.get(c, 0) for c in outp))
            return
        s = in_subs[ti]
        for key in tensors[ti].blocks:
            added = []
            ok = True
            for ch, q in zip(s, key):
                q = int(q)
                if ch in c2q:
                    if c2q[ch] != q:
                        ok = False
                        break
                else:
                    c2q[ch] = q
                    added.append(ch)
            if ok:
                rec(ti + 1)
            for ch in added:
                del c2q[ch]

    rec(0)
    return keys


def fused_charges(leg_a: Leg, leg_b: Leg, fused_flow: int, modulus: int | None) -> np.ndarray:
    """Charges of the fused leg, position i*d_b + j holding
    fused_flow * (flow_a q_a[i] + flow_b q_b[j]) (mod n)
    (algorithms/_tensor_utils.py:168-203)."""
    qa = np.asarray(leg_a.charges, dtype=np.int64)
    qb = np.asarray(leg_b.charges, dtype=np.int64)
    raw = int(leg_a.flow) * qa[:, None] + int(leg_b.flow) * qb[None, :]
    q = raw * int(fused_flow)
    if modulus is not None:
        q = np.mod(q, modulus)
    return q.reshape(-1).astype(np.int32)


def fuse_indices(t: OTensor, axis_a: int, axis_b: int, fused_label, fused_flow: int) -> OTensor:
    """Fuse two legs of a block-sparse tensor (_tensor_utils.py:206-325).

    Charge pairs (q_a, q_b) are enumerated over the sorted unique charges of
    each leg, q_a outer; each fused charge's sector stacks the pairs mapping
    to it in that order, a pair occupying d(q_a) * d(q_b) consecutive rows
    (row-major over the two legs' in-sector positions).  Every input block is
    permuted so the two legs are adjacent at min(axis_a, axis_b), merged and
    placed at its pair's offset in a zero-initialised fused block."""
    a, b = sorted((axis_a, axis_b))
    leg_a, leg_b = t.legs[a], t.legs[b]
    fq = fused_charges(leg_a, leg_b, fused_flow, t.modulus)
    ua, ub = np.unique(leg_a.charges), np.unique(leg_b.charges)
    da = {int(q): int(np.sum(leg_a.charges == q)) for q in ua}
    db = {int(q): int(np.sum(leg_b.charges == q)) for q in ub}
    groups: dict = {}
    for qa in ua:
        for qb in ub:
            qf = int(fused_flow) * (int(leg_a.flow) * int(qa) + int(leg_b.flow) * int(qb))
            if t.modulus is not None:
                qf %= t.modulus
            groups.setdefault(qf, []).append((int(qa), int(qb)))
    where, fdim = {}, {}
    for qf, pairs in groups.items():
        off = 0
        for p in pairs:
            where[p] = (qf, off)
            off += da[p[0]] * db[p[1]]
        fdim[qf] = off
    others = [i for i in range(len(t.legs)) if i not in (a, b)]
    legs = [t.legs[i] for i in others]
    legs.insert(a, Leg(fq, int(fused_flow), fused_label))
    perm = others[:a] + [a, b] + others[a:]
    out: dict = {}
    for key, blk in t.blocks.items():
        qf, off = where[(int(key[a]), int(key[b]))]
        x = np.transpose(blk, perm)
        shp = list(x.shape)
        x = x.reshape(shp[:a] + [shp[a] * shp[a + 1]] + shp[a + 2:])
        ok = [key[i] for i in others]
        nk = tuple(ok[:a]) + (qf,) + tuple(ok[a:])
        if nk not in out:
            full = list(x.shape)
            full[a] = fdim[qf]
            out[nk] = np.zeros(full, dtype=x.dtype)
        sl = [slice(None)] * x.ndim
        sl[a] = slice(off, off + x.shape[a])
        out[nk][tuple(sl)] = x
    return OTensor(tuple(legs), out, t.modulus)


def fused_row_map(leg_a: Leg, leg_b: Leg, fused_flow: int, modulus: int | None) -> np.ndarray:
    """Where todense() of a fused tensor puts each natural row.

    Natural row n = i*d_b + j of the pair (leg a, leg b) is row
    off(q_a, q_b) + rank_a(i)*d(q_b) + rank_b(j) of its fused sector
    (fuse_indices above); todense() places a sector's k-th row at the k-th
    position of the fused leg carrying that sector's charge
    (core/tensor.py:760-781).  Returns map[n] = that position."""
    fq = fused_charges(leg_a, leg_b, fused_flow, modulus)
    qa, qb = np.asarray(leg_a.charges), np.asarray(leg_b.charges)
    ua, ub = np.unique(qa), np.unique(qb)
    da = {int(q): int(np.sum(qa == q)) for q in ua}
    db = {int(q): int(np.sum(qb == q)) for q in ub}
    off, fill = {}, {}
    for x in ua:
        for y in ub:
            qf = int(fused_flow) * (int(leg_a.flow) * int(x) + int(leg_b.flow) * int(y))
            if modulus is not None:
                qf %= modulus
            off[(int(x), int(y))] = fill.get(qf, 0)
            fill[qf] = fill.get(qf, 0) + da[int(x)] * db[int(y)]
    pos = {int(q): np.nonzero(fq == q)[0] for q in np.unique(fq)}
    rank_a = np.array([int(np.sum(qa[:i] == qa[i])) for i in range(len(qa))])
    rank_b = np.array([int(np.sum(qb[:j] == qb[j])) for j in range(len(qb))])
    out = np.empty(len(qa) * len(qb), dtype=np.int64)
    for i in range(len(qa)):
        for j in range(len(qb)):
            n = i * len(qb) + j
            k = off[(int(qa[i]), int(qb[j]))] + rank_a[i] * db[int(qb[j])] + rank_b[j]
            out[n] = pos[int(fq[n])][k]
    return out
