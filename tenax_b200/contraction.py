"""Label-based block-sparse contraction on the GPU.

Same surface as tenax ``contraction/contractor.py``: ``contract`` (:490-531),
``contract_with_subscripts`` (:534-569) and the label-to-subscript mapping
(:48-144).  Symmetric operands go through the C ABI planner + kernels with
``_contract_symmetric`` semantics (:291-484); ``blockwise_contract`` gives
the DMRG engine's ``_blockwise_contract`` semantics (algorithms/dmrg.py:
1048-1151).  Plans are cached by block structure.
"""

from __future__ import annotations

import ctypes as C
import string
from collections import Counter, OrderedDict

import numpy as np
import torch

from tenax_b200 import _capi
from tenax_b200.tensor import SymmetricTensor, _device

_PLANS: "OrderedDict[tuple, Plan]" = OrderedDict()
_PLAN_CACHE_SIZE = 512
DEFAULT_PRECISION = "fp64"


def _stream_ptr() -> int:
    return torch.cuda.current_stream().cuda_stream


class Plan:
    """An owned ``tnx_plan`` handle plus its output structure."""

    def __init__(self, tensors, in_subs, out_subs, mode, out_indices, fermionic: bool = False):
        self.holders = [
            _capi.DescHolder([i.charges for i in t.indices], [int(i.flow) for i in t.indices], t.keys, s)
            for t, s in zip(tensors, in_subs)
        ]
        descs = (_capi.TensorDesc * len(tensors))(*[h.desc for h in self.holders])
        out_h = _capi.DescHolder([i.charges for i in out_indices], [int(i.flow) for i in out_indices], [], None)
        modulus = tensors[0].indices[0].symmetry.n_values() if tensors[0].indices else None
        h = C.c_void_p()
        _capi.check(_capi.LIB.tnx_plan_create_graded(descs, len(tensors), out_subs.encode(), mode,
                                                     0 if modulus is None else int(modulus), out_h.charges.ctypes.data,
                                                     out_h.leg_dims.ctypes.data, out_h.flows.ctypes.data,
                                                     int(bool(fermionic)), C.byref(h)))
        self.handle = h
        nb, tot, has_t, tgt = C.c_int64(), C.c_int64(), C.c_int32(), C.c_int64()
        _capi.check(_capi.LIB.tnx_plan_output(h, C.byref(nb), None, C.byref(tot), C.byref(has_t), C.byref(tgt)))
        nl = len(out_subs)
        keys = np.zeros(max(1, nb.value * max(nl, 1)), dtype=np.int32)
        _capi.check(_capi.LIB.tnx_plan_output(h, C.byref(nb), keys.ctypes.data, None, None, None))
        self.out_keys = ([tuple(int(q) for q in r) for r in keys[: nb.value * nl].reshape(-1, nl)]
                         if nl else [()] * nb.value)
        self.total = tot.value
        self.target = tgt.value if has_t.value else None
        self.flops = float(_capi.LIB.tnx_plan_flops(h))

    def execute(self, tensors, precision: str) -> torch.Tensor:
        out = torch.empty(max(1, self.total), dtype=torch.float64, device=_device())
        ptrs = (C.c_void_p * max(1, len(tensors)))(*[t.data.data_ptr() for t in tensors])
        _capi.check(_capi.LIB.tnx_plan_execute(self.handle, ptrs, out.data_ptr(), _capi.PRECISIONS[precision], None,
                                               0, _stream_ptr()))
        return out[: self.total]

    def __del__(self):
        if getattr(self, "handle", None) and _capi is not None and _capi.LIB is not None:
            _capi.LIB.tnx_plan_destroy(self.handle)
            self.handle = None


def _fermionic(tensors) -> bool:
    """Whether the operands carry a fermionic grading the engine signs with
    (parity = charge mod 2); other gradings are rejected."""
    sym = tensors[0].indices[0].symmetry if tensors and tensors[0].indices else None
    if sym is None or not sym.is_fermionic:
        return False
    if not getattr(sym, "builtin_grading", True):
        raise _capi.TnxUnsupported("fermionic contraction with a custom grading function: only the built-in "
                                   "gradings (parity = charge mod 2) are supported")
    return True


def _structure_key(tensors, in_subs, out_subs, mode, out_indices, fermionic=False):
    parts = [mode, out_subs, bool(fermionic)]
    for t, s in zip(tensors, in_subs):
        parts.append((s, tuple(int(i.flow) for i in t.indices), tuple(i.charges.tobytes() for i in t.indices),
                      tuple(t.keys)))
    parts.append(tuple((int(i.flow), i.charges.tobytes()) for i in out_indices))
    return tuple(parts)


def get_plan(tensors, in_subs, out_subs, mode, out_indices, fermionic: bool = False) -> Plan:
    key = _structure_key(tensors, in_subs, out_subs, mode, out_indices, fermionic)
    p = _PLANS.get(key)
    if p is not None:
        _PLANS.move_to_end(key)
        return p
    p = Plan(tensors, in_subs, out_subs, mode, out_indices, fermionic)
    _PLANS[key] = p
    if len(_PLANS) > _PLAN_CACHE_SIZE:
        _PLANS.popitem(last=False)
    return p


def _labels_to_subscripts(tensors, output_labels=None):
    """Labels -> einsum subscripts and output indices (contractor.py:48-144)."""
    counts: Counter = Counter()
    first: dict = {}
    for t in tensors:
        for idx in t.indices:
            counts[idx.label] += 1
            first.setdefault(idx.label, idx)
    for lbl, c in counts.items():
        if c > 2:
            raise ValueError(f"Label {lbl!r} appears {c} times across tensors. "
                             f"Labels must appear at most 2 times (one per tensor to contract).")
    free = [l for l, c in counts.items() if c == 1]
    all_labels = sorted(counts.keys(), key=str)
    if len(all_labels) > 52:
        raise ValueError(f"Too many unique labels ({len(all_labels)}) for einsum encoding. "
                         f"Maximum supported is 52 (a-z + A-Z).")
    chars = string.ascii_lowercase + string.ascii_uppercase
    l2c = {l: chars[i] for i, l in enumerate(all_labels)}
    subs = ["".join(l2c[i.label] for i in t.indices) for t in tensors]
    if output_labels is None:
        seen: set = set()
        output_labels = []
        for t in tensors:
            for i in t.indices:
                if i.label in free and i.label not in seen:
                    output_labels.append(i.label)
                    seen.add(i.label)
    else:
        fs = set(free)
        for lbl in output_labels:
            if lbl not in fs:
                raise ValueError(f"output_labels contains {lbl!r} which is not a free label. Free labels are: {free}")
    out = "".join(l2c[l] for l in output_labels)
    return ",".join(subs) + "->" + out, tuple(first[l] for l in output_labels)


def _contract_symmetric(tensors, subscripts, output_indices=None, precision=None) -> SymmetricTensor:
    """Filtered block-sparse contraction (contractor.py:291-484) on the GPU."""
    lhs, out_subs = subscripts.split("->")
    in_subs = lhs.split(",")
    c2i = {}
    for t, s in zip(tensors, in_subs):
        for ch, idx in zip(s, t.indices):
            c2i[ch] = idx
    out_indices = tuple(c2i[c] for c in out_subs)
    # fermionic operands: the exchange sign of the leg reordering (contractor.py:460-470)
    plan = get_plan(tensors, in_subs, out_subs, _capi.MATCH_FILTERED, out_indices, _fermionic(tensors))
    data = plan.execute(tensors, precision or DEFAULT_PRECISION)
    out = SymmetricTensor.from_flat(out_indices, plan.out_keys, data)
    if plan.target is None:
        out._validate()
    return out


def blockwise_contract(tensors, subscripts, output_indices, precision=None) -> SymmetricTensor:
    """Unfiltered multi-operand contraction (algorithms/dmrg.py:1048-1151) on the GPU."""
    lhs, out_subs = subscripts.split("->")
    in_subs = lhs.split(",")
    plan = get_plan(tensors, in_subs, out_subs, _capi.MATCH_UNFILTERED, tuple(output_indices))
    data = plan.execute(tensors, precision or DEFAULT_PRECISION)
    return SymmetricTensor.from_flat(tuple(output_indices), plan.out_keys, data)


def transpose_symmetric(t: SymmetricTensor, axes) -> SymmetricTensor:
    """Leg permutation of every block (core/tensor.py:832-861); fermionic
    blocks take the Koszul sign of the permutation (core/tensor.py:32-50)."""
    chars = string.ascii_letters[: t.ndim]
    sub = chars + "->" + "".join(chars[a] for a in axes)
    new_idx = tuple(t.indices[a] for a in axes)
    lhs, out_subs = sub.split("->")
    plan = get_plan([t], [lhs], out_subs, _capi.MATCH_UNFILTERED, new_idx, _fermionic([t]))
    data = plan.execute([t], DEFAULT_PRECISION)
    return SymmetricTensor.from_flat(new_idx, plan.out_keys, data)


def contract_with_subscripts(tensors, subscripts, output_indices, optimize="auto", precision=None):
    """(contractor.py:534-569)"""
    if all(isinstance(t, SymmetricTensor) for t in tensors):
        return _contract_symmetric(list(tensors), subscripts, output_indices, precision)
    types = [type(t).__name__ for t in tensors]
    raise TypeError("Cannot mix DenseTensor and SymmetricTensor in a single contraction. "
                    f"Got types: {types}. Convert all tensors to the same type first."
                    if any(isinstance(t, SymmetricTensor) for t in tensors)
                    else f"tenax_b200 contracts SymmetricTensor operands only; got {types}")


def contract(*tensors, output_labels=None, optimize="auto", precision=None):
    """Contract tensors over shared labels (contractor.py:490-531)."""
    if not tensors:
        raise ValueError("contract() requires at least one tensor")
    subscripts, output_indices = _labels_to_subscripts(tensors, output_labels)
    if len(tensors) == 1:
        lhs, rhs = subscripts.split("->")
        if lhs == rhs:
            return tensors[0]
    return contract_with_subscripts(tensors, subscripts, output_indices, optimize, precision)


# ---------------------------------------------------------------------------
# differentiable block-sparse contraction
# ---------------------------------------------------------------------------

def _onto_keys(t: SymmetricTensor, keys) -> torch.Tensor:
    """Flat data of ``t`` laid out over ``keys``: blocks ``t`` has are copied,
    the others are zero, blocks of ``t`` outside ``keys`` are dropped."""
    from tenax_b200.tensor import embed_in_keys, restrict_to_keys

    keys = sorted(keys)
    common = sorted(set(t.keys) & set(keys))
    return embed_in_keys(restrict_to_keys(t, common), keys).data


class _SymContract(torch.autograd.Function):
    """C = A (x) B over shared subscripts on the block-sparse engine, with
    the adjoint written out: dA = dC (x) B and dB = A (x) dC, each another
    contraction of the same engine (unfiltered matching), laid out on the
    operand's own key set (blocks an operand does not store get no gradient:
    they are structurally zero)."""

    @staticmethod
    def forward(ctx, spec, a_data, b_data):
        a_idx, a_keys, b_idx, b_keys, subs, out_idx, filtered, precision = spec
        a = SymmetricTensor.from_flat(a_idx, a_keys, a_data)
        b = SymmetricTensor.from_flat(b_idx, b_keys, b_data)
        if filtered:
            out = _contract_symmetric([a, b], subs, out_idx, precision)
        else:
            out = blockwise_contract([a, b], subs, out_idx, precision)
        ctx.spec = spec
        ctx.out_keys = out.keys
        ctx.save_for_backward(a_data, b_data)
        return out.data

    @staticmethod
    def backward(ctx, g):
        a_idx, a_keys, b_idx, b_keys, subs, out_idx, _, precision = ctx.spec
        a_data, b_data = ctx.saved_tensors
        lhs, so = subs.split("->")
        sa, sb = lhs.split(",")
        gc = SymmetricTensor.from_flat(out_idx, ctx.out_keys, g.contiguous())
        ga = gb = None
        if ctx.needs_input_grad[1]:
            b = SymmetricTensor.from_flat(b_idx, b_keys, b_data)
            ga = _onto_keys(blockwise_contract([gc, b], f"{so},{sb}->{sa}", a_idx, precision), a_keys)
        if ctx.needs_input_grad[2]:
            a = SymmetricTensor.from_flat(a_idx, a_keys, a_data)
            gb = _onto_keys(blockwise_contract([a, gc], f"{sa},{so}->{sb}", b_idx, precision), b_keys)
        return None, ga, gb


def contract_ad(a: SymmetricTensor, b: SymmetricTensor, output_labels=None, precision=None) -> SymmetricTensor:
    """``contract(a, b)`` (contractor.py:490-531, filtered semantics) whose
    result's flat ``data`` carries autograd history: gradients flow to
    ``a.data`` / ``b.data`` through the hand-written block-sparse adjoint."""
    if _fermionic((a, b)):
        raise TnxUnsupportedAD("contract_ad: the adjoint of a fermionic contraction carries exchange signs "
                               "this engine does not apply to gradients")
    subscripts, out_idx = _labels_to_subscripts((a, b), output_labels)
    lhs, so = subscripts.split("->")
    sa, sb = lhs.split(",")
    for s, other in ((sa, sb + so), (sb, sa + so)):
        if any(c not in other for c in s):
            raise TnxUnsupportedAD(f"'{subscripts}': a leg summed within one operand has no adjoint here")
    spec = (a.indices, a.keys, b.indices, b.keys, subscripts, tuple(out_idx), True, precision)
    data = _SymContract.apply(spec, a.data, b.data)
    probe = get_plan([a, b], [sa, sb], so, _capi.MATCH_FILTERED, tuple(out_idx))
    return SymmetricTensor.from_flat(tuple(out_idx), probe.out_keys, data)


class TnxUnsupportedAD(NotImplementedError):
    """A contraction form whose adjoint is not a contraction of the same kind."""
