"""Leg fusion of block-sparse tensors on the GPU.

Same function as tenax ``algorithms/_tensor_utils.py:106-325``
(``fuse_indices``).  The integer work -- the fused leg's charges, the pair
offsets inside each fused sector and the output block list -- is done by the
library's planner (``tnx_fuse_plan_*``) and matches the reference exactly;
the values are moved by one strided-copy launch into a zeroed output buffer.
Plans are cached by block structure.
"""

from __future__ import annotations

import ctypes as C
from collections import OrderedDict

import numpy as np
import torch

from tenax_b200 import _capi
from tenax_b200.core import FlowDirection, TensorIndex
from tenax_b200.tensor import SymmetricTensor

_PLANS: "OrderedDict[tuple, _FusePlan]" = OrderedDict()
_PLAN_CACHE_SIZE = 256


class _FusePlan:
    def __init__(self, t: SymmetricTensor, a: int, b: int, fused_flow: int):
        sym = t.indices[0].symmetry
        mod = sym.n_values()
        self.holder = _capi.DescHolder([i.charges for i in t.indices], [int(i.flow) for i in t.indices], t.keys, None)
        h = C.c_void_p()
        _capi.check(_capi.LIB.tnx_fuse_plan_create(C.byref(self.holder.desc), 0 if mod is None else int(mod), a, b,
                                                   int(fused_flow), C.byref(h)))
        self.handle = h
        nf, nb, tot = C.c_int64(), C.c_int64(), C.c_int64()
        _capi.check(_capi.LIB.tnx_fuse_plan_output(h, None, C.byref(nf), C.byref(nb), None, C.byref(tot)))
        self.fused_charges = np.zeros(max(1, nf.value), dtype=np.int32)
        nl = t.ndim - 1
        keys = np.zeros(max(1, nb.value * nl), dtype=np.int32)
        _capi.check(_capi.LIB.tnx_fuse_plan_output(h, self.fused_charges.ctypes.data, None, None, keys.ctypes.data,
                                                   None))
        self.fused_charges = self.fused_charges[: nf.value]
        self.out_keys = [tuple(int(q) for q in r) for r in keys[: nb.value * nl].reshape(-1, nl)]
        self.total = tot.value

    def __del__(self):
        if getattr(self, "handle", None) and _capi is not None and _capi.LIB is not None:
            _capi.LIB.tnx_fuse_plan_destroy(self.handle)
            self.handle = None


def _plan(t: SymmetricTensor, a: int, b: int, fused_flow: int) -> _FusePlan:
    key = (a, b, int(fused_flow), tuple((int(i.flow), i.charges.tobytes()) for i in t.indices), tuple(t.keys),
           t.indices[0].symmetry.n_values())
    p = _PLANS.get(key)
    if p is None:
        p = _FusePlan(t, a, b, fused_flow)
        _PLANS[key] = p
        if len(_PLANS) > _PLAN_CACHE_SIZE:
            _PLANS.popitem(last=False)
    else:
        _PLANS.move_to_end(key)
    return p


def fuse_indices(tensor: SymmetricTensor, axis_a: int, axis_b: int, fused_label, fused_flow) -> SymmetricTensor:
    """Fuse two legs into one at ``min(axis_a, axis_b)`` (_tensor_utils.py:106-134).

    The fused leg has dimension ``d_a * d_b``; its position ``i*d_b + j`` has
    charge ``fused_flow * (flow_a q_a[i] + flow_b q_b[j])`` (mod n).  Inside
    each fused sector the (q_a, q_b) pairs are stacked in sorted order, so a
    fused sector's rows are grouped by pair, not by position; ``todense()``
    of the result places them at the sector's positions in order, exactly as
    the reference does."""
    if not isinstance(tensor, SymmetricTensor):
        raise TypeError(f"fuse_indices takes a SymmetricTensor, got {type(tensor).__name__}")
    nd = tensor.ndim
    if nd < 2:
        raise ValueError("fuse_indices needs a tensor with at least two legs")
    a_in, b_in = int(axis_a) % nd if axis_a < 0 else int(axis_a), int(axis_b) % nd if axis_b < 0 else int(axis_b)
    flow = int(fused_flow.value if isinstance(fused_flow, FlowDirection) else fused_flow)
    plan = _plan(tensor, a_in, b_in, flow)
    a, b = sorted((a_in, b_in))
    sym = tensor.indices[a].symmetry
    fused_idx = TensorIndex(sym, plan.fused_charges.copy(), FlowDirection(flow), fused_label)
    others = [tensor.indices[i] for i in range(nd) if i not in (a, b)]
    new_indices = tuple(others[:a]) + (fused_idx,) + tuple(others[a:])
    out = torch.empty(max(1, plan.total), dtype=torch.float64, device=tensor.data.device)
    if plan.total:
        _capi.check(_capi.LIB.tnx_fuse_execute(plan.handle, tensor.data.data_ptr(), out.data_ptr(),
                                               torch.cuda.current_stream(out.device).cuda_stream))
    return SymmetricTensor.from_flat(new_indices, plan.out_keys, out[: plan.total])


def fused_charges(tensor: SymmetricTensor, axis_a: int, axis_b: int, fused_flow) -> np.ndarray:
    """The fused leg's charges alone (_tensor_utils.py:168-203), from the planner."""
    flow = int(fused_flow.value if isinstance(fused_flow, FlowDirection) else fused_flow)
    return _plan(tensor, int(axis_a), int(axis_b), flow).fused_charges.copy()
