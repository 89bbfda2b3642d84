"""Dense tensor contractions on the block-sparse engine, with adjoints.

A dense tensor is a block-sparse tensor with one block: every leg carries
the trivial charge 0, so the planner sees a single sector and the contraction
becomes one permute-pack, one grouped tensor-core GEMM and one scatter in the
library -- the same kernels as the symmetric path.  ``einsum`` evaluates one
pairwise contraction (or a single-operand permutation) given as subscripts;
``Contract`` makes it differentiable: the adjoint of ``C = A *_{s} B`` is two
more contractions of the same engine, dA = C' *_{sC,sB} B and dB = A *_{sA,sC} C'.

Plans are cached per (subscripts, shapes); each owns its device buffers, and
calls that share a plan are ordered by the stream they run on.
"""

from __future__ import annotations

import ctypes as C
from collections import OrderedDict

import numpy as np
import torch

from tenax_b200 import _capi

_PLANS: "OrderedDict[tuple, _DensePlan]" = OrderedDict()
_PLAN_CACHE_SIZE = 256


class _DensePlan:
    """A ``tnx_plan`` over single-block operands with trivial charges."""

    def __init__(self, in_subs, out_subs, shapes, precision):
        self.holders = [
            _capi.DescHolder([np.zeros(n, np.int32) for n in shp], [1] * len(shp), [[0] * len(shp)], s)
            for s, shp in zip(in_subs, shapes)
        ]
        dims = {}
        for s, shp in zip(in_subs, shapes):
            for ch, n in zip(s, shp):
                if dims.setdefault(ch, n) != n:
                    raise ValueError(f"size mismatch for subscript '{ch}': {dims[ch]} vs {n}")
        self.out_shape = tuple(dims[c] for c in out_subs)
        out_h = _capi.DescHolder([np.zeros(n, np.int32) for n in self.out_shape], [1] * len(out_subs), [], None)
        descs = (_capi.TensorDesc * len(shapes))(*[h.desc for h in self.holders])
        h = C.c_void_p()
        _capi.check(_capi.LIB.tnx_plan_create(descs, len(shapes), out_subs.encode(), _capi.MATCH_UNFILTERED, 0,
                                              out_h.charges.ctypes.data, out_h.leg_dims.ctypes.data,
                                              out_h.flows.ctypes.data, C.byref(h)))
        self.handle = h
        self.precision = _capi.PRECISIONS[precision]
        self.flops = float(_capi.LIB.tnx_plan_flops(h))
        self.n_in = len(shapes)

    def __call__(self, *tensors):
        out = torch.empty(self.out_shape, dtype=torch.float64, device=tensors[0].device)
        if out.numel() == 0:
            return out
        ptrs = (C.c_void_p * self.n_in)(*[t.data_ptr() for t in tensors])
        _capi.check(_capi.LIB.tnx_plan_execute(self.handle, ptrs, out.data_ptr(), self.precision, None, 0,
                                               torch.cuda.current_stream(out.device).cuda_stream))
        return out

    def __del__(self):
        if getattr(self, "handle", None) and _capi is not None and _capi.LIB is not None:
            _capi.LIB.tnx_plan_destroy(self.handle)
            self.handle = None


def _plan(subscripts, shapes, precision) -> _DensePlan:
    key = (subscripts, shapes, precision)
    p = _PLANS.get(key)
    if p is not None:
        _PLANS.move_to_end(key)
        return p
    lhs, out = subscripts.split("->")
    p = _DensePlan(lhs.split(","), out, shapes, precision)
    _PLANS[key] = p
    if len(_PLANS) > _PLAN_CACHE_SIZE:
        _PLANS.popitem(last=False)
    return p


def _operand(t: torch.Tensor) -> torch.Tensor:
    if not t.is_cuda or t.dtype != torch.float64:
        raise TypeError("dense contractions take float64 CUDA tensors")
    return t.contiguous()


def einsum(subscripts: str, *tensors: torch.Tensor, precision: str = "fp64") -> torch.Tensor:
    """One pairwise contraction (or single-operand permutation) on the engine.

    ``subscripts`` is explicit (``"ab,bc->ac"``); repeated subscripts within
    one operand (traces) are not supported.  No autograd: see ``contract``.
    """
    ops = [_operand(t) for t in tensors]
    plan = _plan(subscripts, tuple(tuple(t.shape) for t in ops), precision)
    return plan(*ops)


def flops(subscripts: str, *shapes) -> float:
    """FLOPs the engine performs for ``einsum(subscripts, ...)`` on these shapes."""
    return _plan(subscripts, tuple(tuple(s) for s in shapes), "fp64").flops


class Contract(torch.autograd.Function):
    """Differentiable pairwise contraction: forward and adjoint on the engine."""

    @staticmethod
    def forward(ctx, subscripts, precision, a, b):
        ctx.subscripts = subscripts
        ctx.precision = precision
        ctx.save_for_backward(a, b)
        return einsum(subscripts, a, b, precision=precision)

    @staticmethod
    def backward(ctx, g):
        a, b = ctx.saved_tensors
        lhs, so = ctx.subscripts.split("->")
        sa, sb = lhs.split(",")
        p = ctx.precision
        ga = einsum(f"{so},{sb}->{sa}", g, b, precision=p) if ctx.needs_input_grad[2] else None
        gb = einsum(f"{sa},{so}->{sb}", a, g, precision=p) if ctx.needs_input_grad[3] else None
        return None, None, ga, gb


def contract(subscripts: str, a: torch.Tensor, b: torch.Tensor, precision: str = "fp64") -> torch.Tensor:
    """``einsum`` of two operands that records its adjoint for autograd.

    Every subscript of each operand must appear in the other operand or in
    the output (a pure contraction), which is what makes the adjoint two
    contractions of the same form.  The adjoint runs in the forward's
    precision."""
    lhs, so = subscripts.split("->")
    sa, sb = lhs.split(",")
    for s, other in ((sa, sb + so), (sb, sa + so)):
        missing = [c for c in s if c not in other]
        if missing:
            raise ValueError(f"'{subscripts}': subscripts {missing} are summed within one operand")
    return Contract.apply(subscripts, precision, a, b)
