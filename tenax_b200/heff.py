"""Two-site effective-Hamiltonian matvec on the GPU.

``Y[c,s,t,g] = L[a,b,c] th[a,p,q,d] W_l[b,p,s,e] W_r[e,q,t,f] R[d,f,g]``
(tenax algorithms/dmrg.py:1282-1289, evaluated there by
``_blockwise_contract`` one block combination at a time).  Here it runs as
three stages over all sectors at once:

1. ``X1 = L . th`` over a -- grouped sector GEMM (DMMA FP64 or tcgen05),
2. ``X3 = (W_l W_r) . X1`` over (b,p,q) -- fused sparse MPO kernel that
   writes the stage-3 operand images directly,
3. ``Y = X3 . R`` over (f,d) -- grouped sector GEMM whose epilogue writes
   the theta block layout.

Operator images (L, R, W_l W_r terms) are packed once per site; a matvec
only packs theta.  Many independent problems share each launch
(``HeffBatch``).
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from tenax_b200 import _capi
from tenax_b200.tensor import SymmetricTensor


def _desc(t_indices, keys):
    return _capi.DescHolder([i.charges for i in t_indices], [int(i.flow) for i in t_indices], keys, None)


def _create(L, th_indices, th_keys, Wl, Wr, R, precision: str = "fp64"):
    hold = [_desc(L.indices, L.keys), _desc(th_indices, th_keys), _desc(Wl.indices, Wl.keys),
            _desc(Wr.indices, Wr.keys), _desc(R.indices, R.keys)]
    h = C.c_void_p()
    _capi.check(_capi.LIB.tnx_heff_create_for(*[C.byref(x.desc) for x in hold], _capi.PRECISIONS[precision],
                                              C.byref(h)))
    return h, hold


def _out_keys(h):
    n = C.c_int64()
    _capi.check(_capi.LIB.tnx_heff_out_keys(h, C.byref(n), None))
    buf = np.zeros(max(1, 4 * n.value), dtype=np.int32)
    _capi.check(_capi.LIB.tnx_heff_out_keys(h, C.byref(n), buf.ctypes.data))
    return [tuple(int(q) for q in r) for r in buf[: 4 * n.value].reshape(-1, 4)]


def problem_flops(p) -> float:
    """Algorithmic FLOPs of one H_eff application on a problem's own theta
    key set (host planning only; no operator images are built)."""
    h, _hold = _create(p.L, p.theta.indices, p.theta.keys, p.Wl, p.Wr, p.R)
    try:
        return float(_capi.LIB.tnx_heff_flops(h))
    finally:
        _capi.LIB.tnx_heff_destroy(h)


def heff_key_closure(L, th_indices, th_keys, Wl, Wr, R, max_iter: int = 64):
    """Key sets K_0 = theta's keys, K_{k+1} = K_k | out(K_k), up to the fixed point.

    The reference's Lanczos grows the key set of its Krylov vectors exactly
    this way (key-union addition, core/tensor.py:933-952, of matvec outputs
    whose keys are never filtered, dmrg.py:1097).
    """
    seq, h, _hold = _closure(L, th_indices, th_keys, Wl, Wr, R, "fp64", max_iter)
    _capi.LIB.tnx_heff_destroy(h)
    return seq


def _closure(L, th_indices, th_keys, Wl, Wr, R, precision, max_iter: int = 64):
    """heff_key_closure, also returning the plan of the fixed point (created
    for ``precision``) and the descriptors it points into."""
    seq = [sorted(th_keys)]
    for _ in range(max_iter):
        h, hold = _create(L, th_indices, seq[-1], Wl, Wr, R, precision)
        out = _out_keys(h)
        nxt = sorted(set(seq[-1]) | set(out))
        if nxt == seq[-1]:
            return seq, h, hold
        _capi.LIB.tnx_heff_destroy(h)
        seq.append(nxt)
    raise RuntimeError("H_eff key closure did not converge")


HEFF_SUBSCRIPTS = "abc,apqd,bpse,eqtf,dfg->cstg"  # algorithms/dmrg.py:1282-1289


class HeffOperator:
    """H_eff of one two-site problem; theta/outputs live on a closed key set.

    The fused path (three or four launches per apply, batchable) needs every
    stage-4 group to write a single output charge, which the sector
    structures of U(1) MPS/MPO problems satisfy.  With a mixed precision,
    ``schedule={"fuse_mpo": 1}`` runs stages 1-3 as one kernel that applies
    W_l W_r straight from tensor memory (``c_per_tile`` sets the fused
    tile's c extent), ``{"fuse_mpo": 2}`` (routed) a stage-1 GEMM whose
    epilogue writes every single-term W_l W_r output straight into the
    stage-4 operand and keeps X1 only for the multi-term outputs, which the
    MPO kernel forms, ``{"fuse_mpo": 0}`` the stage-1 GEMM, all of X1 in HBM
    and the MPO kernel; with no schedule given, routed from 5e9 stage FLOPs
    (``self.flops``) on and unfused below.  ``self.schedule`` reports the
    schedule in effect.  Other structures (``fused`` False) apply
    H_eff through the general unfiltered contraction engine, the
    reference's ``_blockwise_contract`` semantics, one pairwise chain per
    apply: the same result, without the fused kernels."""

    def __init__(self, L: SymmetricTensor, Wl: SymmetricTensor, Wr: SymmetricTensor, R: SymmetricTensor,
                 theta_indices, theta_keys, precision: str = "fp64", schedule: dict | None = None):
        self.theta_indices = tuple(theta_indices)
        # the closure's last plan is the operator's plan (created for its precision)
        self.key_seq, self.handle, self._hold = _closure(L, theta_indices, theta_keys, Wl, Wr, R, precision)
        self.keys = self.key_seq[-1]
        closed = C.c_int32()
        _capi.check(_capi.LIB.tnx_heff_closed(self.handle, C.byref(closed)))
        self.fused = bool(closed.value)
        self.precision = precision
        self.flops = float(_capi.LIB.tnx_heff_flops(self.handle))
        self.schedule = {"fuse_mpo": 0, "c_per_tile": 0}
        if self.fused:
            if schedule is not None:
                req = _capi.HeffSchedule(int(schedule.get("fuse_mpo", 1)), int(schedule.get("c_per_tile", 0)))
                _capi.check(_capi.LIB.tnx_heff_set_schedule(self.handle, C.byref(req)))
            _capi.check(_capi.LIB.tnx_heff_set_operators(self.handle, L.data.data_ptr(), Wl.data.data_ptr(),
                                                         Wr.data.data_ptr(), R.data.data_ptr(),
                                                         _capi.PRECISIONS[precision],
                                                         torch.cuda.current_stream().cuda_stream))
            got = _capi.HeffSchedule()
            _capi.check(_capi.LIB.tnx_heff_get_schedule(self.handle, C.byref(got)))
            self.schedule = {"fuse_mpo": int(got.fuse_mpo), "c_per_tile": int(got.c_per_tile)}
        else:
            self._operands = (L, Wl, Wr, R)
        sizes = [int(np.prod([int(np.count_nonzero(i.charges == q)) for i, q in zip(self.theta_indices, k)]))
                 for k in self.keys]
        self.size = int(sum(sizes))
        self._batch = None

    def out_like(self) -> torch.Tensor:
        return torch.empty(self.size, dtype=torch.float64, device=torch.device("cuda", torch.cuda.current_device()))

    def apply(self, x: torch.Tensor, out: torch.Tensor | None = None) -> torch.Tensor:
        if out is None:
            out = self.out_like()
        if not self.fused:
            from tenax_b200.contraction import blockwise_contract
            from tenax_b200.tensor import embed_in_keys

            L, Wl, Wr, R = self._operands
            th = SymmetricTensor.from_flat(self.theta_indices, self.keys, x)
            y = blockwise_contract([L, th, Wl, Wr, R], HEFF_SUBSCRIPTS, self.theta_indices,
                                   None if self.precision == "fp64" else self.precision)
            out.copy_(embed_in_keys(y, self.keys).data)
            return out
        if self._batch is None:
            self._batch = HeffBatch([self])
        self._batch.apply([x], [out])
        return out

    def device_error(self) -> int:
        """The fused kernels' device-side timeout flag (0 on the general path)."""
        return self._batch.device_error() if self._batch is not None else 0

    def release_scratch(self) -> None:
        """Free the device buffers ``apply`` keeps between calls (its one-operator
        batch: images and intermediates); the next ``apply`` rebuilds them."""
        self._batch = None

    def __del__(self):
        if getattr(self, "handle", None) is not None and _capi.LIB is not None:
            self._batch = None
            _capi.LIB.tnx_heff_destroy(self.handle)
            self.handle = None


class HeffBatch:
    """Independent H_eff problems applied together: one launch per stage.

    Operators on the routed and the unfused schedule share a batch (one
    stage-1 launch holds both kinds of groups, the MPO tables are per
    problem); operators on the fused schedule cannot be mixed with the
    others (ValueError)."""

    def __init__(self, ops, skip_flag: torch.Tensor | None = None):
        self.ops = list(ops)
        if not all(o.fused for o in self.ops):
            raise _capi.TnxUnsupported("HeffBatch needs the fused H_eff path: an operator's sector structure "
                                       "has a stage-4 group writing several output charges")
        prec = {o.precision for o in self.ops}
        if len(prec) != 1:
            raise ValueError("all problems of a batch must use one precision")
        self.precision = prec.pop()
        arr = (C.c_void_p * len(self.ops))(*[o.handle for o in self.ops])
        h = C.c_void_p()
        _capi.check(_capi.LIB.tnx_heff_batch_create(arr, len(self.ops), _capi.PRECISIONS[self.precision],
                                                    C.byref(h)))
        self.handle = h
        self.skip_flag = skip_flag
        if skip_flag is not None:
            _capi.check(_capi.LIB.tnx_heff_batch_set_skip_flag(h, skip_flag.data_ptr()))
        n = C.c_int32()
        _capi.check(_capi.LIB.tnx_heff_batch_launches(h, C.byref(n)))
        self.launches_per_apply = n.value
        self.flops = sum(o.flops for o in self.ops)
        tot = C.c_int64()
        offs = np.zeros(len(self.ops), dtype=np.int64)
        _capi.check(_capi.LIB.tnx_heff_batch_size(h, C.byref(tot), offs.ctypes.data))
        self.total = tot.value  # elements of the concatenated theta buffer (problems in batch order)
        self.offsets = offs

    def apply(self, thetas, outs):
        tp = (C.c_void_p * len(thetas))(*[t.data_ptr() for t in thetas])
        op = (C.c_void_p * len(outs))(*[o.data_ptr() for o in outs])
        _capi.check(_capi.LIB.tnx_heff_batch_apply(self.handle, tp, op, torch.cuda.current_stream().cuda_stream))

    def route_stats(self) -> tuple:
        """(route records, largest window of records one epilogue warp scans
        for one 32-column chunk of a tile) of the routed stage-1 launch; (0, 0)
        when no operator is routed."""
        n, w = C.c_int64(), C.c_int32()
        _capi.check(_capi.LIB.tnx_heff_batch_route_stats(self.handle, C.byref(n), C.byref(w)))
        return n.value, w.value

    def capture(self, thetas, outs) -> "torch.cuda.CUDAGraph":
        """A CUDA graph of one apply with these buffers: the batch's pointer
        tables are bound by an eager apply first, so the captured apply
        issues kernels only.  ``graph.replay()`` then runs the whole batched
        matvec (every stage, every problem) as one launch on the current
        stream."""
        side = torch.cuda.Stream()
        side.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(side):
            self.apply(thetas, outs)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=side):
            self.apply(thetas, outs)
        torch.cuda.current_stream().wait_stream(side)
        return g

    def apply_host(self, host_inputs, host_outputs):
        """Stream independent applications from host memory: host_inputs[s]
        and host_outputs[s] are CPU float64 tensors of ``total`` elements
        (every problem's theta concatenated in batch order, at ``offsets``).
        Step s+1's copy in and step s-1's copy out overlap step s's compute;
        pinned buffers make the copies asynchronous.  Work is queued on the
        current stream and complete when it is."""
        if len(host_inputs) != len(host_outputs):
            raise ValueError("host_inputs and host_outputs must have the same length")
        for t in list(host_inputs) + list(host_outputs):
            if t.device.type != "cpu" or t.dtype != torch.float64 or not t.is_contiguous() or t.numel() != self.total:
                raise ValueError(f"host buffers must be contiguous CPU float64 tensors of {self.total} elements")
        n = len(host_inputs)
        ip = (C.c_void_p * max(1, n))(*[t.data_ptr() for t in host_inputs])
        op = (C.c_void_p * max(1, n))(*[t.data_ptr() for t in host_outputs])
        _capi.check(_capi.LIB.tnx_heff_batch_apply_host(self.handle, ip, op, n,
                                                        torch.cuda.current_stream().cuda_stream))

    def device_error(self) -> int:
        e = C.c_int32()
        _capi.check(_capi.LIB.tnx_heff_batch_error(self.handle, C.byref(e)))
        return e.value

    def __del__(self):
        if getattr(self, "handle", None) is not None and _capi.LIB is not None:
            _capi.LIB.tnx_heff_batch_destroy(self.handle)
            self.handle = None
