"""The allocation-free contraction entry point, checked against the regular one.

``tnx_plan_execute_static`` serves callers that cannot allocate device
memory themselves (for example an XLA custom call inside a JAX process whose
memory pool already holds most of the GPU).  It must give the same result as
``tnx_plan_execute`` (FP64 sector GEMMs; tolerance rtol 1e-12) on two calls
in a row, because its scratch array is shared and keeps the previous call's
contents.  This file is collected last so that a failing run that stops at
the first failure has already run every other test; it also passes alone in a
fresh process (the first call sets up the scratch address on this device).
"""

import ctypes as C
import json
import os

import numpy as np
import pytest

from fixture_io import unpack_tensor

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a CUDA device", allow_module_level=True)

from tenax_b200 import _capi  # noqa: E402
from tenax_b200.contraction import get_plan  # noqa: E402
from tenax_b200.core import FlowDirection, TensorIndex, U1Symmetry, ZnSymmetry  # noqa: E402
from tenax_b200.tensor import SymmetricTensor  # noqa: E402


def _dev(t):
    sym = U1Symmetry() if t.modulus is None else ZnSymmetry(t.modulus)
    return SymmetricTensor(t.blocks, tuple(TensorIndex(sym, l.charges, FlowDirection(l.flow), l.label)
                                           for l in t.legs), _validate=False)


def _run_static(plan, tensors):
    out = torch.full((max(1, plan.total),), float("nan"), dtype=torch.float64, device="cuda")
    ptrs = (C.c_void_p * len(tensors))(*[t.data.data_ptr() for t in tensors])
    _capi.check(_capi.LIB.tnx_plan_execute_static(plan.handle, ptrs, out.data_ptr(),
                                                 torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    return out[: plan.total]


def _case(golden_dir, name):
    z = np.load(os.path.join(golden_dir, "contract.npz"))
    cases = {c["name"]: c for c in json.load(open(os.path.join(golden_dir, "contract.json")))}
    c = cases[name]
    ins = [_dev(unpack_tensor(z, f"{name}.in{i}")) for i in range(c["n_in"])]
    lhs, out_subs = c["subscripts"].split("->")
    c2i = {}
    for t, s in zip(ins, lhs.split(",")):
        for ch, idx in zip(s, t.indices):
            c2i[ch] = idx
    plan = get_plan(ins, lhs.split(","), out_subs, _capi.MATCH_FILTERED, tuple(c2i[ch] for ch in out_subs))
    return plan, ins


def test_static_matches_regular_two_calls(golden_dir):
    for name in ("mps_pair", "two_legs", "pair_u1_perm"):
        plan, ins = _case(golden_dir, name)
        ref = plan.execute(ins, "fp64")
        torch.cuda.synchronize()
        for _ in range(2):
            got = _run_static(plan, ins)
            torch.testing.assert_close(got, ref, rtol=1e-12, atol=1e-14)


def test_static_multi_operand_and_size_limit():
    from tenax_b200.contraction import blockwise_contract
    from tenax_b200.workloads import chain_bulk_w, make_heff_problem

    Wl, Wr = chain_bulk_w()
    p = make_heff_problem(40, 40, Wl, Wr, np.random.default_rng(9), n_sectors=6, hi=16)
    ts = [p.L, p.theta, p.Wl, p.Wr, p.R]
    subs = "abc,apqd,bpse,eqtf,dfg->cstg"
    ref = blockwise_contract(ts, subs, p.theta.indices).data
    plan = get_plan(ts, subs.split("->")[0].split(","), "cstg", _capi.MATCH_UNFILTERED, p.theta.indices)
    for _ in range(2):
        torch.testing.assert_close(_run_static(plan, ts), ref, rtol=1e-12, atol=1e-14)
    # a contraction whose scratch exceeds the static array is rejected, nothing runs
    big = make_heff_problem(1024, 1024, Wl, Wr, np.random.default_rng(1), n_sectors=8, hi=256)
    bts = [big.L, big.theta, big.Wl, big.Wr, big.R]
    bplan = get_plan(bts, subs.split("->")[0].split(","), "cstg", _capi.MATCH_UNFILTERED, big.theta.indices)
    out = torch.empty(max(1, bplan.total), dtype=torch.float64, device="cuda")
    ptrs = (C.c_void_p * 5)(*[t.data.data_ptr() for t in bts])
    st = _capi.LIB.tnx_plan_execute_static(bplan.handle, ptrs, out.data_ptr(), torch.cuda.current_stream().cuda_stream)
    assert st == _capi.TNX_ERR_VALUE
    assert b"static arena" in _capi.LIB.tnx_last_error()


def test_static_single_operand_transpose():
    """A one-operand plan (a leg permutation, contracted with the library's
    scalar 1.0): the caller passes a single input pointer, and the static
    path must read nothing beyond it.  Two calls in a row, against the
    regular entry point."""
    u1 = U1Symmetry()
    q = np.array([-2, -1, -1, 0, 0, 0, 1, 1, 2], np.int32)
    idx = (TensorIndex(u1, q, FlowDirection.IN, "a"), TensorIndex(u1, np.array([-1, 1], np.int32),
                                                                 FlowDirection.IN, "p"),
           TensorIndex(u1, q, FlowDirection.OUT, "b"))
    t = SymmetricTensor.random_normal(idx, key=5)
    out_idx = (idx[2], idx[0], idx[1])
    plan = get_plan([t], ["apb"], "bap", _capi.MATCH_FILTERED, out_idx)
    ref = plan.execute([t], "fp64")
    torch.cuda.synchronize()
    dense = t.todense().cpu().numpy().transpose(2, 0, 1)
    got_t = SymmetricTensor.from_flat(out_idx, plan.out_keys, ref)
    np.testing.assert_allclose(got_t.todense().cpu().numpy(), dense, rtol=0, atol=0)
    for _ in range(2):
        torch.testing.assert_close(_run_static(plan, [t]), ref, rtol=1e-12, atol=1e-14)
