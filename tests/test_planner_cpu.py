"""Host-side checks of the C-ABI library: exports and exact integer planning.

No GPU needed: planning is host work inside ``libtenax_b200.so``.
"""

import ctypes as C
import json
import os
import re

import numpy as np
import pytest

from fixture_io import unpack_tensor
from oracle.blocksparse import blockwise_keys, contract_symmetric

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_library_exports_every_header_symbol():
    from tenax_b200 import _capi

    header = open(os.path.join(ROOT, "include", "tenax_b200.h")).read()
    declared = set(re.findall(r"\b(tnx_[a-z0-9_]+)\s*\(", header))
    assert declared, "no declarations found"
    for name in declared:
        assert hasattr(_capi.LIB, name), f"{name} declared but not exported"
    assert declared == set(_capi.EXPORTED)


def test_valid_blocks_matches_reference(golden_dir):
    from tenax_b200 import _capi

    for c in json.load(open(os.path.join(golden_dir, "valid_blocks.json"))):
        keys = _capi.valid_blocks(c["charges"], c["flows"], c["modulus"], c["target"])
        assert [list(k) for k in keys] == c["keys"], c["name"]


def _plan_from_otensors(ts, subscripts, mode, out_legs):
    from tenax_b200 import _capi

    lhs, out = subscripts.split("->")
    subs = lhs.split(",")
    hold = [_capi.DescHolder([l.charges for l in t.legs], [l.flow for l in t.legs], sorted(t.blocks), s)
            for t, s in zip(ts, subs)]
    descs = (_capi.TensorDesc * len(ts))(*[h.desc for h in hold])
    oh = _capi.DescHolder([l.charges for l in out_legs], [l.flow for l in out_legs], [], None)
    h = C.c_void_p()
    mod = ts[0].modulus or 0
    st = _capi.LIB.tnx_plan_create(descs, len(ts), out.encode(), mode, mod, oh.charges.ctypes.data,
                                   oh.leg_dims.ctypes.data, oh.flows.ctypes.data, C.byref(h))
    if st != 0:
        return None, st
    nb, tot, ht, tg = C.c_int64(), C.c_int64(), C.c_int32(), C.c_int64()
    _capi.check(_capi.LIB.tnx_plan_output(h, C.byref(nb), None, C.byref(tot), C.byref(ht), C.byref(tg)))
    nl = len(out)
    buf = np.zeros(max(1, nb.value * nl), np.int32)
    _capi.check(_capi.LIB.tnx_plan_output(h, C.byref(nb), buf.ctypes.data, None, None, None))
    flops = _capi.LIB.tnx_plan_flops(h)
    _capi.LIB.tnx_plan_destroy(h)
    keys = [tuple(int(q) for q in r) for r in buf[: nb.value * nl].reshape(-1, nl)] if nl else []
    return (keys, tot.value, ht.value, tg.value, flops), 0


def test_filtered_plan_keys_match_reference(golden_dir):
    from tenax_b200 import _capi

    z = np.load(os.path.join(golden_dir, "contract.npz"))
    for c in json.load(open(os.path.join(golden_dir, "contract.json"))):
        ins = [unpack_tensor(z, f"{c['name']}.in{i}") for i in range(c["n_in"])]
        ref = unpack_tensor(z, f"{c['name']}.out")
        res, st = _plan_from_otensors(ins, c["subscripts"], _capi.MATCH_FILTERED, ref.legs)
        assert st == 0, (c["name"], _capi.LIB.tnx_last_error())
        keys, total, *_ = res
        assert keys == sorted(ref.blocks), c["name"]
        assert total == sum(b.size for b in ref.blocks.values())


def test_unfiltered_plan_keys_match_blockwise(golden_dir):
    from tenax_b200 import _capi

    z = np.load(os.path.join(golden_dir, "dmrg_pieces.npz"))
    L, th, Wl, Wr, R = (unpack_tensor(z, f"heff.{n}") for n in ("L", "theta", "Wl", "Wr", "R"))
    subs = "abc,apqd,bpse,eqtf,dfg->cstg"
    res, st = _plan_from_otensors([L, th, Wl, Wr, R], subs, _capi.MATCH_UNFILTERED, th.legs)
    assert st == 0, _capi.LIB.tnx_last_error()
    assert res[0] == sorted(blockwise_keys([L, th, Wl, Wr, R], subs))
    assert res[0] == sorted(unpack_tensor(z, "heff.out").blocks)


def test_heff_plan_out_keys(golden_dir):
    from tenax_b200 import _capi

    z = np.load(os.path.join(golden_dir, "dmrg_pieces.npz"))
    L, th, Wl, Wr, R = (unpack_tensor(z, f"heff.{n}") for n in ("L", "theta", "Wl", "Wr", "R"))
    hold = [_capi.DescHolder([l.charges for l in t.legs], [l.flow for l in t.legs], sorted(t.blocks), None)
            for t in (L, th, Wl, Wr, R)]
    h = C.c_void_p()
    _capi.check(_capi.LIB.tnx_heff_create(*[C.byref(x.desc) for x in hold], C.byref(h)))
    n = C.c_int64()
    _capi.check(_capi.LIB.tnx_heff_out_keys(h, C.byref(n), None))
    buf = np.zeros(4 * n.value, np.int32)
    _capi.check(_capi.LIB.tnx_heff_out_keys(h, C.byref(n), buf.ctypes.data))
    keys = [tuple(r) for r in buf.reshape(-1, 4).tolist()]
    assert keys == sorted(unpack_tensor(z, "heff.out").blocks)
    # algorithmic flops: 4 pairwise stages
    assert _capi.LIB.tnx_heff_flops(h) > 0
    _capi.LIB.tnx_heff_destroy(h)


def test_errors_map_to_reference_exceptions():
    from tenax_b200 import _capi

    with pytest.raises(ValueError):
        _capi.check(_capi.TNX_ERR_VALUE)
    with pytest.raises(TypeError):
        _capi.check(_capi.TNX_ERR_TYPE)
    # label used three times -> ValueError from the planner
    d = _capi.DescHolder([[0, 1], [0, 1]], [1, -1], [(0, 0), (1, 1)], "aa")
    descs = (_capi.TensorDesc * 1)(d.desc)
    h = C.c_void_p()
    st = _capi.LIB.tnx_plan_create(descs, 1, b"", _capi.MATCH_UNFILTERED, 0, None, None, None, C.byref(h))
    assert st == _capi.TNX_ERR_UNSUPPORTED
