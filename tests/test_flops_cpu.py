"""The oracle's H_eff FLOP count (used by the CPU timing arm, which must not
load the device library) equals the planner's count on the benchmark's
structures: the width-6 cylinder MPO, 30 U(1) sectors per bond, each chi of
the batch.  Host planning only; no GPU."""

import ctypes as C
import importlib.util
import os

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench_flops_test", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


@pytest.mark.parametrize("chi", [256, 512, 1024, 2048])
def test_oracle_flops_equal_planner(chi):
    from tenax_b200 import _capi

    b = _bench()
    hp = b.HostProblems(3)
    args, f_oracle = hp.make(chi)
    hold = [_capi.DescHolder([l.charges for l in t.legs], [l.flow for l in t.legs], sorted(t.blocks), None)
            for t in args]
    h = C.c_void_p()
    _capi.check(_capi.LIB.tnx_heff_create(*[C.byref(x.desc) for x in hold], C.byref(h)))
    f_plan = _capi.LIB.tnx_heff_flops(h)
    _capi.LIB.tnx_heff_destroy(h)
    assert f_oracle == f_plan
    assert f_oracle > 0


@pytest.mark.parametrize("chi", [256, 512, 1024, 2048])
def test_benchmark_structures_plan_fused(chi):
    """Host planning of the fused stages 1-3 on the benchmark's structures:
    asked for, every split-BF16x3 and TF32 operator gets the fused kernel
    (cylinder MPO: at most 36 input slots per sector pair), FP64 never does,
    and out-of-range tile extents are rejected."""
    from tenax_b200 import _capi

    b = _bench()
    args, _ = b.HostProblems(3).make(chi, fill=False)
    hold = [_capi.DescHolder([l.charges for l in t.legs], [l.flow for l in t.legs], sorted(t.blocks), None)
            for t in args]
    for prec, want in (("bf16x3", 1), ("tf32", 1), ("fp64", 0)):
        h = C.c_void_p()
        _capi.check(_capi.LIB.tnx_heff_create_for(*[C.byref(x.desc) for x in hold], _capi.PRECISIONS[prec],
                                                  C.byref(h)))
        # no schedule given: routed for the mixed precisions from 5e9 stage FLOPs on
        s = _capi.HeffSchedule()
        _capi.check(_capi.LIB.tnx_heff_get_schedule(h, C.byref(s)))
        big = _capi.LIB.tnx_heff_flops(h) >= 5e9
        assert s.fuse_mpo == (2 if want and big else 0), (chi, prec)
        assert big == (chi >= 1024), chi
        on = _capi.HeffSchedule(1, 0)
        _capi.check(_capi.LIB.tnx_heff_set_schedule(h, C.byref(on)))
        _capi.check(_capi.LIB.tnx_heff_get_schedule(h, C.byref(s)))
        assert s.fuse_mpo == want, (chi, prec)
        assert (s.c_per_tile >= 1) == bool(want)
        routed = _capi.HeffSchedule(2, 0)
        _capi.check(_capi.LIB.tnx_heff_set_schedule(h, C.byref(routed)))
        _capi.check(_capi.LIB.tnx_heff_get_schedule(h, C.byref(s)))
        assert s.fuse_mpo == 2 * want and s.c_per_tile == 0
        off = _capi.HeffSchedule(0, 0)
        _capi.check(_capi.LIB.tnx_heff_set_schedule(h, C.byref(off)))
        _capi.check(_capi.LIB.tnx_heff_get_schedule(h, C.byref(s)))
        assert s.fuse_mpo == 0
        bad = _capi.HeffSchedule(1, 99)
        assert _capi.LIB.tnx_heff_set_schedule(h, C.byref(bad)) == _capi.TNX_ERR_VALUE
        bad = _capi.HeffSchedule(3, 0)
        assert _capi.LIB.tnx_heff_set_schedule(h, C.byref(bad)) == _capi.TNX_ERR_VALUE
        _capi.LIB.tnx_heff_destroy(h)
