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
