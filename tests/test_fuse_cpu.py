"""fuse_indices (algorithms/_tensor_utils.py:106-325): the oracle and the
library's planner tables against the reference's own outputs.

The fused leg's charges, the output key set and order, each block's
contents (pair-grouped in-sector layout) and todense() are compared
bit-exactly: fusion moves values without arithmetic.
"""

import json
import os

import numpy as np
import pytest

from fixture_io import unpack_tensor
from oracle.blocksparse import fuse_indices, todense


@pytest.fixture(scope="module")
def fuse_fix(golden_dir):
    return (np.load(os.path.join(golden_dir, "fuse.npz")),
            json.load(open(os.path.join(golden_dir, "fuse.json"))))


def test_oracle_fuse_matches_reference(fuse_fix):
    z, cases = fuse_fix
    for c in cases:
        t = unpack_tensor(z, f"{c['name']}.in")
        ref = unpack_tensor(z, f"{c['name']}.out")
        out = fuse_indices(t, c["axis_a"], c["axis_b"], "fused", c["fused_flow"])
        assert [list(k) for k in out.blocks] == c["out_key_order"], c["name"]
        for lo, lr in zip(out.legs, ref.legs):
            assert np.array_equal(lo.charges, lr.charges) and lo.flow == lr.flow, c["name"]
        assert sorted(out.blocks) == sorted(ref.blocks)
        for k in ref.blocks:
            assert np.array_equal(out.blocks[k], ref.blocks[k]), (c["name"], k)
        assert np.array_equal(todense(out), z[f"{c['name']}.out_dense"]), c["name"]


def test_library_planner_tables_match_reference(fuse_fix):
    """The C-ABI planner's fused charges, output keys and sizes (no GPU needed)."""
    import ctypes as C

    from tenax_b200 import _capi

    z, cases = fuse_fix
    for c in cases:
        t = unpack_tensor(z, f"{c['name']}.in")
        ref = unpack_tensor(z, f"{c['name']}.out")
        keys = t.sorted_keys()
        h = _capi.DescHolder([l.charges for l in t.legs], [l.flow for l in t.legs], keys, None)
        p = C.c_void_p()
        _capi.check(_capi.LIB.tnx_fuse_plan_create(C.byref(h.desc), c["modulus"] or 0, c["axis_a"], c["axis_b"],
                                                   c["fused_flow"], C.byref(p)))
        try:
            nf, nb, tot = C.c_int64(), C.c_int64(), C.c_int64()
            _capi.check(_capi.LIB.tnx_fuse_plan_output(p, None, C.byref(nf), C.byref(nb), None, C.byref(tot)))
            fc = np.zeros(nf.value, np.int32)
            ks = np.zeros(nb.value * (len(t.legs) - 1), np.int32)
            _capi.check(_capi.LIB.tnx_fuse_plan_output(p, fc.ctypes.data, None, None, ks.ctypes.data, None))
        finally:
            _capi.LIB.tnx_fuse_plan_destroy(p)
        a = min(c["axis_a"], c["axis_b"])
        assert np.array_equal(fc, ref.legs[a].charges), c["name"]
        assert [tuple(int(q) for q in r) for r in ks.reshape(nb.value, -1)] == ref.sorted_keys(), c["name"]
        assert tot.value == sum(b.size for b in ref.blocks.values()), c["name"]


def test_library_fuse_rejects_bad_axes():
    import ctypes as C

    from tenax_b200 import _capi

    h = _capi.DescHolder([np.array([0, 1], np.int32), np.array([0, 1], np.int32)], [1, -1], [(0, 0), (1, 1)], None)
    p = C.c_void_p()
    for a, b, f in ((0, 0, 1), (0, 2, 1), (0, 1, 2)):
        with pytest.raises(ValueError):
            _capi.check(_capi.LIB.tnx_fuse_plan_create(C.byref(h.desc), 0, a, b, f, C.byref(p)))


def test_oracle_fused_row_map_reproduces_todense(fuse_fix):
    """todense() of a fused tensor is the natural reshape with rows moved by
    fused_row_map (adjacent-axis cases: fused leg first or in the middle)."""
    from oracle.blocksparse import fused_row_map

    z, cases = fuse_fix
    for c in cases:
        a, b = sorted((c["axis_a"], c["axis_b"]))
        t = unpack_tensor(z, f"{c['name']}.in")
        dense = z[f"{c['name']}.in_dense"]
        perm = [i for i in range(dense.ndim) if i not in (a, b)]
        perm = perm[:a] + [a, b] + perm[a:]
        nat = np.transpose(dense, perm)
        shp = nat.shape
        nat = nat.reshape(shp[:a] + (shp[a] * shp[a + 1],) + shp[a + 2:])
        m = fused_row_map(t.legs[a], t.legs[b], c["fused_flow"], c["modulus"])
        moved = np.zeros_like(nat)
        idx = [slice(None)] * nat.ndim
        for n, p in enumerate(m):
            src = list(idx); src[a] = n
            dst = list(idx); dst[a] = p
            moved[tuple(dst)] = nat[tuple(src)]
        assert np.array_equal(moved, z[f"{c['name']}.out_dense"]), c["name"]
        assert sorted(m.tolist()) == list(range(len(m)))
