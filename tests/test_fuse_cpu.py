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
