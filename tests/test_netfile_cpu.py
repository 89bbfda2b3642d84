"""Network-file parsing (tenax_b200.netfile) against the reference's own
results (tests/golden/netfile.json from network/netfile.py): topology,
pairwise ORDER steps, precomputed subscripts and error messages."""

import json
import os

import pytest

from tenax_b200 import netfile as nf


@pytest.fixture(scope="module")
def cases(golden_dir):
    with open(os.path.join(golden_dir, "netfile.json")) as fh:
        return json.load(fh)["parse"]


def test_parse_matches_reference(cases):
    for name, c in cases.items():
        if "error" in c:
            with pytest.raises(ValueError) as ei:
                nf.NetworkBlueprint(c["source"])
            assert str(ei.value) == c["error"], name
            continue
        spec = nf.parse_netfile(c["source"])
        assert spec["tensors"] == c["tensors"], name
        assert spec["tout"] == c["tout"], name
        assert spec["order"] == c["order"], name
        steps = nf._order_steps(spec["order"], set(spec["tensors"])) if spec["order"] is not None else None
        assert (steps if steps is None else [list(s) for s in steps]) == c["steps"], name
        bp = nf.from_netfile(c["source"])
        assert bp.subscripts == c["subscripts"], name
        assert bp.tensor_names == c["tensor_names"], name
        assert bp.output_labels == c["output_labels"], name


def test_sources_from_lines_and_files(tmp_path, cases):
    src = cases["chain3_order"]["source"]
    p = tmp_path / "net.net"
    p.write_text(src)
    for s in (src.splitlines(), p, str(p)):
        assert nf.NetworkBlueprint(s).subscripts == cases["chain3_order"]["subscripts"]


def test_launch_needs_every_slot(cases):
    bp = nf.NetworkBlueprint(cases["pair"]["source"])
    assert not bp.is_ready()
    with pytest.raises(RuntimeError, match="missing tensors"):
        bp.launch()
    with pytest.raises(KeyError):
        bp.put_tensor("Z", None)


def test_launch_block_structure_matches_reference(golden_dir):
    """The planner's output blocks for each einsum-path launch (no GPU
    needed for planning) equal the reference's, including the scalar of a
    closed ring and the empty result of a 3-chain without ORDER."""
    import ctypes as C

    import numpy as np

    from tenax_b200 import _capi
    from tests.golden.fixture_io import unpack_tensor

    z = np.load(os.path.join(golden_dir, "netfile.npz"))
    meta = json.load(open(os.path.join(golden_dir, "netfile.json")))
    ins = {n: unpack_tensor(z, f"in.{n}") for n in ("A", "B", "C", "Bring")}
    slots = {"pair": ("A", "B"), "chain3": ("A", "B", "C"), "ring_scalar": ("A", "Bring")}
    for name, use in slots.items():
        bp = nf.NetworkBlueprint(meta["parse"][name]["source"])
        lhs, out = bp.subscripts.split("->")
        ts = [ins[u] for u in use]
        hold = [_capi.DescHolder([l.charges for l in t.legs], [l.flow for l in t.legs], sorted(t.blocks), s)
                for t, s in zip(ts, lhs.split(","))]
        descs = (_capi.TensorDesc * len(ts))(*[h.desc for h in hold])
        ref = unpack_tensor(z, f"out.{name}")
        oh = _capi.DescHolder([l.charges for l in ref.legs], [l.flow for l in ref.legs], [], None)
        h = C.c_void_p()
        _capi.check(_capi.LIB.tnx_plan_create(descs, len(ts), out.encode(), _capi.MATCH_FILTERED, 0,
                                              oh.charges.ctypes.data, oh.leg_dims.ctypes.data, oh.flows.ctypes.data,
                                              C.byref(h)))
        nb, tot, ht, tg = C.c_int64(), C.c_int64(), C.c_int32(), C.c_int64()
        _capi.check(_capi.LIB.tnx_plan_output(h, C.byref(nb), None, C.byref(tot), C.byref(ht), C.byref(tg)))
        nl = len(out)
        buf = np.zeros(max(1, nb.value * max(nl, 1)), np.int32)
        _capi.check(_capi.LIB.tnx_plan_output(h, C.byref(nb), buf.ctypes.data, None, None, None))
        _capi.LIB.tnx_plan_destroy(h)
        keys = [tuple(int(q) for q in r) for r in buf[: nb.value * nl].reshape(-1, nl)] if nl else [()] * nb.value
        assert keys == sorted(ref.blocks), name
        assert tot.value == sum(b.size for b in ref.blocks.values()), name
