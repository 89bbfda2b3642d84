"""Device-side sector planning against the host planner and the reference's
pinned outputs, bit for bit:
  * valid block keys in the reference's order (_compute_valid_blocks,
    core/tensor.py:53-165): every golden case (U(1), Z2, Z3, with and without
    a target) and the benchmark's theta, L and R structures at every chi;
  * the output structure of two-operand filtered contractions
    (_contract_symmetric, contractor.py:344-441): sorted output keys and block
    offsets equal the host plan's, and the matched pairs equal a direct count
    of the reference's signature matching, on the golden contraction cases
    and the benchmark's L . theta stage;
  * fused-leg charges (_compute_fused_charges, _tensor_utils.py:191-203)
    equal the oracle's on the golden fuse cases.
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

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _stream():
    return torch.cuda.current_stream().cuda_stream


def _dev_i32(a):
    return torch.from_numpy(np.ascontiguousarray(np.asarray(a, dtype=np.int32))).cuda()


def _valid_dev(charges, flows, modulus, target):
    dims = np.array([len(c) for c in charges], np.int64)
    ch = _dev_i32(np.concatenate([np.asarray(c, np.int32) for c in charges]) if charges else np.zeros(1, np.int32))
    fl = np.asarray(flows, np.int32)
    n = C.c_int64()
    args = (len(charges), ch.data_ptr(), dims.ctypes.data, fl.ctypes.data, int(modulus or 0),
            int(target is not None), int(target or 0), C.byref(n))
    _capi.check(_capi.LIB.tnx_valid_blocks_dev(*args, None, 0, _stream()))
    out = torch.empty(max(1, n.value * len(charges)), dtype=torch.int32, device="cuda")
    _capi.check(_capi.LIB.tnx_valid_blocks_dev(*args, out.data_ptr(), out.numel(), _stream()))
    return [tuple(int(x) for x in r) for r in out[: n.value * len(charges)].cpu().numpy().reshape(-1, len(charges))]


def test_valid_blocks_golden(golden_dir):
    cases = json.load(open(os.path.join(golden_dir, "valid_blocks.json")))
    for c in cases:
        charges = [np.asarray(x, np.int32) for x in c["charges"]]
        got = _valid_dev(charges, c["flows"], c["modulus"], c["target"])
        assert [list(k) for k in got] == c["keys"], c["name"]
        host = _capi.valid_blocks(charges, c["flows"], c["modulus"], c["target"])
        assert got == [tuple(k) for k in host], c["name"]


def _bench_mod():
    import importlib.util

    spec = importlib.util.spec_from_file_location("bench_pd", os.path.join(ROOT, "bench.py"))
    b = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(b)
    return b


@pytest.mark.parametrize("chi", [256, 512, 1024, 2048])
def test_valid_blocks_benchmark_structures(chi):
    args, _ = _bench_mod().HostProblems(2).make(chi, fill=False)
    for name, t in (("L", args[0]), ("theta", args[1]), ("R", args[4])):
        ch = [l.charges for l in t.legs]
        fl = [l.flow for l in t.legs]
        got = _valid_dev(ch, fl, None, None)
        host = [tuple(k) for k in _capi.valid_blocks(ch, fl, None, None)]
        assert got == host, name
        # theta conserves charge; the environments carry the MPO's charge
        # transfer, so only theta's blocks are a subset of the target-0 keys
        if name == "theta":
            assert set(t.blocks) <= set(got)


def _structure_dev(a, b, subs_a, subs_b, out_subs, modulus):
    """(sorted out keys, offsets, pairs) from the device planner."""
    keep = []

    def desc(t, subs):
        charges = _dev_i32(np.concatenate([l.charges for l in t.legs]))
        keys = _dev_i32(np.array(sorted(t.blocks), np.int32).reshape(-1, len(t.legs)) if t.blocks
                        else np.zeros((1, len(t.legs)), np.int32))
        dims = np.array([len(l.charges) for l in t.legs], np.int64)
        flows = np.array([l.flow for l in t.legs], np.int32)
        sb = subs.encode()
        keep.extend([charges, keys, dims, flows, sb])
        return _capi.TensorDesc(len(t.legs), sb, flows.ctypes.data_as(C.POINTER(C.c_int32)),
                                C.cast(charges.data_ptr(), C.POINTER(C.c_int32)),
                                dims.ctypes.data_as(C.POINTER(C.c_int64)), len(t.blocks),
                                C.cast(keys.data_ptr(), C.POINTER(C.c_int32)))

    da, db = desc(a, subs_a), desc(b, subs_b)
    no, npairs = C.c_int64(), C.c_int64()
    _capi.check(_capi.LIB.tnx_contract_structure_dev(C.byref(da), C.byref(db), out_subs.encode(), int(modulus or 0),
                                                     C.byref(no), None, None, 0, C.byref(npairs), None, 0, _stream()))
    lo = max(1, len(out_subs))
    keys = torch.empty(max(1, no.value * lo), dtype=torch.int32, device="cuda")
    offs = torch.empty(no.value + 1, dtype=torch.int64, device="cuda")
    pairs = torch.empty(max(1, 3 * npairs.value), dtype=torch.int32, device="cuda")
    _capi.check(_capi.LIB.tnx_contract_structure_dev(C.byref(da), C.byref(db), out_subs.encode(), int(modulus or 0),
                                                     C.byref(no), keys.data_ptr(), offs.data_ptr(), no.value,
                                                     C.byref(npairs), pairs.data_ptr(), npairs.value, _stream()))
    k = keys[: no.value * len(out_subs)].cpu().numpy().reshape(no.value, len(out_subs))
    return ([tuple(int(x) for x in r) for r in k], offs.cpu().numpy().tolist(),
            pairs[: 3 * npairs.value].cpu().numpy().reshape(-1, 3).tolist())


def _host_plan(a, b, subs_a, subs_b, out_subs, modulus):
    """Sorted output keys and block offsets of the host plan."""
    holders = [_capi.DescHolder([l.charges for l in t.legs], [l.flow for l in t.legs], sorted(t.blocks), s)
               for t, s in ((a, subs_a), (b, subs_b))]
    descs = (_capi.TensorDesc * 2)(*[h.desc for h in holders])
    src = {}
    for t, s in ((a, subs_a), (b, subs_b)):
        for ch, leg in zip(s, t.legs):
            src.setdefault(ch, leg)
    out_legs = [src[c] for c in out_subs]
    oh = _capi.DescHolder([l.charges for l in out_legs], [l.flow for l in out_legs], [], None)
    h = C.c_void_p()
    _capi.check(_capi.LIB.tnx_plan_create(descs, 2, out_subs.encode(), _capi.MATCH_FILTERED, int(modulus or 0),
                                          oh.charges.ctypes.data, oh.leg_dims.ctypes.data, oh.flows.ctypes.data,
                                          C.byref(h)))
    nb, tot = C.c_int64(), C.c_int64()
    _capi.check(_capi.LIB.tnx_plan_output(h, C.byref(nb), None, C.byref(tot), None, None))
    lo = len(out_subs)
    buf = np.zeros(max(1, nb.value * lo), np.int32)
    _capi.check(_capi.LIB.tnx_plan_output(h, C.byref(nb), buf.ctypes.data, None, None, None))
    _capi.LIB.tnx_plan_destroy(h)
    keys = [tuple(int(x) for x in r) for r in buf[: nb.value * lo].reshape(nb.value, lo)]
    mult = [dict(zip(*np.unique(l.charges, return_counts=True))) for l in out_legs]
    offs = [0]
    for k in keys:
        offs.append(offs[-1] + int(np.prod([mult[i].get(q, 0) for i, q in enumerate(k)])))
    assert offs[-1] == tot.value
    return keys, offs


def _ref_pairs(a, b, subs_a, subs_b, out_keys_sorted, out_subs):
    """The reference's signature matching, counted directly (A then B order)."""
    con = sorted(set(subs_a) & set(subs_b))
    ia_pos = [subs_a.index(c) for c in con]
    ib_pos = [subs_b.index(c) for c in con]
    valid = {k: i for i, k in enumerate(out_keys_sorted)}
    out = []
    for i, x in enumerate(sorted(a.blocks)):
        for j, y in enumerate(sorted(b.blocks)):
            if [x[p] for p in ia_pos] != [y[p] for p in ib_pos]:
                continue
            c2q = dict(zip(subs_a, x))
            c2q.update(dict(zip(subs_b, y)))
            ok = tuple(int(c2q[c]) for c in out_subs)
            if ok in valid:
                out.append([i, j, valid[ok]])
    return out


def test_contract_structure_golden(golden_dir):
    z = np.load(os.path.join(golden_dir, "contract.npz"))
    n_checked = 0
    for c in json.load(open(os.path.join(golden_dir, "contract.json"))):
        if c["n_in"] != 2:
            continue
        lhs, out_subs = c["subscripts"].split("->")
        if not out_subs:
            continue
        sa, sb = lhs.split(",")
        a, b = (unpack_tensor(z, f"{c['name']}.in{i}") for i in range(2))
        keys, offs, pairs = _structure_dev(a, b, sa, sb, out_subs, a.modulus)
        hkeys, hoffs = _host_plan(a, b, sa, sb, out_subs, a.modulus)
        assert keys == hkeys and offs == hoffs, c["name"]
        ref = unpack_tensor(z, f"{c['name']}.out")
        assert set(keys) == set(ref.blocks), c["name"]
        assert pairs == _ref_pairs(a, b, sa, sb, keys, out_subs), c["name"]
        n_checked += 1
    assert n_checked >= 3


@pytest.mark.parametrize("chi", [256, 2048])
def test_contract_structure_benchmark_stage1(chi):
    """L . theta over a (the H_eff's first pairwise stage) on the benchmark's
    structures: output keys, offsets and pairs."""
    args, _ = _bench_mod().HostProblems(2).make(chi, fill=False)
    L, T = args[0], args[1]
    keys, offs, pairs = _structure_dev(L, T, "abc", "apqd", "bcpqd", None)
    hkeys, hoffs = _host_plan(L, T, "abc", "apqd", "bcpqd", None)
    assert keys == hkeys and offs == hoffs
    assert pairs == _ref_pairs(L, T, "abc", "apqd", keys, "bcpqd")


def test_fused_charges_golden(golden_dir):
    from oracle.blocksparse import fused_charges

    cases = json.load(open(os.path.join(golden_dir, "fuse.json")))
    z = np.load(os.path.join(golden_dir, "fuse.npz"))
    for c in cases:
        t = unpack_tensor(z, f"{c['name']}.in")
        la, lb = t.legs[c["axis_a"]], t.legs[c["axis_b"]]
        ref = fused_charges(la, lb, c["fused_flow"], t.modulus)
        qa, qb = _dev_i32(la.charges), _dev_i32(lb.charges)
        out = torch.empty(len(la.charges) * len(lb.charges), dtype=torch.int32, device="cuda")
        _capi.check(_capi.LIB.tnx_fused_charges_dev(qa.data_ptr(), len(la.charges), int(la.flow), qb.data_ptr(),
                                                    len(lb.charges), int(lb.flow), int(c["fused_flow"]),
                                                    int(t.modulus or 0), out.data_ptr(), _stream()))
        np.testing.assert_array_equal(out.cpu().numpy(), np.asarray(ref, np.int32), err_msg=c["name"])
