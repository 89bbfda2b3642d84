"""ctypes binding of ``libtenax_b200.so`` (declared in ``include/tenax_b200.h``).

The library is required: importing this module without it raises, and every
product code path goes through it -- there is no CPU fallback.
"""

from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libtenax_b200.so")

TNX_OK = 0
TNX_ERR_VALUE = 1
TNX_ERR_TYPE = 2
TNX_ERR_RUNTIME = 3
TNX_ERR_CUDA = 4
TNX_ERR_TIMEOUT = 5
TNX_ERR_UNSUPPORTED = 6

PREC_FP64 = 0
PREC_BF16X3 = 1
PREC_TF32 = 2
PRECISIONS = {"fp64": PREC_FP64, "bf16x3": PREC_BF16X3, "tf32": PREC_TF32}

MATCH_FILTERED = 0
MATCH_UNFILTERED = 1


class TnxUnsupported(NotImplementedError):
    """Valid input outside what this build implements."""


class HeffSchedule(C.Structure):
    """tnx_heff_schedule: fused stages 1-3 on/off and c values per tile (0 = auto)."""

    _fields_ = [("fuse_mpo", C.c_int32), ("c_per_tile", C.c_int32)]


class TensorDesc(C.Structure):
    _fields_ = [
        ("n_legs", C.c_int32),
        ("subs", C.c_char_p),
        ("flows", C.POINTER(C.c_int32)),
        ("charges", C.POINTER(C.c_int32)),
        ("leg_dims", C.POINTER(C.c_int64)),
        ("n_blocks", C.c_int64),
        ("keys", C.POINTER(C.c_int32)),
    ]


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python tenax_b200/build.py` "
            "(the package has no CPU fallback)"
        )
    lib = C.CDLL(LIB_PATH)
    P = C.c_void_p
    i32, i64, dbl = C.c_int32, C.c_int64, C.c_double
    sig = {
        "tnx_last_error": (C.c_char_p, []),
        "tnx_version": (C.c_int, []),
        "tnx_valid_blocks": (C.c_int, [i32, P, P, P, i32, i32, i64, P, P, i64]),
        "tnx_plan_create": (C.c_int, [P, i32, C.c_char_p, i32, i32, P, P, P, P]),
        "tnx_plan_create_graded": (C.c_int, [P, i32, C.c_char_p, i32, i32, P, P, P, i32, P]),
        "tnx_plan_output": (C.c_int, [P, P, P, P, P, P]),
        "tnx_plan_workspace": (C.c_int, [P, i32, P]),
        "tnx_plan_flops": (dbl, [P]),
        "tnx_plan_execute": (C.c_int, [P, P, P, i32, P, C.c_size_t, P]),
        "tnx_plan_destroy": (None, [P]),
        "tnx_plan_execute_static": (C.c_int, [P, P, P, P]),
        "tnx_valid_blocks_dev": (C.c_int, [i32, P, P, P, i32, i32, i64, P, P, i64, P]),
        "tnx_contract_structure_dev": (C.c_int, [P, P, C.c_char_p, i32, P, P, P, i64, P, P, i64, P]),
        "tnx_fused_charges_dev": (C.c_int, [P, i64, i32, P, i64, i32, i32, i32, P, P]),
        "tnx_heff_create": (C.c_int, [P, P, P, P, P, P]),
        "tnx_heff_create_for": (C.c_int, [P, P, P, P, P, i32, P]),
        "tnx_heff_closed": (C.c_int, [P, P]),
        "tnx_heff_set_schedule": (C.c_int, [P, P]),
        "tnx_heff_get_schedule": (C.c_int, [P, P]),
        "tnx_heff_out_keys": (C.c_int, [P, P, P]),
        "tnx_heff_flops": (dbl, [P]),
        "tnx_heff_set_operators": (C.c_int, [P, P, P, P, P, i32, P]),
        "tnx_heff_destroy": (None, [P]),
        "tnx_heff_batch_create": (C.c_int, [P, i32, i32, P]),
        "tnx_heff_batch_apply": (C.c_int, [P, P, P, P]),
        "tnx_heff_batch_apply_host": (C.c_int, [P, P, P, i32, P]),
        "tnx_heff_batch_size": (C.c_int, [P, P, P]),
        "tnx_heff_batch_launches": (C.c_int, [P, P]),
        "tnx_heff_batch_route_stats": (C.c_int, [P, P, P]),
        "tnx_heff_batch_apply_stage": (C.c_int, [P, i32, P]),
        "tnx_heff_stage_flops": (C.c_int, [P, P]),
        "tnx_heff_batch_error": (C.c_int, [P, P]),
        "tnx_heff_batch_set_skip_flag": (C.c_int, [P, P]),
        "tnx_heff_batch_destroy": (None, [P]),
        "tnx_reduce_scratch_len": (i64, []),
        "tnx_dot": (C.c_int, [P, P, i64, P, P, P]),
        "tnx_nrm2": (C.c_int, [P, i64, P, P, P]),
        "tnx_wait_flag": (C.c_int, [P, i32, i64, P, P]),
        "tnx_svd_batch": (C.c_int, [i32, P, P, P, P, P, P, i64, i32, P, P]),
        "tnx_lanczos_step": (C.c_int, [P, P, P, P, i64, P, P, i32, dbl, dbl, P, P, P]),
        "tnx_combine": (C.c_int, [P, P, i32, i64, P, P]),
        "tnx_scale": (C.c_int, [P, P, i64, P, i32, P]),
        "tnx_fuse_plan_create": (C.c_int, [P, i32, i32, i32, i32, P]),
        "tnx_fuse_plan_output": (C.c_int, [P, P, P, P, P, P]),
        "tnx_fuse_execute": (C.c_int, [P, P, P, P]),
        "tnx_fuse_plan_destroy": (None, [P]),
        "tnx_fuse_row_map": (C.c_int, [P, i64, i32, P, i64, i32, i32, i32, P]),
        "tnx_renorm_scratch_len": (i64, []),
        "tnx_renorm_maxabs": (C.c_int, [C.c_int, P, P, P, dbl, P, P, P]),
        "tnx_renorm_maxabs_adjoint": (C.c_int, [C.c_int, P, P, P, P, dbl, P, P, P]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


LIB = _load()
EXPORTED = [
    "tnx_last_error", "tnx_version", "tnx_valid_blocks", "tnx_plan_create", "tnx_plan_create_graded",
    "tnx_plan_output",
    "tnx_plan_workspace", "tnx_plan_flops", "tnx_plan_execute", "tnx_plan_destroy", "tnx_plan_execute_static",
    "tnx_valid_blocks_dev", "tnx_contract_structure_dev", "tnx_fused_charges_dev",
    "tnx_heff_create", "tnx_heff_create_for",
    "tnx_heff_closed", "tnx_heff_set_schedule", "tnx_heff_get_schedule", "tnx_heff_out_keys", "tnx_heff_flops", "tnx_heff_set_operators", "tnx_heff_destroy",
    "tnx_heff_batch_create", "tnx_heff_batch_apply", "tnx_heff_batch_apply_host", "tnx_heff_batch_size",
    "tnx_heff_batch_apply_stage", "tnx_heff_stage_flops",
    "tnx_heff_batch_launches", "tnx_heff_batch_route_stats", "tnx_heff_batch_error",
    "tnx_heff_batch_set_skip_flag", "tnx_heff_batch_destroy", "tnx_reduce_scratch_len", "tnx_dot", "tnx_nrm2", "tnx_wait_flag",
    "tnx_svd_batch",
    "tnx_lanczos_step", "tnx_combine", "tnx_scale", "tnx_fuse_plan_create", "tnx_fuse_plan_output",
    "tnx_fuse_execute", "tnx_fuse_plan_destroy", "tnx_fuse_row_map", "tnx_renorm_scratch_len", "tnx_renorm_maxabs",
    "tnx_renorm_maxabs_adjoint",
]


def check(status: int) -> None:
    """Map a status code to the exception the reference raises."""
    if status == TNX_OK:
        return
    msg = LIB.tnx_last_error().decode(errors="replace")
    if status == TNX_ERR_VALUE:
        raise ValueError(msg)
    if status == TNX_ERR_TYPE:
        raise TypeError(msg)
    if status == TNX_ERR_UNSUPPORTED:
        raise TnxUnsupported(msg)
    raise RuntimeError(f"tenax_b200 error {status}: {msg}")


class DescHolder:
    """Owns the numpy arrays a ``TensorDesc`` points into."""

    def __init__(self, charges_per_leg, flows, keys, subs: str | None):
        self.nl = len(flows)
        self.flows = np.ascontiguousarray(np.asarray(flows, dtype=np.int32))
        self.leg_dims = np.ascontiguousarray(np.array([len(c) for c in charges_per_leg], dtype=np.int64))
        self.charges = np.ascontiguousarray(
            np.concatenate([np.asarray(c, dtype=np.int32) for c in charges_per_leg])
            if charges_per_leg
            else np.zeros(1, np.int32)
        )
        k = np.asarray(keys, dtype=np.int32).reshape(-1, self.nl) if self.nl else np.zeros((len(keys), 0), np.int32)
        self.keys = np.ascontiguousarray(k if k.size else np.zeros(1, np.int32))
        self.n_blocks = len(keys)
        self.subs = subs.encode() if subs is not None else None
        self.desc = TensorDesc(
            self.nl,
            self.subs,
            self.flows.ctypes.data_as(C.POINTER(C.c_int32)),
            self.charges.ctypes.data_as(C.POINTER(C.c_int32)),
            self.leg_dims.ctypes.data_as(C.POINTER(C.c_int64)),
            self.n_blocks,
            self.keys.ctypes.data_as(C.POINTER(C.c_int32)),
        )


def valid_blocks(charges_per_leg, flows, modulus: int | None, target: int | None):
    """Valid block keys in the reference's order (core/tensor.py:53-165)."""
    d = DescHolder(charges_per_leg, flows, [], None)
    n = C.c_int64(0)
    mod = 0 if modulus is None else int(modulus)
    has_t = 0 if target is None else 1
    tgt = 0 if target is None else int(target)
    check(LIB.tnx_valid_blocks(d.nl, d.charges.ctypes.data, d.leg_dims.ctypes.data, d.flows.ctypes.data, mod,
                               has_t, tgt, C.byref(n), None, 0))
    out = np.zeros(max(1, n.value * d.nl), dtype=np.int32)
    check(LIB.tnx_valid_blocks(d.nl, d.charges.ctypes.data, d.leg_dims.ctypes.data, d.flows.ctypes.data, mod,
                               has_t, tgt, C.byref(n), out.ctypes.data, out.size))
    if d.nl == 0:
        return [()] * n.value
    return [tuple(int(q) for q in row) for row in out[: n.value * d.nl].reshape(-1, d.nl)]
