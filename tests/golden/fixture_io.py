"""Serialisation of block-sparse tensors for the golden fixtures.

A tensor ``T`` is stored in an ``.npz`` as flat arrays under a name prefix:
``<p>.charges`` (all legs' int32 charges concatenated), ``<p>.legdims``,
``<p>.flows``, ``<p>.labels`` (JSON), ``<p>.keys`` (n_blocks x n_legs int32,
sorted-key order), ``<p>.data`` (float64 blocks concatenated in key order,
each row-major) and ``<p>.modulus`` (0 for U(1)).
"""

from __future__ import annotations

import json

import numpy as np

from oracle.blocksparse import Leg, OTensor, block_shape


def pack_tensor(prefix: str, legs, blocks: dict, modulus=None) -> dict:
    keys = sorted(blocks.keys())
    charges = [np.asarray(l[0], dtype=np.int32) for l in legs]
    out = {
        f"{prefix}.charges": np.concatenate(charges) if charges else np.zeros(0, np.int32),
        f"{prefix}.legdims": np.array([len(c) for c in charges], dtype=np.int64),
        f"{prefix}.flows": np.array([int(l[1]) for l in legs], dtype=np.int32),
        f"{prefix}.labels": np.array(json.dumps([l[2] for l in legs])),
        f"{prefix}.keys": np.array(keys, dtype=np.int32).reshape(len(keys), len(legs)),
        f"{prefix}.data": (
            np.concatenate([np.asarray(blocks[k], dtype=np.float64).ravel() for k in keys])
            if keys
            else np.zeros(0)
        ),
        f"{prefix}.modulus": np.array(0 if modulus is None else int(modulus)),
    }
    return out


def unpack_tensor(z, prefix: str) -> OTensor:
    dims = z[f"{prefix}.legdims"]
    charges = np.split(z[f"{prefix}.charges"], np.cumsum(dims)[:-1]) if len(dims) else []
    flows = z[f"{prefix}.flows"]
    labels = json.loads(str(z[f"{prefix}.labels"]))
    legs = tuple(Leg(np.asarray(c, np.int32), int(f), lab) for c, f, lab in zip(charges, flows, labels))
    keys = [tuple(int(q) for q in k) for k in z[f"{prefix}.keys"]]
    data = z[f"{prefix}.data"]
    mod = int(z[f"{prefix}.modulus"])
    blocks = {}
    off = 0
    for k in keys:
        shp = block_shape([l.charges for l in legs], k)
        n = int(np.prod(shp))
        blocks[k] = data[off:off + n].reshape(shp)
        off += n
    return OTensor(legs, blocks, None if mod == 0 else mod)
