"""Device-resident block-sparse ``SymmetricTensor``.

Same storage model as tenax (core/tensor.py:505-974): a set of charge
sectors (one charge per leg, conservation law sum(flow*q) == identity), each
a dense row-major block whose dims are the leg multiplicities of its charges.
Here all blocks of a tensor live in ONE flat float64 CUDA buffer in
sorted-key order (tenax's pytree leaf order, core/tensor.py:572-578), with a
host-side key list and offset table; ``.blocks`` exposes per-key views.
"""

from __future__ import annotations

from typing import Any

import numpy as np
import torch

from tenax_b200 import _capi
from tenax_b200.core import TensorIndex

BlockKey = tuple


def _device() -> torch.device:
    if not torch.cuda.is_available():
        raise RuntimeError("tenax_b200 stores tensors on a CUDA device; none is available")
    return torch.device("cuda", torch.cuda.current_device())


def _modulus(indices) -> int | None:
    return indices[0].symmetry.n_values() if indices else None


def block_shape(indices, key) -> tuple:
    return tuple(int(np.count_nonzero(idx.charges == q)) for idx, q in zip(indices, key))


def compute_valid_blocks(indices, target=None):
    """Valid keys in the reference's order (core/tensor.py:53-165), via the planner."""
    if not indices:
        return [()]
    return _capi.valid_blocks([i.charges for i in indices], [int(i.flow) for i in indices], _modulus(indices), target)


class SymmetricTensor:
    """Block-sparse tensor; blocks in one flat CUDA float64 buffer."""

    __slots__ = ("_indices", "_keys", "_data", "_offsets", "_shapes", "_key_pos", "_blocks_cache")

    def __init__(self, blocks: dict, indices, _validate: bool = True):
        indices = tuple(indices)
        keys = sorted(tuple(int(q) for q in k) for k in blocks)
        arrays = []
        for k in keys:
            v = blocks[k] if k in blocks else blocks[tuple(np.int32(q) for q in k)]
            t = torch.as_tensor(np.asarray(v) if not isinstance(v, torch.Tensor) else v)
            arrays.append(t.reshape(-1).to(dtype=torch.float64))
        dev = _device()
        data = torch.cat(arrays).to(dev) if arrays else torch.zeros(0, dtype=torch.float64, device=dev)
        self._init_flat(indices, keys, data)
        if _validate:
            self._validate()

    # ------------------------------------------------------------ construction
    def _init_flat(self, indices, keys, data):
        self._indices = tuple(indices)
        self._keys = list(keys)
        shapes = [block_shape(self._indices, k) for k in self._keys]
        sizes = [int(np.prod(s)) if s else 1 for s in shapes]
        offs = np.zeros(len(keys) + 1, dtype=np.int64)
        if sizes:
            offs[1:] = np.cumsum(sizes)
        if data.numel() != int(offs[-1]):
            raise ValueError(f"flat buffer has {data.numel()} elements, blocks need {int(offs[-1])}")
        self._data = data
        self._offsets = offs
        self._shapes = shapes
        self._key_pos = {k: i for i, k in enumerate(self._keys)}
        self._blocks_cache = None

    @classmethod
    def from_flat(cls, indices, keys, data: torch.Tensor) -> "SymmetricTensor":
        """Wrap an existing flat buffer (blocks in the given sorted key order)."""
        obj = object.__new__(cls)
        obj._init_flat(indices, [tuple(int(q) for q in k) for k in keys], data)
        return obj

    def _validate(self):
        if not self._indices:
            return
        sym = self._indices[0].symmetry
        for key in self._keys:
            eff = [int(i.flow) * int(q) for i, q in zip(self._indices, key)]
            fused = sym.fuse_many(eff)
            if fused != sym.identity():
                raise ValueError(f"Block {key} violates charge conservation: fused={fused}, "
                                 f"expected identity={sym.identity()}")

    @classmethod
    def zeros(cls, indices, dtype: Any = np.float64, target=None) -> "SymmetricTensor":
        keys = [k for k in compute_valid_blocks(tuple(indices), target) if all(s > 0 for s in block_shape(indices, k))]
        keys = sorted(keys)
        total = sum(int(np.prod(block_shape(indices, k))) for k in keys)
        t = cls.from_flat(indices, keys, torch.zeros(total, dtype=torch.float64, device=_device()))
        if target in (None, 0):
            t._validate()
        return t

    @classmethod
    def random_normal(cls, indices, key=0, dtype: Any = np.float64, stddev: float = 1.0,
                      target=None) -> "SymmetricTensor":
        """N(0, stddev) blocks over the valid keys in sorted order.

        ``key`` is an int seed or a ``numpy.random.Generator`` (the reference
        takes a jax PRNG key; values are drawn with numpy here).
        """
        rng = key if isinstance(key, np.random.Generator) else np.random.default_rng(int(np.asarray(key).sum()))
        keys = sorted(k for k in compute_valid_blocks(tuple(indices), target)
                      if all(s > 0 for s in block_shape(indices, k)))
        parts = [rng.standard_normal(block_shape(indices, k)).ravel() * stddev for k in keys]
        flat = np.concatenate(parts) if parts else np.zeros(0)
        t = cls.from_flat(indices, keys, torch.from_numpy(flat).to(_device()))
        if target in (None, 0):
            t._validate()
        return t

    @classmethod
    def from_dense(cls, data, indices, tol: float = 1e-12) -> "SymmetricTensor":
        """Extract the valid sectors of a dense array (core/tensor.py:670-732).

        Every valid key whose legs all have basis states gets a block (zero
        blocks included).  A CUDA tensor is cut on the device by index
        gathers; host arrays are cut on the host and copied once."""
        if isinstance(data, torch.Tensor) and data.is_cuda:
            return cls._from_dense_device(data, tuple(indices), tol)
        arr = data.detach().cpu().numpy() if isinstance(data, torch.Tensor) else np.asarray(data)
        if arr.shape != tuple(i.dim for i in indices):
            raise ValueError(f"data.shape {arr.shape} does not match index dims {tuple(i.dim for i in indices)}")
        keys = sorted(compute_valid_blocks(tuple(indices)))
        mask = np.zeros(arr.shape, dtype=bool)
        blocks = {}
        for k in keys:
            pos = [np.where(i.charges == q)[0] for i, q in zip(indices, k)]
            if not all(len(p) for p in pos):
                continue
            grid = np.ix_(*pos)
            blocks[k] = arr[grid]
            mask[grid] = True
        if tol != float("inf"):
            outside = arr[~mask]
            if np.any(np.abs(outside) > tol):
                raise ValueError(f"data has {int(np.sum(np.abs(outside) > tol))} non-zero elements outside "
                                 f"symmetry-allowed sectors (max abs value: {np.max(np.abs(outside)):.3e})")
        return cls(blocks, indices)

    @classmethod
    def _from_dense_device(cls, x: torch.Tensor, indices, tol: float) -> "SymmetricTensor":
        if tuple(x.shape) != tuple(i.dim for i in indices):
            raise ValueError(f"data.shape {tuple(x.shape)} does not match index dims {tuple(i.dim for i in indices)}")
        x = x.detach().to(dtype=torch.float64)
        keys, parts = [], []
        mask = torch.zeros(x.shape, dtype=torch.bool, device=x.device) if tol != float("inf") else None
        for k in sorted(compute_valid_blocks(indices)):
            pos = [np.flatnonzero(i.charges == q) for i, q in zip(indices, k)]
            if not all(len(p) for p in pos):
                continue
            grid = torch.meshgrid(*[torch.as_tensor(p, device=x.device) for p in pos], indexing="ij")
            parts.append(x[grid].reshape(-1))
            keys.append(tuple(int(q) for q in k))
            if mask is not None:
                mask[grid] = True
        if mask is not None:
            outside = x[~mask].abs()
            n_bad = int((outside > tol).sum())
            if n_bad:
                raise ValueError(f"data has {n_bad} non-zero elements outside symmetry-allowed sectors "
                                 f"(max abs value: {float(outside.max()):.3e})")
        data = torch.cat(parts) if parts else torch.zeros(0, dtype=torch.float64, device=x.device)
        return cls.from_flat(indices, keys, data)

    # ------------------------------------------------------------ accessors
    @property
    def indices(self):
        return self._indices

    @property
    def ndim(self) -> int:
        return len(self._indices)

    @property
    def dtype(self):
        return torch.float64

    @property
    def n_blocks(self) -> int:
        return len(self._keys)

    @property
    def keys(self) -> list:
        return self._keys

    @property
    def data(self) -> torch.Tensor:
        """The flat device buffer (blocks in sorted-key order)."""
        return self._data

    @property
    def offsets(self) -> np.ndarray:
        return self._offsets

    @property
    def blocks(self) -> dict:
        if self._blocks_cache is None:
            self._blocks_cache = {
                k: self._data[self._offsets[i]:self._offsets[i + 1]].view(self._shapes[i])
                for i, k in enumerate(self._keys)
            }
        return self._blocks_cache

    def labels(self) -> tuple:
        return tuple(i.label for i in self._indices)

    def block_shapes(self) -> dict:
        return {k: s for k, s in zip(self._keys, self._shapes)}

    def numpy_blocks(self) -> dict:
        host = self._data.detach().cpu().numpy()
        return {k: host[self._offsets[i]:self._offsets[i + 1]].reshape(self._shapes[i]) for i, k in enumerate(self._keys)}

    # ------------------------------------------------------------ dense view
    def todense(self) -> torch.Tensor:
        shape = tuple(i.dim for i in self._indices)
        out = torch.zeros(shape, dtype=torch.float64, device=self._data.device)
        for k, blk in self.blocks.items():
            pos = [torch.as_tensor(np.where(i.charges == q)[0], device=out.device) for i, q in zip(self._indices, k)]
            out[torch.meshgrid(*pos, indexing="ij")] = blk
        return out

    # ------------------------------------------------------------ algebra
    def _like(self, data, indices=None) -> "SymmetricTensor":
        return SymmetricTensor.from_flat(self._indices if indices is None else indices, self._keys, data)

    def conj(self) -> "SymmetricTensor":
        return self._like(self._data)  # real float64 data

    def bar(self) -> "SymmetricTensor":
        return self._like(self._data, tuple(i.flip_flow() for i in self._indices))

    def dagger(self) -> "SymmetricTensor":
        """Conjugate with dual legs (core/tensor.py:795-820); blocks of a
        fermionic tensor take the twist phase, (-1) to the total parity of
        their charges."""
        sym = self._indices[0].symmetry if self._indices else None
        new_idx = tuple(i.dual() for i in self._indices)
        new_keys = [tuple(int(sym.dual(np.int64(q))) for q in k) for k in self._keys]
        blocks = {}
        for nk, k in zip(new_keys, self._keys):
            b = self.blocks[k]
            if sym is not None and sym.is_fermionic and int(np.sum(sym.parity(np.asarray(k)))) % 2:
                b = -b
            blocks[nk] = b
        return SymmetricTensor(blocks, new_idx, _validate=False)

    def transpose(self, axes) -> "SymmetricTensor":
        from tenax_b200.contraction import transpose_symmetric

        return transpose_symmetric(self, tuple(axes))

    def norm(self) -> torch.Tensor:
        """Frobenius norm (core/tensor.py:863-868), FP64 two-pass reduction on device."""
        from tenax_b200.vector import nrm2

        return nrm2(self._data)

    def max_abs(self) -> torch.Tensor:
        if self._data.numel() == 0:
            return torch.zeros((), dtype=torch.float64, device=self._data.device)
        return self._data.abs().max()

    def relabel(self, old, new) -> "SymmetricTensor":
        if old not in self.labels():
            raise KeyError(f"Label {old!r} not found in tensor with labels {self.labels()}")
        return self._like(self._data, tuple(i.relabel(new) if i.label == old else i for i in self._indices))

    def relabels(self, mapping: dict) -> "SymmetricTensor":
        return self._like(self._data, tuple(i.relabel(mapping[i.label]) if i.label in mapping else i
                                            for i in self._indices))

    def __mul__(self, scalar) -> "SymmetricTensor":
        return self._like(self._data * float(scalar))

    __rmul__ = __mul__

    def __neg__(self):
        return self * -1.0

    def __add__(self, other) -> "SymmetricTensor":
        """Key-union addition (core/tensor.py:933-952)."""
        if not isinstance(other, SymmetricTensor):
            raise TypeError(f"Cannot add SymmetricTensor and {type(other).__name__}; convert to matching type first.")
        if self._keys == other._keys:
            return self._like(self._data + other._data)
        keys = sorted(set(self._keys) | set(other._keys))
        out = SymmetricTensor.from_flat(self._indices, keys, torch.zeros(
            sum(int(np.prod(block_shape(self._indices, k))) for k in keys), dtype=torch.float64,
            device=self._data.device))
        for src in (self, other):
            idx = _scatter_index(src, out)
            out._data.index_add_(0, idx, src._data)
        return out

    def __sub__(self, other) -> "SymmetricTensor":
        if not isinstance(other, SymmetricTensor):
            raise TypeError(f"Cannot subtract {type(other).__name__} from SymmetricTensor.")
        return self + other * -1.0

    def __repr__(self):
        return (f"SymmetricTensor(ndim={self.ndim}, n_blocks={self.n_blocks}, nnz={self._data.numel()}, "
                f"dtype=float64, labels={self.labels()})")


def _scatter_index(src: SymmetricTensor, dst: SymmetricTensor) -> torch.Tensor:
    """Positions in ``dst``'s flat buffer of every element of ``src``."""
    parts = []
    for i, k in enumerate(src._keys):
        j = dst._key_pos[k]
        n = src._offsets[i + 1] - src._offsets[i]
        parts.append(np.arange(dst._offsets[j], dst._offsets[j] + n, dtype=np.int64))
    idx = np.concatenate(parts) if parts else np.zeros(0, np.int64)
    return torch.from_numpy(idx).to(src._data.device)


def restrict_to_keys(t: SymmetricTensor, keys) -> SymmetricTensor:
    """Copy of ``t`` with only ``keys`` (a subset of its keys), sorted."""
    keys = sorted(keys)
    if keys == t._keys:
        return t
    parts = [t._data[t._offsets[t._key_pos[k]]:t._offsets[t._key_pos[k] + 1]] for k in keys]
    data = torch.cat(parts) if parts else torch.zeros(0, dtype=torch.float64, device=t._data.device)
    return SymmetricTensor.from_flat(t._indices, keys, data)


def embed_in_keys(t: SymmetricTensor, keys) -> SymmetricTensor:
    """``t`` laid out over a superset of its keys (missing blocks are zero)."""
    keys = sorted(keys)
    if keys == t._keys:
        return t
    out = SymmetricTensor.from_flat(t._indices, keys, torch.zeros(
        sum(int(np.prod(block_shape(t._indices, k))) for k in keys), dtype=torch.float64, device=t._data.device))
    out._data.index_copy_(0, _scatter_index(t, out), t._data)
    return out


def inner(a: SymmetricTensor, b: SymmetricTensor) -> torch.Tensor:
    """sum over common keys of conj(a)*b (core/tensor.py:296-319), FP64 on device."""
    from tenax_b200.vector import dot

    if a._keys == b._keys:
        return dot(a._data, b._data)
    common = sorted(set(a._keys) & set(b._keys))
    return dot(restrict_to_keys(a, common)._data, restrict_to_keys(b, common)._data)
