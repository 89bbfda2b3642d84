"""Leg metadata of block-sparse tensors: symmetry groups, flows, indices.

Host-side integer metadata with the same meaning as tenax's
``core/symmetry.py`` (U1: charges add; Z_n: charges add mod n) and
``core/index.py`` (``TensorIndex(symmetry, charges, flow, label)``).
"""

from __future__ import annotations

from dataclasses import dataclass
from enum import IntEnum

import numpy as np

Label = str | int


class BaseSymmetry:
    """Abelian charge algebra: ``fuse``, ``dual``, ``identity``, ``n_values``."""

    modulus: int | None = None

    def fuse(self, a, b):
        raise NotImplementedError

    def dual(self, q):
        raise NotImplementedError

    def identity(self) -> int:
        return 0

    def n_values(self):
        return self.modulus

    def fuse_many(self, charge_list):
        if not charge_list:
            raise ValueError("charge_list must be non-empty")
        out = charge_list[0]
        for c in charge_list[1:]:
            out = self.fuse(out, c)
        return out

    @property
    def is_fermionic(self) -> bool:
        return False


class U1Symmetry(BaseSymmetry):
    """Integer charges fused by addition (core/symmetry.py:182-213)."""

    modulus = None

    def fuse(self, a, b):
        return a + b

    def dual(self, q):
        return -q

    def __eq__(self, other):
        return isinstance(other, U1Symmetry)

    def __hash__(self):
        return hash("U1Symmetry")

    def __repr__(self):
        return "U1Symmetry()"


class ZnSymmetry(BaseSymmetry):
    """Charges mod n (core/symmetry.py:216-255); n >= 2."""

    def __init__(self, n: int):
        if n < 2:
            raise ValueError(f"n must be >= 2, got {n}")
        self.n = int(n)
        self.modulus = self.n

    def fuse(self, a, b):
        return (a + b) % self.n

    def dual(self, q):
        return (-q) % self.n

    def __eq__(self, other):
        return isinstance(other, ZnSymmetry) and other.n == self.n

    def __hash__(self):
        return hash(("ZnSymmetry", self.n))

    def __repr__(self):
        return f"ZnSymmetry({self.n})"


class FlowDirection(IntEnum):
    """IN (+1) / OUT (-1); a valid block has sum(flow * charge) == identity."""

    IN = 1
    OUT = -1


@dataclass(frozen=True, eq=False)
class TensorIndex:
    """One leg: symmetry, int32 charge of each basis state, flow, label."""

    symmetry: BaseSymmetry
    charges: np.ndarray
    flow: FlowDirection
    label: Label = ""

    def __post_init__(self):
        c = np.asarray(self.charges)
        if c.ndim != 1:
            raise ValueError(f"charges must be 1-D, got shape {c.shape}")
        if c.dtype != np.int32:
            c = c.astype(np.int32)
        object.__setattr__(self, "charges", c)
        object.__setattr__(self, "flow", FlowDirection(int(self.flow)))

    @property
    def dim(self) -> int:
        return int(len(self.charges))

    def dual(self) -> "TensorIndex":
        return TensorIndex(self.symmetry, np.asarray(self.symmetry.dual(self.charges), np.int32),
                           FlowDirection(-int(self.flow)), self.label)

    def flip_flow(self) -> "TensorIndex":
        return TensorIndex(self.symmetry, self.charges, FlowDirection(-int(self.flow)), self.label)

    def relabel(self, new_label: Label) -> "TensorIndex":
        return TensorIndex(self.symmetry, self.charges, self.flow, new_label)

    def charge_dims(self) -> dict:
        """Multiplicity of each charge on this leg."""
        u, c = np.unique(self.charges, return_counts=True)
        return {int(q): int(n) for q, n in zip(u, c)}

    def __eq__(self, other):
        if not isinstance(other, TensorIndex):
            return NotImplemented
        return (type(self.symmetry) is type(other.symmetry) and self.symmetry == other.symmetry
                and np.array_equal(self.charges, other.charges) and self.flow == other.flow
                and self.label == other.label)

    def __hash__(self):
        return hash((self.symmetry, self.charges.tobytes(), int(self.flow), self.label))

    def __repr__(self):
        return f"TensorIndex(sym={self.symmetry!r}, dim={self.dim}, flow={self.flow.name}, label={self.label!r})"
