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


def _parity_mod2(q):
    return np.mod(np.asarray(q, dtype=np.int64), 2).astype(np.int32)


class FermionParity(BaseSymmetry):
    """Z2 charges with fermionic exchange statistics (core/symmetry.py:311-364):
    fuse mod 2, self-dual, parity q mod 2."""

    modulus = 2

    def fuse(self, a, b):
        return (a + b) % 2

    def dual(self, q):
        return q

    @property
    def is_fermionic(self) -> bool:
        return True

    def parity(self, q):
        return _parity_mod2(q)

    def exchange_sign(self, qa: int, qb: int) -> int:
        return 1 - 2 * ((int(qa) % 2) * (int(qb) % 2))

    def twist_phase(self, q: int) -> float:
        return (-1.0) ** (int(q) % 2)

    def __eq__(self, other):
        return isinstance(other, FermionParity)

    def __hash__(self):
        return hash("FermionParity")

    def __repr__(self):
        return "FermionParity()"


class FermionicU1(BaseSymmetry):
    """Integer charges with fermionic statistics (core/symmetry.py:374-440).
    The built-in gradings ("abs_mod_2", "mod_2") both give parity q mod 2 on
    integers, which is what the contraction engine's signs use; a custom
    grading function is kept for ``parity`` but the engine rejects it."""

    modulus = None
    _BUILTIN = ("abs_mod_2", "mod_2")

    def __init__(self, grading=None, grading_key: str = "abs_mod_2"):
        if grading is None and grading_key not in self._BUILTIN:
            raise ValueError(f"Unknown grading_key: {grading_key!r}")
        self._grading = grading
        self.grading_key = grading_key

    @property
    def builtin_grading(self) -> bool:
        return self._grading is None

    def fuse(self, a, b):
        return a + b

    def dual(self, q):
        return -q

    @property
    def is_fermionic(self) -> bool:
        return True

    def parity(self, q):
        if self._grading is None:
            return _parity_mod2(q)
        return np.array([self._grading(int(x)) for x in np.atleast_1d(q)], dtype=np.int32)

    def exchange_sign(self, qa: int, qb: int) -> int:
        pa, pb = int(self.parity([qa])[0]), int(self.parity([qb])[0])
        return 1 - 2 * (pa * pb)

    def twist_phase(self, q: int) -> float:
        return (-1.0) ** int(self.parity([q])[0])

    def __eq__(self, other):
        return isinstance(other, FermionicU1) and other.grading_key == self.grading_key

    def __hash__(self):
        return hash(("FermionicU1", self.grading_key))

    def __repr__(self):
        return f"FermionicU1(grading_key={self.grading_key!r})"


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
