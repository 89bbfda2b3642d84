"""``.net`` network files and ``NetworkBlueprint`` (tenax ``network/netfile.py``).

A ``.net`` source declares a network's topology apart from its data::

    # comment
    A: i, j, k          tensor name and its leg labels, in order
    B: k, l
    TOUT: i, j, l       output label order (an empty TOUT contracts to a scalar)
    ORDER: ((A,B),C)    optional pairwise contraction order

The blueprint is parsed once, filled with block-sparse tensors and launched
repeatedly.  Without ORDER, ``launch()`` is one N-operand symmetric
contraction on the library's planner, with the reference's filtered
semantics -- including its silently empty result when three or more
operands contract different label sets (``contractor.py:398-403``);
``launch(pairwise=True)`` contracts the tensors pairwise in declaration
order instead, which gives the full contraction.  With ORDER each step is a
pairwise contraction and TOUT is applied by a final transpose.
"""

from __future__ import annotations

import string
from collections import Counter
from pathlib import Path
from typing import Any

from tenax_b200.contraction import _labels_to_subscripts, contract, contract_with_subscripts

__all__ = ["NetworkBlueprint", "from_netfile", "parse_netfile"]


def _lines_of(source) -> list:
    """A list of lines from a list, a Path, a path string or inline text
    (netfile.py:133-144)."""
    if isinstance(source, list):
        return source
    if isinstance(source, Path):
        return source.read_text().splitlines()
    p = Path(source)
    if p.is_file():
        return p.read_text().splitlines()
    return source.splitlines()


def parse_netfile(source) -> dict:
    """Topology of a ``.net`` source (netfile.py:48-130).

    Returns ``{"tensors": {name: [labels]}, "tout": [labels] | None,
    "order": str | None}``; raises ValueError on a line without ':', a
    duplicate TOUT/ORDER/tensor name, a tensor without labels, no tensors, or
    a label on more than two tensors."""
    tensors: dict = {}
    tout = None
    tout_seen = False
    order = None
    for lineno, raw in enumerate(_lines_of(source), 1):
        line = raw.strip()
        if not line or line.startswith("#"):
            continue
        if ":" not in line:
            raise ValueError(f"Line {lineno}: expected 'Name: labels' or 'TOUT:/ORDER:', got {line!r}")
        key, _, value = (x.strip() for x in line.partition(":"))
        if key == "TOUT":
            if tout_seen:
                raise ValueError(f"Line {lineno}: duplicate TOUT declaration")
            tout_seen = True
            tout = [x.strip() for x in value.split(",") if x.strip()] if value else []
        elif key == "ORDER":
            if order is not None:
                raise ValueError(f"Line {lineno}: duplicate ORDER declaration")
            order = value or None
        else:
            if key in tensors:
                raise ValueError(f"Line {lineno}: duplicate tensor name {key!r}")
            labels = [x.strip() for x in value.split(",") if x.strip()]
            if not labels:
                raise ValueError(f"Line {lineno}: tensor {key!r} has no labels")
            tensors[key] = labels
    if not tensors:
        raise ValueError("No tensor declarations found")
    uses = Counter(lbl for labels in tensors.values() for lbl in labels)
    for lbl, n in uses.items():
        if n > 2:
            raise ValueError(f"Label {lbl!r} appears on {n} tensors (max 2 allowed)")
    return {"tensors": tensors, "tout": tout, "order": order}


def _order_tokens(s: str) -> list:
    """'(', ')', ',' and names (netfile.py:198-216)."""
    out, i, s = [], 0, s.strip()
    while i < len(s):
        ch = s[i]
        if ch in "(),":
            out.append(ch)
            i += 1
        elif ch.isspace():
            i += 1
        else:
            j = i
            while j < len(s) and s[j] not in "(), \t\n":
                j += 1
            out.append(s[i:j])
            i = j
    return out


def _order_tree(tokens: list, pos: int):
    """Recursive descent over ``name | '(' tree ',' tree ')'`` (netfile.py:219-249)."""
    if pos >= len(tokens):
        raise ValueError("ORDER: unexpected end of expression")
    if tokens[pos] == "(":
        left, pos = _order_tree(tokens, pos + 1)
        if pos >= len(tokens) or tokens[pos] != ",":
            raise ValueError(f"ORDER: expected ',' after first operand at position {pos}")
        right, pos = _order_tree(tokens, pos + 1)
        if pos >= len(tokens) or tokens[pos] != ")":
            raise ValueError(f"ORDER: expected ')' at position {pos}")
        return (left, right), pos + 1
    name = tokens[pos]
    if name in "(),":
        raise ValueError(f"ORDER: unexpected token {name!r} at position {pos}")
    return name, pos + 1


def _order_steps(order: str, names: set) -> list:
    """Pairwise steps of an ORDER string, post-order; the k-th result is
    named ``_k`` (netfile.py:149-195)."""
    tokens = _order_tokens(order)
    tree, pos = _order_tree(tokens, 0)
    if pos != len(tokens):
        raise ValueError(f"ORDER: unexpected tokens after position {pos}: {tokens[pos:]}")
    steps: list = []

    def walk(node) -> str:
        if isinstance(node, str):
            if node not in names:
                raise ValueError(f"ORDER: unknown tensor name {node!r}. Known: {sorted(names)}")
            return node
        a, b = walk(node[0]), walk(node[1])
        steps.append((a, b))
        return f"_{len(steps) - 1}"

    walk(tree)
    return steps


def _subscripts_from_names(labels: dict, order: list, tout) -> str:
    """Einsum subscripts from label names alone, the rule of
    ``_labels_to_subscripts`` (netfile.py:252-322)."""
    uses = Counter(lbl for name in order for lbl in labels[name])
    for lbl, n in uses.items():
        if n > 2:
            raise ValueError(f"Label {lbl!r} appears {n} times (max 2)")
    free = {lbl for lbl, n in uses.items() if n == 1}
    every = sorted(uses)
    if len(every) > 52:
        raise ValueError(f"Too many unique labels ({len(every)}); max 52")
    letter = dict(zip(every, string.ascii_lowercase + string.ascii_uppercase))
    if tout is None:
        tout, seen = [], set()
        for name in order:
            for lbl in labels[name]:
                if lbl in free and lbl not in seen:
                    tout.append(lbl)
                    seen.add(lbl)
    else:
        for lbl in tout:
            if lbl not in free:
                raise ValueError(f"output_labels contains {lbl!r} which is not a free label. "
                                 f"Free labels are: {sorted(free)}")
    lhs = ",".join("".join(letter[lbl] for lbl in labels[name]) for name in order)
    return lhs + "->" + "".join(letter[lbl] for lbl in tout)


class NetworkBlueprint:
    """Parse once, fill slots, launch repeatedly (netfile.py:325-569)."""

    def __init__(self, source) -> None:
        spec = parse_netfile(source)
        self._labels: dict = spec["tensors"]
        self._names: list = list(self._labels)
        self._tout = spec["tout"]
        self._order_str = spec["order"]
        self._steps = _order_steps(self._order_str, set(self._names)) if self._order_str is not None else None
        self._subscripts = _subscripts_from_names(self._labels, self._names, self._tout)
        self._tensors: dict = {}

    @property
    def tensor_names(self) -> list:
        return list(self._names)

    @property
    def subscripts(self) -> str:
        return self._subscripts

    @property
    def output_labels(self):
        return self._tout

    def put_tensor(self, name: str, tensor, label_order=None) -> None:
        """Fill slot ``name``.  ``label_order`` names the meaning of each
        axis of ``tensor`` (relabelled to the blueprint's labels); without it
        the tensor must carry the blueprint's label set and is transposed to
        its order (netfile.py:385-447)."""
        if name not in self._labels:
            raise KeyError(f"Unknown tensor name {name!r}. Known: {self._names}")
        want = self._labels[name]
        if tensor.ndim != len(want):
            raise ValueError(f"Tensor {name!r} has rank {tensor.ndim} but blueprint expects rank {len(want)}")
        if label_order is not None:
            if len(label_order) != len(want):
                raise ValueError(f"label_order has {len(label_order)} entries but blueprint expects {len(want)}")
            ren = {old: new for old, new in zip(label_order, want) if old != new}
            if ren:
                tensor = tensor.relabels(ren)
        else:
            have = [str(lbl) for lbl in tensor.labels()]
            if sorted(have) != sorted(want):
                raise ValueError(f"Tensor {name!r} labels {list(tensor.labels())} don't match blueprint labels "
                                 f"{want} (as sets). Pass label_order to map them explicitly.")
            if have != want:
                tensor = tensor.transpose(tuple(have.index(lbl) for lbl in want))
        self._tensors[name] = tensor

    def put_tensors(self, mapping: dict) -> None:
        for name, tensor in mapping.items():
            self.put_tensor(name, tensor)

    def clear_tensors(self) -> None:
        self._tensors.clear()

    def is_ready(self) -> bool:
        return set(self._tensors) == set(self._names)

    def launch(self, optimize: str = "auto", *, pairwise: bool = False, precision=None):
        """Contract the network (netfile.py:468-528).  ``pairwise`` (no
        ORDER line) contracts in declaration order, pair by pair, instead of
        the one N-operand contraction whose result the reference empties
        when three or more operands contract different label sets."""
        if not self.is_ready():
            missing = set(self._names) - set(self._tensors)
            raise RuntimeError(f"Cannot launch: missing tensors {sorted(missing)}")
        if self._steps is not None:
            return self._launch_steps(self._steps, precision)
        if pairwise and len(self._names) > 2:
            steps, acc = [], self._names[0]
            for i, name in enumerate(self._names[1:]):
                steps.append((acc, name))
                acc = f"_{i}"
            return self._launch_steps(steps, precision)
        tensors = [self._tensors[n] for n in self._names]
        _, out_idx = _labels_to_subscripts(tensors, self._tout)
        return contract_with_subscripts(tensors, self._subscripts, out_idx, optimize, precision=precision)

    def _launch_steps(self, steps, precision):
        live = dict(self._tensors)
        for i, (a, b) in enumerate(steps):
            live[f"_{i}"] = contract(live.pop(a), live.pop(b), precision=precision)
        assert len(live) == 1, f"ORDER did not reduce to a single tensor: {list(live)}"
        out = next(iter(live.values()))
        if self._tout:
            have = [str(lbl) for lbl in out.labels()]
            if have != self._tout:
                out = out.transpose(tuple(have.index(lbl) for lbl in self._tout))
        return out

    def to_tensor_network(self) -> Any:
        """The filled blueprint as a ``TensorNetwork`` with legs of equal
        label connected (netfile.py:531-569)."""
        if not self.is_ready():
            missing = set(self._names) - set(self._tensors)
            raise RuntimeError(f"Cannot convert: missing tensors {sorted(missing)}")
        from tenax_b200.network import TensorNetwork

        tn = TensorNetwork(name="from_netfile")
        for name in self._names:
            tn.add_node(name, self._tensors[name])
        for i, a in enumerate(self._names):
            for b in self._names[i + 1:]:
                for lbl in sorted(set(self._labels[a]) & set(self._labels[b])):
                    try:
                        tn.connect(a, lbl, b, lbl)
                    except (ValueError, KeyError):
                        pass
        return tn


def from_netfile(source) -> NetworkBlueprint:
    """Same as ``NetworkBlueprint(source)`` (netfile.py:572-583)."""
    return NetworkBlueprint(source)
