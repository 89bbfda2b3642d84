"""Minimal tensor-network container for the ``dmrg()`` call site.

Holds the nodes and labelled bonds the way tenax's ``TensorNetwork``
(network/network.py:51-507) does for MPS/MPO inputs and the DMRG result;
graph-wide contraction is not part of this package.
"""

from __future__ import annotations


class TensorNetwork:
    def __init__(self, name: str = ""):
        self.name = name
        self._nodes: dict = {}
        self._edges: list = []

    def add_node(self, node_id, tensor) -> None:
        if node_id in self._nodes:
            raise ValueError(f"Node {node_id!r} already exists")
        self._nodes[node_id] = tensor

    def replace_tensor(self, node_id, tensor) -> None:
        if node_id not in self._nodes:
            raise KeyError(f"Node {node_id!r} not found")
        self._nodes[node_id] = tensor

    def get_tensor(self, node_id):
        if node_id not in self._nodes:
            raise KeyError(f"Node {node_id!r} not found")
        return self._nodes[node_id]

    def connect(self, node_a, label_a, node_b, label_b) -> None:
        for n, l in ((node_a, label_a), (node_b, label_b)):
            if l not in self.get_tensor(n).labels():
                raise ValueError(f"Node {n!r} has no leg labelled {l!r}")
        self._edges.append((node_a, label_a, node_b, label_b))

    def node_ids(self) -> list:
        return list(self._nodes)

    def n_nodes(self) -> int:
        return len(self._nodes)

    def n_edges(self) -> int:
        return len(self._edges)

    def neighbors(self, node_id) -> list:
        out = []
        for a, _, b, _ in self._edges:
            if a == node_id:
                out.append(b)
            elif b == node_id:
                out.append(a)
        return out

    def __repr__(self):
        return f"TensorNetwork(name={self.name!r}, nodes={self.n_nodes()}, edges={self.n_edges()})"
