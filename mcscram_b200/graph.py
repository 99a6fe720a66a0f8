"""Flattened PDAG container shared by the engine bindings, generator and tests.

Node ids: ``[0, n_be)`` are basic events, ``[n_be, n_be + n_gates)`` gates in
a topological order (every input id of gate ``g`` is smaller than
``n_be + g``).  Gate ``g`` reads ``inputs[in_begin[g]:in_begin[g] + in_count[g]]``
and the last ``neg_count[g]`` of those are complemented, the layout of the
reference's gate blocks (mcSCRAM src/mc/event/node.h:234-252, 655-662).
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Optional

import numpy as np

# core::Connective values (mcSCRAM src/pdag.h:265-276).
AND, OR, ATLEAST, XOR, NOT, NAND, NOR, NULL = range(8)
CONNECTIVE_NAMES = {AND: "and", OR: "or", ATLEAST: "atleast", XOR: "xor", NOT: "not",
                    NAND: "nand", NOR: "nor", NULL: "null"}

TWO_32 = float(1 << 32)


def probability_threshold(p) -> np.ndarray:
    """``(uint64)(p * 2^32)`` truncated, as the reference's basic-event block
    computes it (mcSCRAM src/mc/event/node.h:372-376)."""
    p = np.asarray(p, dtype=np.float64)
    if np.any(p < 0) or np.any(p > 1):
        raise ValueError("probabilities must lie in [0, 1]")
    return (p * TWO_32).astype(np.uint64)


@dataclass
class FlatGraph:
    be_pdag_idx: np.ndarray
    be_event_idx: np.ndarray
    be_threshold: np.ndarray
    gate_op: np.ndarray
    gate_k: np.ndarray
    gate_in_begin: np.ndarray
    gate_in_count: np.ndarray
    gate_neg_count: np.ndarray
    inputs: np.ndarray
    tally_nodes: np.ndarray
    gate_pdag_idx: Optional[np.ndarray] = None
    be_prob: Optional[np.ndarray] = None
    root: int = -1
    name: str = "graph"
    meta: dict = field(default_factory=dict)

    def __post_init__(self):
        self.be_pdag_idx = np.ascontiguousarray(self.be_pdag_idx, dtype=np.int32)
        self.be_event_idx = np.ascontiguousarray(self.be_event_idx, dtype=np.uint32)
        self.be_threshold = np.ascontiguousarray(self.be_threshold, dtype=np.uint64)
        self.gate_op = np.ascontiguousarray(self.gate_op, dtype=np.uint8)
        self.gate_k = np.ascontiguousarray(self.gate_k, dtype=np.uint32)
        self.gate_in_begin = np.ascontiguousarray(self.gate_in_begin, dtype=np.uint32)
        self.gate_in_count = np.ascontiguousarray(self.gate_in_count, dtype=np.uint32)
        self.gate_neg_count = np.ascontiguousarray(self.gate_neg_count, dtype=np.uint32)
        self.inputs = np.ascontiguousarray(self.inputs, dtype=np.uint32)
        self.tally_nodes = np.ascontiguousarray(self.tally_nodes, dtype=np.uint32)
        if self.gate_pdag_idx is None:
            self.gate_pdag_idx = np.arange(self.n_gates, dtype=np.int32) + 2 + self.n_be
        self.gate_pdag_idx = np.ascontiguousarray(self.gate_pdag_idx, dtype=np.int32)
        if self.root < 0:
            self.root = self.n_nodes - 1

    @property
    def n_be(self) -> int:
        return int(self.be_threshold.shape[0])

    @property
    def n_gates(self) -> int:
        return int(self.gate_op.shape[0])

    @property
    def n_nodes(self) -> int:
        return self.n_be + self.n_gates

    def gate_inputs(self, g: int) -> np.ndarray:
        b = int(self.gate_in_begin[g])
        return self.inputs[b:b + int(self.gate_in_count[g])]

    def with_tallies(self, nodes) -> "FlatGraph":
        import copy
        out = copy.copy(self)
        out.tally_nodes = np.ascontiguousarray(nodes, dtype=np.uint32)
        return out

    def with_thresholds(self, thr) -> "FlatGraph":
        import copy
        out = copy.copy(self)
        out.be_threshold = np.ascontiguousarray(thr, dtype=np.uint64)
        return out

    def quantised_probabilities(self) -> np.ndarray:
        """p~ = threshold / 2^32: the probability the sampler actually draws."""
        return self.be_threshold.astype(np.float64) / TWO_32

    def layers(self) -> np.ndarray:
        """Depth of every gate: 1 + max depth of its gate inputs (basic events are 0),
        the LayeredTopologicalOrder of mcSCRAM src/preprocessor.cc:130-171."""
        depth = np.zeros(self.n_nodes, dtype=np.int64)
        nb = self.n_be
        for g in range(self.n_gates):
            ins = self.gate_inputs(g)
            depth[nb + g] = 1 + (int(depth[ins].max()) if ins.size else 0)
        return depth

    def validate(self) -> None:
        nb = self.n_be
        for g in range(self.n_gates):
            if self.gate_neg_count[g] > self.gate_in_count[g]:
                raise ValueError(f"gate {g}: neg_count > in_count")
            ins = self.gate_inputs(g)
            if ins.size and int(ins.max()) >= nb + g:
                raise ValueError(f"gate {g}: inputs not topologically ordered")
        if np.any(self.be_threshold > (1 << 32)):
            raise ValueError("threshold above 2^32")
        if self.tally_nodes.size and int(self.tally_nodes.max()) >= self.n_nodes:
            raise ValueError("tally node out of range")

    def summary(self) -> dict:
        ops = np.bincount(self.gate_op, minlength=8)
        fanout = np.bincount(self.inputs, minlength=self.n_nodes)
        return {
            "n_be": self.n_be,
            "n_gates": self.n_gates,
            "n_inputs": int(self.inputs.size),
            "n_layers": int(self.layers().max()) if self.n_gates else 0,
            "ops": {CONNECTIVE_NAMES[i]: int(ops[i]) for i in range(8) if ops[i]},
            "frac_nodes_fanout_ge2": float((fanout >= 2).mean()) if self.n_nodes else 0.0,
            "frac_be_fanout_ge2": float((fanout[: self.n_be] >= 2).mean()) if self.n_be else 0.0,
            "n_tally": int(self.tally_nodes.size),
        }
