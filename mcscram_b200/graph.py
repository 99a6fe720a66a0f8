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

    def edges(self):
        """Every input slot in gate order: (gate index, input node, position
        within the gate), int64 arrays of length sum(gate_in_count)."""
        cnt = self.gate_in_count.astype(np.int64)
        gid = np.repeat(np.arange(self.n_gates, dtype=np.int64), cnt)
        within = np.arange(int(cnt.sum()), dtype=np.int64) - np.repeat(np.cumsum(cnt) - cnt, cnt)
        pos = np.repeat(self.gate_in_begin.astype(np.int64), cnt) + within
        return gid, self.inputs[pos].astype(np.int64), within

    def layers(self) -> np.ndarray:
        """Depth of every gate: 1 + max depth of its gate inputs (basic events are 0),
        the LayeredTopologicalOrder of mcSCRAM src/preprocessor.cc:130-171.
        Computed by relaxation over all gates at once (as many sweeps as
        there are layers)."""
        nb, ng = self.n_be, self.n_gates
        depth = np.zeros(self.n_nodes, dtype=np.int64)
        if ng == 0:
            return depth
        gid, src, _ = self.edges()
        cnt = self.gate_in_count.astype(np.int64)
        has = cnt > 0
        starts = (np.cumsum(cnt) - cnt)[has]
        depth[nb:] = 1
        for _ in range(ng + 1):
            new = np.ones(ng, dtype=np.int64)
            if starts.size:
                new[has] = np.maximum.reduceat(depth[src], starts) + 1
            if np.array_equal(new, depth[nb:]):
                break
            depth[nb:] = new
        return depth

    def validate(self) -> None:
        nb = self.n_be
        bad = np.nonzero(self.gate_neg_count > self.gate_in_count)[0]
        if bad.size:
            raise ValueError(f"gate {int(bad[0])}: neg_count > in_count")
        if np.any(self.gate_in_begin.astype(np.int64) + self.gate_in_count > self.inputs.size):
            raise ValueError("gate input range outside the input array")
        gid, src, _ = self.edges()
        bad = np.nonzero(src >= nb + gid)[0]
        if bad.size:
            raise ValueError(f"gate {int(gid[bad[0]])}: inputs not topologically ordered")
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


def concat(graphs) -> "tuple[FlatGraph, np.ndarray, np.ndarray]":
    """Disjoint union of several graphs as one graph: the basic events of all
    graphs first, graph by graph, then their gates, graph by graph (each
    graph's gates stay in topological order and read only its own nodes).
    Basic event j of the union gets event index j and PDAG index 2 + j, so
    every event of the union draws from its own Philox counter stream; the
    tally list holds the root of every graph.  Returns (union, be_begin,
    roots): graph k owns basic events [be_begin[k], be_begin[k + 1]) and
    its top event is node roots[k]."""
    nbs = np.array([g.n_be for g in graphs], dtype=np.int64)
    ngs = np.array([g.n_gates for g in graphs], dtype=np.int64)
    nis = np.array([g.inputs.size for g in graphs], dtype=np.int64)
    be_begin = np.concatenate([[0], np.cumsum(nbs)])
    gate_begin = np.concatenate([[0], np.cumsum(ngs)])
    in_begin = np.concatenate([[0], np.cumsum(nis)])
    NB = int(be_begin[-1])
    inputs, begins, roots = [], [], []
    for k, g in enumerate(graphs):
        x = g.inputs.astype(np.int64)
        inputs.append(np.where(x < g.n_be, x + be_begin[k], x - g.n_be + NB + gate_begin[k]))
        begins.append(g.gate_in_begin.astype(np.int64) + in_begin[k])
        roots.append(g.root - g.n_be + NB + gate_begin[k])
    cat = lambda arrs, dt: np.concatenate(arrs).astype(dt) if arrs else np.zeros(0, dtype=dt)
    roots = np.array(roots, dtype=np.int64)
    u = FlatGraph(
        be_pdag_idx=np.arange(NB, dtype=np.int64) + 2,
        be_event_idx=np.arange(NB, dtype=np.uint32),
        be_threshold=cat([g.be_threshold for g in graphs], np.uint64),
        gate_op=cat([g.gate_op for g in graphs], np.uint8),
        gate_k=cat([g.gate_k for g in graphs], np.uint32),
        gate_in_begin=cat(begins, np.uint32),
        gate_in_count=cat([g.gate_in_count for g in graphs], np.uint32),
        gate_neg_count=cat([g.gate_neg_count for g in graphs], np.uint32),
        inputs=cat(inputs, np.uint32),
        tally_nodes=roots.astype(np.uint32),
        gate_pdag_idx=np.arange(int(gate_begin[-1]), dtype=np.int64) + 2 + NB,
        root=int(roots[-1]) if roots.size else -1,
        name=f"union-of-{len(graphs)}",
    )
    return u, be_begin, roots
