"""TEST INFRASTRUCTURE ONLY: Python access to the CPU oracle libraries.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module, and only as the checker (or the timed CPU baseline); the product
package mcscram_b200 never imports it.

  liboracle.so       plain-C restatement of the reference's MC dataflow
                     (mc_oracle.c, philox_oracle.h)
  _ref/libref_mc.so  the same dataflow drawing every basic-event word from
                     the reference's own philox128.h compiled from its sources
  libbdd_oracle.so   exact FP64 top-event probability by BDD (bdd_oracle.cc)
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path
from typing import Optional

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"
REF_LIB = HERE / "_ref" / "libref_mc.so"
BDD_LIB = HERE / "libbdd_oracle.so"

_u32p = C.POINTER(C.c_uint32)
_i32p = C.POINTER(C.c_int32)
_u64p = C.POINTER(C.c_uint64)
_u8p = C.POINTER(C.c_uint8)


class OrcGraph(C.Structure):
    _fields_ = [
        ("n_be", C.c_uint32), ("n_gates", C.c_uint32),
        ("be_pdag_idx", _i32p), ("be_event_idx", _u32p), ("be_threshold", _u64p),
        ("gate_op", _u8p), ("gate_k", _u32p), ("gate_in_begin", _u32p), ("gate_in_count", _u32p),
        ("gate_neg_count", _u32p), ("inputs", _u32p),
    ]


def build(force: bool = False) -> None:
    """Runs oracle/Makefile (builds _ref/ only where the reference sources exist)."""
    if force or not LIB.exists() or not BDD_LIB.exists():
        subprocess.run(["make", "-C", str(HERE), "all"], check=True, stdout=subprocess.DEVNULL)


_libs: dict = {}


def _load(path: Path) -> C.CDLL:
    if path not in _libs:
        if not path.exists():
            build()
        lib = C.CDLL(str(path))
        if hasattr(lib, "orc_word"):
            lib.orc_word.restype = C.c_uint64
            lib.orc_word.argtypes = [C.c_uint32] * 4 + [C.c_uint64]
            lib.orc_be_word_at.restype = C.c_uint64
            lib.orc_be_word_at.argtypes = [C.c_uint32] * 4 + [C.c_uint64]
            lib.orc_eval_words.restype = C.c_int
            lib.orc_eval_words.argtypes = [C.POINTER(OrcGraph), C.c_uint32, C.c_uint64, C.c_uint64, _u64p, C.c_int]
            lib.orc_tallies.restype = C.c_int
            lib.orc_tallies.argtypes = [C.POINTER(OrcGraph), C.c_uint32, C.c_uint32, C.c_uint64, C.c_uint64,
                                        C.c_uint32, _u32p, _u64p, C.c_int]
            lib.orc_max_threads.restype = C.c_int
        if hasattr(lib, "bdd_top_probability"):
            lib.bdd_top_probability.restype = C.c_int
            lib.bdd_top_probability.argtypes = [C.c_uint32, C.c_uint32, _u8p, _u32p, _u32p, _u32p, _u32p, _u32p,
                                                C.POINTER(C.c_double), C.c_uint32, C.c_uint64,
                                                C.POINTER(C.c_double), _u64p]
        _libs[path] = lib
    return _libs[path]


def lib(reference: bool = False) -> C.CDLL:
    return _load(REF_LIB if reference else LIB)


def has_reference_build() -> bool:
    return REF_LIB.exists()


def _p(a, t):
    return a.ctypes.data_as(C.POINTER(t))


class _View:
    def __init__(self, g):
        self.keep = [g.be_pdag_idx, g.be_event_idx, g.be_threshold, g.gate_op, g.gate_k, g.gate_in_begin,
                     g.gate_in_count, g.gate_neg_count, g.inputs]
        self.s = OrcGraph(g.n_be, g.n_gates, _p(g.be_pdag_idx, C.c_int32), _p(g.be_event_idx, C.c_uint32),
                          _p(g.be_threshold, C.c_uint64), _p(g.gate_op, C.c_uint8), _p(g.gate_k, C.c_uint32),
                          _p(g.gate_in_begin, C.c_uint32), _p(g.gate_in_count, C.c_uint32),
                          _p(g.gate_neg_count, C.c_uint32), _p(g.inputs, C.c_uint32))


def word(c0: int, c1: int, c2: int, c3: int, thr: int, reference: bool = False) -> int:
    """One packed word for counter base {c0, c1, c2, c3}."""
    return int(lib(reference).orc_word(c0, c1, c2, c3, thr))


def be_word(pdag_idx: int, event_idx: int, sample_idx: int, iteration: int, thr: int, reference: bool = False) -> int:
    return int(lib(reference).orc_be_word_at(pdag_idx, event_idx, sample_idx, iteration, thr))


def eval_words(g, iteration: int, word_begin: int, n_words: int, reference: bool = False,
               threads: int = 0) -> np.ndarray:
    """All node words, shape [n_nodes, n_words]."""
    out = np.zeros((g.n_nodes, n_words), dtype=np.uint64)
    v = _View(g)
    rc = lib(reference).orc_eval_words(C.byref(v.s), iteration, word_begin, n_words, _p(out, C.c_uint64), threads)
    if rc != 0:
        raise ValueError(f"oracle rejected the graph ({rc})")
    return out


def tallies(g, iteration_first: int, n_iterations: int, word_begin: int, n_words: int,
            tally_nodes: Optional[np.ndarray] = None, reference: bool = False, threads: int = 0) -> np.ndarray:
    nodes = np.ascontiguousarray(g.tally_nodes if tally_nodes is None else tally_nodes, dtype=np.uint32)
    ones = np.zeros(max(nodes.size, 1), dtype=np.uint64)
    v = _View(g)
    rc = lib(reference).orc_tallies(C.byref(v.s), iteration_first, n_iterations, word_begin, n_words, nodes.size,
                                    _p(nodes, C.c_uint32), _p(ones, C.c_uint64), threads)
    if rc != 0:
        raise ValueError(f"oracle rejected the graph ({rc})")
    return ones[: nodes.size]


def max_threads() -> int:
    return int(lib().orc_max_threads())


def bdd_probability(g, p: Optional[np.ndarray] = None, root: Optional[int] = None,
                    max_nodes: int = 20_000_000) -> float:
    """Exact P(root) with basic-event probabilities p (default: the quantised
    thresholds / 2^32 the sampler actually uses)."""
    L = _load(BDD_LIB)
    p = np.ascontiguousarray(g.quantised_probabilities() if p is None else p, dtype=np.float64)
    root = g.root if root is None else root
    out = C.c_double()
    nodes = C.c_uint64()
    rc = L.bdd_top_probability(g.n_be, g.n_gates, _p(g.gate_op, C.c_uint8), _p(g.gate_k, C.c_uint32),
                               _p(g.gate_in_begin, C.c_uint32), _p(g.gate_in_count, C.c_uint32),
                               _p(g.gate_neg_count, C.c_uint32), _p(g.inputs, C.c_uint32), _p(p, C.c_double),
                               root, max_nodes, C.byref(out), C.byref(nodes))
    if rc == -2:
        raise MemoryError(f"BDD exceeded {max_nodes} nodes")
    if rc != 0:
        raise ValueError(f"BDD oracle rejected the graph ({rc})")
    return float(out.value)
