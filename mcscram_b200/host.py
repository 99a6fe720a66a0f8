"""Python bindings of the host layer (include/mcg_host.h).

``Pdag`` builds the caller-side PDAG; ``LayerManager`` mirrors the
reference's ``scram::mc::queue::layer_manager``; ``compute_tallies`` mirrors
``ProbabilityAnalyzer<DirectEval>::ComputeTallies`` (mcSCRAM
src/mc/core/probability_analysis.cc:98-209).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Dict, Iterable, List, Optional, Sequence

import numpy as np

from . import _capi
from .graph import FlatGraph

POLICY_BAYES = 0
POLICY_WALD = 1


class Tally(C.Structure):
    _fields_ = [
        ("index", C.c_int32), ("num_one_bits", C.c_uint64), ("total_bits", C.c_uint64), ("mean", C.c_double),
        ("std_err", C.c_double), ("ci", C.c_double * 4), ("linear_epsilon", C.c_double),
        ("linear_target_epsilon", C.c_double), ("linear_target_trials", C.c_uint64), ("log10_epsilon", C.c_double),
        ("log10_target_epsilon", C.c_double), ("log10_target_trials", C.c_uint64),
    ]

    def as_dict(self) -> dict:
        d = {n: getattr(self, n) for n, _ in self._fields_}
        d["ci"] = list(self.ci)
        return d


class Settings(C.Structure):
    _fields_ = [
        ("num_trials", C.c_uint64), ("early_stop", C.c_uint32), ("policy", C.c_uint32),
        ("ci_confidence", C.c_double), ("ci_rel_margin_error", C.c_double), ("ci_burnin_trials", C.c_double),
        ("overhead_ratio", C.c_double), ("oracle_p", C.c_double), ("max_words_per_iteration", C.c_uint64),
        ("pipelined", C.c_uint32),
    ]

    @classmethod
    def default(cls, **kw) -> "Settings":
        s = cls()
        _capi.check(_lib().mcg_settings_default(C.byref(s)))
        for k, v in kw.items():
            setattr(s, k, v)
        return s


class Report(C.Structure):
    _fields_ = [
        ("burn_in_steps", C.c_uint64), ("steps", C.c_uint64), ("passes", C.c_uint64), ("trials", C.c_uint64),
        ("projected_trials", C.c_uint64), ("epsilon_converged", C.c_uint32), ("log10_converged", C.c_uint32),
        ("iteration_limit_reached", C.c_uint32), ("epsilon", C.c_double), ("target_epsilon", C.c_double),
        ("epsilon_log10", C.c_double), ("target_epsilon_log10", C.c_double), ("info_gain_bits", C.c_double),
        ("seconds", C.c_double),
    ]

    def as_dict(self) -> dict:
        return {n: getattr(self, n) for n, _ in self._fields_}


_i32p = C.POINTER(C.c_int32)
_u32p = C.POINTER(C.c_uint32)
_u64p = C.POINTER(C.c_uint64)
_u8p = C.POINTER(C.c_uint8)
_vp = C.c_void_p

_capi.register_signatures({
    "mcg_settings_default": (C.c_int, [C.POINTER(Settings)]),
    "mcg_pdag_create": (C.c_int, [C.POINTER(_vp)]),
    "mcg_pdag_destroy": (C.c_int, [_vp]),
    "mcg_pdag_add_variable": (C.c_int, [_vp, C.c_int32, C.c_double]),
    "mcg_pdag_add_gate": (C.c_int, [_vp, C.c_int32, C.c_uint8, C.c_uint32, _i32p, C.c_uint32]),
    "mcg_pdag_set_root": (C.c_int, [_vp, C.c_int32]),
    "mcg_pdag_set_probability": (C.c_int, [_vp, C.c_int32, C.c_double]),
    "mcg_pdag_event_order": (C.c_int, [_vp, _i32p, C.c_uint32, _u32p]),
    "mcg_pdag_flat_sizes": (C.c_int, [_vp, _u32p, _u32p, _u64p]),
    "mcg_pdag_flatten": (C.c_int, [_vp, _i32p, C.c_uint32, _i32p, _u32p, _u64p, _i32p, _u8p, _u32p, _u32p, _u32p,
                                   _u32p, _u32p, _u32p]),
    "mcg_manager_create": (C.c_int, [_vp, C.c_uint64, _i32p, C.c_uint32, C.c_double, C.POINTER(_capi.RunDesc),
                                     C.c_uint64, C.POINTER(_vp)]),
    "mcg_manager_destroy": (C.c_int, [_vp]),
    "mcg_manager_single_pass": (C.c_int, [_vp]),
    "mcg_manager_pass": (C.c_int, [_vp, C.c_uint64]),
    "mcg_manager_single_pass_and_tally": (C.c_int, [_vp, C.c_int32, C.POINTER(Tally)]),
    "mcg_manager_pass_wait_collect": (C.c_int, [_vp, C.c_uint64, C.c_uint64, C.POINTER(Tally), C.c_uint32]),
    "mcg_manager_collect_tallies": (C.c_int, [_vp, C.POINTER(Tally), C.c_uint32]),
    "mcg_manager_node_count": (C.c_int, [_vp, _u64p]),
    "mcg_manager_shape": (C.c_int, [_vp, _u64p, _u64p, _u64p]),
    "mcg_manager_engine": (C.c_int, [_vp, C.POINTER(_vp)]),
    "mcg_run_to_convergence": (C.c_int, [_vp, C.POINTER(Settings), C.POINTER(Tally), C.c_uint32,
                                         C.POINTER(Report)]),
    "mcg_compute_tallies": (C.c_int, [_vp, C.POINTER(Settings), _i32p, C.c_uint32, C.POINTER(_capi.RunDesc),
                                      C.POINTER(Tally), C.POINTER(Report)]),
    "mcg_normal_quantile_two_sided": (C.c_double, [C.c_double]),
    "mcg_beta_quantile": (C.c_double, [C.c_double, C.c_double, C.c_double]),
    "mcg_sample_shape": (C.c_int, [C.c_uint64, C.c_uint64, _u64p, _u64p, _u64p]),
})


def _lib():
    return _capi.load()


def _arr(values, ctype):
    a = (ctype * max(len(values), 1))(*values)
    return a


class Pdag:
    """Caller-side PDAG: variables (index >= 2) and gates with signed arguments."""

    def __init__(self):
        self.h = _vp()
        _capi.check(_lib().mcg_pdag_create(C.byref(self.h)))

    def __del__(self):
        if getattr(self, "h", None):
            _lib().mcg_pdag_destroy(self.h)
            self.h = None

    def add_variable(self, index: int, probability: float) -> "Pdag":
        _capi.check(_lib().mcg_pdag_add_variable(self.h, index, probability))
        return self

    def add_gate(self, index: int, connective: int, args: Sequence[int], min_number: int = 0) -> "Pdag":
        a = _arr(list(args), C.c_int32)
        _capi.check(_lib().mcg_pdag_add_gate(self.h, index, connective, min_number, a, len(args)))
        return self

    def set_root(self, index: int) -> "Pdag":
        _capi.check(_lib().mcg_pdag_set_root(self.h, index))
        return self

    def set_probability(self, index: int, p: float) -> None:
        _capi.check(_lib().mcg_pdag_set_probability(self.h, index, p))

    def event_order(self) -> List[int]:
        """PDAG indices of the basic events in layer-0 block order (event_idx = position)."""
        n = C.c_uint32()
        _capi.check(_lib().mcg_pdag_event_order(self.h, None, 0, C.byref(n)))
        out = (C.c_int32 * max(n.value, 1))()
        _capi.check(_lib().mcg_pdag_event_order(self.h, out, n.value, C.byref(n)))
        return list(out[: n.value])

    def flatten(self, tally_indices: Sequence[int] = ()) -> FlatGraph:
        nb, ng, ni = C.c_uint32(), C.c_uint32(), C.c_uint64()
        _capi.check(_lib().mcg_pdag_flat_sizes(self.h, C.byref(nb), C.byref(ng), C.byref(ni)))
        nb, ng, ni = nb.value, ng.value, ni.value
        a = {
            "be_pdag_idx": np.zeros(max(nb, 1), np.int32), "be_event_idx": np.zeros(max(nb, 1), np.uint32),
            "be_threshold": np.zeros(max(nb, 1), np.uint64), "gate_pdag_idx": np.zeros(max(ng, 1), np.int32),
            "gate_op": np.zeros(max(ng, 1), np.uint8), "gate_k": np.zeros(max(ng, 1), np.uint32),
            "gate_in_begin": np.zeros(max(ng, 1), np.uint32), "gate_in_count": np.zeros(max(ng, 1), np.uint32),
            "gate_neg_count": np.zeros(max(ng, 1), np.uint32), "inputs": np.zeros(max(ni, 1), np.uint32),
            "tally_nodes": np.zeros(max(len(tally_indices), 1), np.uint32),
        }
        t = _arr(list(tally_indices), C.c_int32)
        p = lambda k, ct: a[k].ctypes.data_as(C.POINTER(ct))
        _capi.check(_lib().mcg_pdag_flatten(
            self.h, t, len(tally_indices), p("be_pdag_idx", C.c_int32), p("be_event_idx", C.c_uint32),
            p("be_threshold", C.c_uint64), p("gate_pdag_idx", C.c_int32), p("gate_op", C.c_uint8),
            p("gate_k", C.c_uint32), p("gate_in_begin", C.c_uint32), p("gate_in_count", C.c_uint32),
            p("gate_neg_count", C.c_uint32), p("inputs", C.c_uint32), p("tally_nodes", C.c_uint32)))
        sizes = {"be_pdag_idx": nb, "be_event_idx": nb, "be_threshold": nb, "gate_pdag_idx": ng, "gate_op": ng,
                 "gate_k": ng, "gate_in_begin": ng, "gate_in_count": ng, "gate_neg_count": ng, "inputs": ni,
                 "tally_nodes": len(tally_indices)}
        kw = {k: v[: sizes[k]] for k, v in a.items()}
        return FlatGraph(**kw)

    @classmethod
    def from_flat(cls, g: FlatGraph) -> "Pdag":
        """A PDAG with the flat graph's nodes (variable index = pdag_idx, gate
        index = gate_pdag_idx), root = g.root; probabilities from the thresholds."""
        p = cls()
        probs = g.be_prob if g.be_prob is not None else g.quantised_probabilities()
        for e in range(g.n_be):
            p.add_variable(int(g.be_pdag_idx[e]), float(probs[e]))
        node_index = list(map(int, g.be_pdag_idx)) + list(map(int, g.gate_pdag_idx))
        for gi in range(g.n_gates):
            ins = g.gate_inputs(gi)
            off = int(g.gate_in_count[gi] - g.gate_neg_count[gi])
            args = [node_index[c] if i < off else -node_index[c] for i, c in enumerate(ins)]
            p.add_gate(int(g.gate_pdag_idx[gi]), int(g.gate_op[gi]), args, int(g.gate_k[gi]))
        p.set_root(node_index[g.root])
        return p


class LayerManager:
    """Mirror of layer_manager(pdag, num_trials, to_tally, overhead_ratio)."""

    def __init__(self, pdag: Pdag, num_trials: int, to_tally: Iterable[int], overhead_ratio: float = 0.05,
                 mode: int = _capi.MODE_AUTO, device: int = 0, max_words_per_iteration: int = 0, **run_kw):
        self.pdag = pdag
        self.order = list(dict.fromkeys(int(x) for x in to_tally))
        run = _capi.RunDesc(mode=mode, device=device, **run_kw)
        idx = _arr(self.order, C.c_int32)
        self.h = _vp()
        _capi.check(_lib().mcg_manager_create(pdag.h, num_trials, idx, len(self.order), overhead_ratio,
                                              C.byref(run), max_words_per_iteration, C.byref(self.h)))

    def close(self):
        if getattr(self, "h", None):
            _lib().mcg_manager_destroy(self.h)
            self.h = None

    __del__ = close

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _tallies(self):
        return (Tally * max(len(self.order), 1))()

    def single_pass(self) -> None:
        _capi.check(_lib().mcg_manager_single_pass(self.h))

    def pass_(self, count: int) -> None:
        _capi.check(_lib().mcg_manager_pass(self.h, count))

    def single_pass_and_tally(self, index: int) -> dict:
        t = Tally()
        _capi.check(_lib().mcg_manager_single_pass_and_tally(self.h, index, C.byref(t)))
        return t.as_dict()

    def pass_wait_collect(self, total_passes: int = 1, passes_between_waits: int = 0) -> Dict[int, dict]:
        out = self._tallies()
        _capi.check(_lib().mcg_manager_pass_wait_collect(self.h, total_passes, passes_between_waits, out,
                                                         len(self.order)))
        return {t.index: t.as_dict() for t in out[: len(self.order)]}

    def collect_tallies(self) -> Dict[int, dict]:
        out = self._tallies()
        _capi.check(_lib().mcg_manager_collect_tallies(self.h, out, len(self.order)))
        return {t.index: t.as_dict() for t in out[: len(self.order)]}

    def node_count(self) -> int:
        n = C.c_uint64()
        _capi.check(_lib().mcg_manager_node_count(self.h, C.byref(n)))
        return n.value

    def shape(self):
        bs, bpb, it = C.c_uint64(), C.c_uint64(), C.c_uint64()
        _capi.check(_lib().mcg_manager_shape(self.h, C.byref(bs), C.byref(bpb), C.byref(it)))
        return {"batch_size": bs.value, "bitpacks_per_batch": bpb.value, "total_iterations": it.value}

    def run_to_convergence(self, settings: Optional[Settings] = None):
        s = settings or Settings.default()
        out = self._tallies()
        rep = Report()
        _capi.check(_lib().mcg_run_to_convergence(self.h, C.byref(s), out, len(self.order), C.byref(rep)))
        return {t.index: t.as_dict() for t in out[: len(self.order)]}, rep.as_dict()


def compute_tallies(pdag: Pdag, settings: Optional[Settings] = None, watch: Sequence[int] = (), device: int = 0,
                    mode: int = _capi.MODE_AUTO):
    """Root tally first, then the watched nodes; plus the convergence report."""
    s = settings or Settings.default()
    w = _arr(list(watch), C.c_int32)
    out = (Tally * (len(watch) + 1))()
    rep = Report()
    run = _capi.RunDesc(mode=mode, device=device)
    _capi.check(_lib().mcg_compute_tallies(pdag.h, C.byref(s), w, len(watch), C.byref(run), out, C.byref(rep)))
    return [t.as_dict() for t in out], rep.as_dict()


def normal_quantile_two_sided(confidence: float) -> float:
    return float(_lib().mcg_normal_quantile_two_sided(confidence))


def beta_quantile(a: float, b: float, q: float) -> float:
    return float(_lib().mcg_beta_quantile(a, b, q))


def sample_shape(num_trials: int, max_words_per_iteration: int = 0):
    w, it, r = C.c_uint64(), C.c_uint64(), C.c_uint64()
    _capi.check(_lib().mcg_sample_shape(num_trials, max_words_per_iteration, C.byref(w), C.byref(it), C.byref(r)))
    return {"words_per_iteration": w.value, "total_iterations": it.value, "num_trials": r.value}
