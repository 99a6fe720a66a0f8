"""Learned importance sampling for rare top events (include/mcg_is.h).

* ``event_features`` -- 16 structural features per basic event (log p,
  fan-out, depths, parent gate-type mix, ATLEAST tightness, path
  connectives, ...), the network's input.
* ``ImportanceSampler`` -- the bit-packed sampler with proposal thresholds
  and FP64 likelihood-ratio estimator (mcg_is_run).
* ``ProposalMLP`` -- 16 -> 64 -> 64 -> 1 network trained on the GPU
  (mcg_mlp_*), BF16 weights with FP32 accumulation.
* ``cross_entropy`` -- the cross-entropy method: sample with the current
  proposal, take the likelihood-weighted failure frequency of every event as
  the next target, fit the network to it, repeat.
* ``estimate`` -- the final IS estimate with an effective-sample-size check
  that falls back to the plain sampler when the weights collapse.
"""
from __future__ import annotations

import ctypes as C
import time
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

from . import _capi
from .graph import AND, ATLEAST, OR, XOR, FlatGraph, probability_threshold

N_FEATURES = 16
N_PARAMS = 16 * 64 + 64 + 64 * 64 + 64 + 64 + 1
TWO_32 = float(1 << 32)

_vp = C.c_void_p
_u64p = C.POINTER(C.c_uint64)
_fp = C.POINTER(C.c_float)
_dp = C.POINTER(C.c_double)


class IsResult(C.Structure):
    _fields_ = [("samples", C.c_uint64), ("hits", C.c_uint64), ("sum_w", C.c_double), ("sum_w2", C.c_double),
                ("estimate", C.c_double), ("std_err", C.c_double), ("rel_err", C.c_double), ("ess", C.c_double),
                ("max_log_w", C.c_double), ("kernel_ms", C.c_double)]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


_capi.register_signatures({
    "mcg_is_create": (C.c_int, [C.POINTER(_capi.GraphDesc), C.POINTER(_capi.RunDesc), C.POINTER(_vp)]),
    "mcg_is_destroy": (C.c_int, [_vp]),
    "mcg_is_run": (C.c_int, [_vp, _u64p, C.c_uint32, C.c_uint64, C.c_uint64, C.POINTER(IsResult), _dp]),
    "mcg_mlp_create": (C.c_int, [C.c_int32, C.c_uint64, C.POINTER(_vp)]),
    "mcg_mlp_destroy": (C.c_int, [_vp]),
    "mcg_mlp_set_params": (C.c_int, [_vp, _fp]),
    "mcg_mlp_get_params": (C.c_int, [_vp, _fp]),
    "mcg_mlp_forward": (C.c_int, [_vp, _fp, C.c_uint32, _fp]),
    "mcg_mlp_grad": (C.c_int, [_vp, _fp, _fp, _fp, C.c_uint32, _fp, _fp]),
    "mcg_mlp_train": (C.c_int, [_vp, _fp, _fp, _fp, C.c_uint32, C.c_uint32, C.c_float, _fp]),
})


def _p(a, t):
    return a.ctypes.data_as(C.POINTER(t))


def event_features(g: FlatGraph) -> np.ndarray:
    """16 features per basic event, float32 [n_be, 16]."""
    nb, ng = g.n_be, g.n_gates
    depth = g.layers()
    L = max(int(depth.max()), 1)
    parents = [[] for _ in range(g.n_nodes)]
    for gi in range(ng):
        for c in g.gate_inputs(gi):
            parents[int(c)].append(gi)
    p = np.clip(g.quantised_probabilities(), 1e-12, 1.0)
    logp = np.log10(p)
    # path from every gate to the top through its first parent
    up_and = np.zeros(ng)
    up_or = np.zeros(ng)
    up_len = np.zeros(ng)
    for gi in range(ng - 1, -1, -1):
        node = nb + gi
        ps = parents[node]
        if ps:
            q = ps[0]
            up_and[gi] = up_and[q] + (g.gate_op[q] == AND)
            up_or[gi] = up_or[q] + (g.gate_op[q] == OR)
            up_len[gi] = up_len[q] + 1
    feats = np.zeros((nb, N_FEATURES), dtype=np.float32)
    for e in range(nb):
        ps = parents[e]
        feats[e, 0] = (logp[e] + 4.0) / 2.0
        feats[e, 1] = len(ps) / 4.0
        if ps:
            d = [depth[nb + q] for q in ps]
            ops = [int(g.gate_op[q]) for q in ps]
            fanin = [int(g.gate_in_count[q]) for q in ps]
            feats[e, 2] = min(d) / L
            feats[e, 3] = max(d) / L
            feats[e, 4] = np.mean([o == AND for o in ops])
            feats[e, 5] = np.mean([o == OR for o in ops])
            feats[e, 6] = np.mean([o == ATLEAST for o in ops])
            feats[e, 7] = np.mean(fanin) / 8.0
            kn = [int(g.gate_k[q]) / max(int(g.gate_in_count[q]), 1) for q in ps if g.gate_op[q] == ATLEAST]
            feats[e, 8] = np.mean(kn) if kn else 0.0
            q0 = ps[0]
            sib = [int(c) for c in g.gate_inputs(q0) if int(c) != e]
            feats[e, 9] = (len(sib)) / 8.0
            sib_be = [logp[c] for c in sib if c < nb]
            feats[e, 10] = (np.mean(sib_be) + 4.0) / 2.0 if sib_be else 0.0
            feats[e, 11] = np.mean([c >= nb for c in sib]) if sib else 0.0
            feats[e, 12] = float(max(d) == L)
            feats[e, 13] = up_and[q0] / max(up_len[q0] + 1, 1)
            feats[e, 14] = up_or[q0] / max(up_len[q0] + 1, 1)
        feats[e, 15] = 1.0
    return feats


class ImportanceSampler:
    """Proposal sampling with FP64 likelihood ratios over one tree (root tallied)."""

    def __init__(self, g: FlatGraph, device: int = 0, chunk_words: int = 0):
        self.lib = _capi.load()
        self.graph = g.with_tallies([g.root])
        self._view = _capi.GraphView(self.graph)
        run = _capi.RunDesc(mode=_capi.MODE_STAGED, device=device, layered_max_words=chunk_words)
        self.h = _vp()
        _capi.check(self.lib.mcg_is_create(C.byref(self._view.desc), C.byref(run), C.byref(self.h)))

    def close(self):
        if getattr(self, "h", None):
            self.lib.mcg_is_destroy(self.h)
            self.h = None

    __del__ = close

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def proposal_thresholds(self, q: np.ndarray) -> np.ndarray:
        """Thresholds for proposal probabilities q; events with a constant
        nominal word (p = 0 or 1) keep their nominal threshold."""
        thr = probability_threshold(np.clip(q, 0.0, 1.0))
        thr = np.clip(thr, 1, (1 << 32) - 1).astype(np.uint64)
        fixed = (self.graph.be_threshold == 0) | (self.graph.be_threshold >= (1 << 32))
        thr[fixed] = self.graph.be_threshold[fixed]
        return np.ascontiguousarray(thr, dtype=np.uint64)

    def run(self, q_thresholds: np.ndarray, iteration: int = 1, word_begin: int = 0, word_count: int = 1 << 20,
            ce: bool = False):
        q_thresholds = np.ascontiguousarray(q_thresholds, dtype=np.uint64)
        res = IsResult()
        ce_num = np.zeros(max(self.graph.n_be, 1), dtype=np.float64) if ce else None
        _capi.check(self.lib.mcg_is_run(self.h, _p(q_thresholds, C.c_uint64), iteration, word_begin, word_count,
                                        C.byref(res), _p(ce_num, C.c_double) if ce else None))
        out = res.as_dict()
        if ce:
            out["ce_num"] = ce_num[: self.graph.n_be]
        return out


class ProposalMLP:
    """16 -> 64 -> 64 -> 1 sigmoid network on the GPU."""

    def __init__(self, device: int = 0, seed: int = 7):
        self.lib = _capi.load()
        self.h = _vp()
        _capi.check(self.lib.mcg_mlp_create(device, seed, C.byref(self.h)))

    def close(self):
        if getattr(self, "h", None):
            self.lib.mcg_mlp_destroy(self.h)
            self.h = None

    __del__ = close

    def params(self) -> np.ndarray:
        out = np.zeros(N_PARAMS, dtype=np.float32)
        _capi.check(self.lib.mcg_mlp_get_params(self.h, _p(out, C.c_float)))
        return out

    def set_params(self, params: np.ndarray) -> None:
        params = np.ascontiguousarray(params, dtype=np.float32)
        _capi.check(self.lib.mcg_mlp_set_params(self.h, _p(params, C.c_float)))

    def forward(self, feats: np.ndarray) -> np.ndarray:
        feats = np.ascontiguousarray(feats, dtype=np.float32)
        q = np.zeros(feats.shape[0], dtype=np.float32)
        _capi.check(self.lib.mcg_mlp_forward(self.h, _p(feats, C.c_float), feats.shape[0], _p(q, C.c_float)))
        return q

    def grad(self, feats, targets, weights=None):
        feats = np.ascontiguousarray(feats, dtype=np.float32)
        targets = np.ascontiguousarray(targets, dtype=np.float32)
        w = None if weights is None else np.ascontiguousarray(weights, dtype=np.float32)
        g = np.zeros(N_PARAMS, dtype=np.float32)
        loss = C.c_float()
        _capi.check(self.lib.mcg_mlp_grad(self.h, _p(feats, C.c_float), _p(targets, C.c_float),
                                          _p(w, C.c_float) if w is not None else None, feats.shape[0],
                                          _p(g, C.c_float), C.byref(loss)))
        return g, float(loss.value)

    def train(self, feats, targets, weights=None, steps: int = 200, lr: float = 3e-3) -> float:
        feats = np.ascontiguousarray(feats, dtype=np.float32)
        targets = np.ascontiguousarray(targets, dtype=np.float32)
        w = None if weights is None else np.ascontiguousarray(weights, dtype=np.float32)
        loss = C.c_float()
        _capi.check(self.lib.mcg_mlp_train(self.h, _p(feats, C.c_float), _p(targets, C.c_float),
                                           _p(w, C.c_float) if w is not None else None, feats.shape[0], steps, lr,
                                           C.byref(loss)))
        return float(loss.value)


@dataclass
class CeHistory:
    rounds: List[dict] = field(default_factory=list)
    seconds: float = 0.0
    gpu_ms: float = 0.0


def initial_proposal(sampler: ImportanceSampler, p: np.ndarray, probe_words: int = 1 << 16,
                     min_hits: int = 200, max_scale: float = 1e6):
    """Uniform inflation q = min(p * s, 0.5), doubling s until a probe run of the
    plain (biased) sampler sees at least min_hits top-event failures."""
    s = 1.0
    gpu_ms = 0.0
    while True:
        q = np.minimum(p * s, 0.5)
        r = sampler.run(sampler.proposal_thresholds(q), iteration=1, word_begin=0, word_count=probe_words)
        gpu_ms += r["kernel_ms"]
        if r["hits"] >= min_hits or s >= max_scale:
            return q, s, gpu_ms
        s *= 2.0


def cross_entropy(g: FlatGraph, rounds: int = 5, words_per_round: int = 1 << 20, mlp: Optional[ProposalMLP] = None,
                  smoothing: float = 0.7, train_steps: int = 300, lr: float = 3e-3, q_max: float = 0.5,
                  device: int = 0, sampler: Optional[ImportanceSampler] = None):
    """Cross-entropy training of the proposal.  Each round samples
    words_per_round * 64 samples with the current proposal (passes 2, 3, ...,
    so rounds use fresh random numbers), sets the target of event i to the
    likelihood-weighted frequency of x_i = 1 among top-event failures,
    smooths it with the current proposal and fits the network to it.
    Returns (q, mlp, history)."""
    t0 = time.perf_counter()
    own = sampler is None
    sampler = sampler or ImportanceSampler(g, device=device)
    p = g.quantised_probabilities()
    feats = event_features(g)
    mlp = mlp or ProposalMLP(device=device)
    hist = CeHistory()
    q, scale, ms = initial_proposal(sampler, p)
    hist.gpu_ms += ms
    hist.rounds.append({"round": 0, "scale": scale})
    for r in range(rounds):
        res = sampler.run(sampler.proposal_thresholds(q), iteration=2 + r, word_begin=0,
                          word_count=words_per_round, ce=True)
        hist.gpu_ms += res["kernel_ms"]
        if res["sum_w"] <= 0 or res["hits"] == 0:
            hist.rounds.append({"round": r + 1, "hits": 0})
            break
        target = np.clip(res["ce_num"] / res["sum_w"], 1e-7, q_max)
        target = smoothing * target + (1.0 - smoothing) * q
        loss = mlp.train(feats, target.astype(np.float32), steps=train_steps, lr=lr)
        q = np.clip(mlp.forward(feats).astype(np.float64), 1e-7, q_max)
        hist.rounds.append({"round": r + 1, "hits": res["hits"], "estimate": res["estimate"],
                            "rel_err": res["rel_err"], "ess": res["ess"], "loss": loss})
    hist.seconds = time.perf_counter() - t0
    if own:
        sampler.close()
    return q, mlp, hist


def estimate(sampler: ImportanceSampler, q: np.ndarray, target_rel_err: float = 0.05, words_per_batch: int = 1 << 20,
             max_words: int = 1 << 28, iteration: int = 100, ess_floor: float = 50.0):
    """Runs batches until the relative standard error at 95% confidence
    (1.96 * std_err / estimate) is at most target_rel_err.  Returns the
    pooled result; 'fallback' is set when the effective sample size stays
    below ess_floor (the proposal is unreliable and the plain sampler should
    be used instead)."""
    thr = sampler.proposal_thresholds(q)
    n = sw = sw2 = 0.0
    hits = 0
    gpu_ms = 0.0
    used = 0
    b = 0
    while used < max_words:
        r = sampler.run(thr, iteration=iteration, word_begin=used, word_count=words_per_batch)
        gpu_ms += r["kernel_ms"]
        used += words_per_batch
        b += 1
        n += r["samples"]
        sw += r["sum_w"]
        sw2 += r["sum_w2"]
        hits += r["hits"]
        est = sw / n
        var = max(sw2 / n - est * est, 0.0)
        se = np.sqrt(var / max(n - 1, 1))
        rel95 = 1.96 * se / est if est > 0 else np.inf
        ess = sw * sw / sw2 if sw2 > 0 else 0.0
        if rel95 <= target_rel_err and ess >= ess_floor:
            break
    return {"estimate": est, "std_err": se, "rel_err95": rel95, "samples": int(n), "hits": hits, "ess": ess,
            "batches": b, "gpu_ms": gpu_ms, "fallback": bool(ess < ess_floor)}
