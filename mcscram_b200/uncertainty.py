"""Batched instances and uncertainty analysis (include/mcg_batch.h).

``Batch`` evaluates many (tree, threshold table) instances in one persistent
launch; ``uncertainty`` samples lognormal basic-event probabilities for every
draw of every tree and summarises P(top) per tree, mirroring
UncertaintyAnalyzer::Sample / CalculateStatistics (mcSCRAM
src/uncertainty_analysis.h:154-168, .cc:122-158).
"""
from __future__ import annotations

import ctypes as C
from typing import List, Optional, Sequence

import numpy as np

from . import _capi
from .graph import FlatGraph

UA_MEDIAN = 0
UA_MEAN = 1

_vp = C.c_void_p
_u32p = C.POINTER(C.c_uint32)
_u64p = C.POINTER(C.c_uint64)
_dp = C.POINTER(C.c_double)


class BatchInfo(C.Structure):
    _fields_ = [("n_trees", C.c_uint32), ("smem_slots", C.c_uint32), ("max_global_slots", C.c_uint32),
                ("grid_ctas", C.c_uint32), ("total_ops", C.c_uint64), ("launches", C.c_uint64),
                ("last_kernel_ms", C.c_double), ("instances_per_item", C.c_uint32)]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


class UaDesc(C.Structure):
    _fields_ = [("base_p", _dp), ("draws_per_tree", C.c_uint32), ("error_factor", C.c_double),
                ("level", C.c_double), ("parameterization", C.c_uint32), ("clip_max", C.c_double),
                ("seed", C.c_uint64), ("words_per_instance", C.c_uint64), ("iteration", C.c_uint32)]


class UaStats(C.Structure):
    _fields_ = [("mean", C.c_double), ("sigma", C.c_double), ("error_factor", C.c_double), ("ci_low", C.c_double),
                ("ci_high", C.c_double), ("p05", C.c_double), ("p50", C.c_double), ("p95", C.c_double),
                ("min", C.c_double), ("max", C.c_double)]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


_capi.register_signatures({
    "mcg_batch_create": (C.c_int, [C.POINTER(_capi.GraphDesc), C.c_uint32, C.POINTER(_capi.RunDesc),
                                   C.POINTER(_vp)]),
    "mcg_batch_destroy": (C.c_int, [_vp]),
    "mcg_batch_run": (C.c_int, [_vp, C.c_uint32, _u32p, _u64p, _u64p, C.c_uint64, C.c_uint32, C.c_uint64, _u64p]),
    "mcg_batch_info_get": (C.c_int, [_vp, C.POINTER(BatchInfo)]),
    "mcg_ua_run": (C.c_int, [_vp, C.POINTER(UaDesc), _dp, C.POINTER(UaStats), _u64p, _dp]),
})


class Batch:
    """Compiled programs of many trees; instances are (tree, thresholds)."""

    def __init__(self, trees: Sequence[FlatGraph], device: int = 0, ctas_per_sm: int = 0, smem_slots: int = 0,
                 stream: Optional[int] = None):
        self.lib = _capi.load()
        self.trees = list(trees)
        self._views = [_capi.GraphView(t) for t in self.trees]
        descs = (_capi.GraphDesc * len(self.trees))(*[v.desc for v in self._views])
        run = _capi.RunDesc(mode=_capi.MODE_FUSED, device=device, stream=C.c_void_p(stream) if stream else None,
                            ctas_per_sm=ctas_per_sm, smem_slots=smem_slots)
        self.h = _vp()
        _capi.check(self.lib.mcg_batch_create(descs, len(self.trees), C.byref(run), C.byref(self.h)))

    def close(self):
        if getattr(self, "h", None):
            self.lib.mcg_batch_destroy(self.h)
            self.h = None

    __del__ = close

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def run(self, inst_tree: Sequence[int], thresholds: Sequence[np.ndarray], iteration: int = 1,
            words_per_instance: int = 1 << 16) -> np.ndarray:
        """ones[i] of instance i (tree inst_tree[i], thresholds[i])."""
        inst_tree = np.ascontiguousarray(inst_tree, dtype=np.uint32)
        offs = np.zeros(len(inst_tree), dtype=np.uint64)
        acc = 0
        for i, t in enumerate(thresholds):
            offs[i] = acc
            acc += len(t)
        thr = np.ascontiguousarray(np.concatenate([np.asarray(t, np.uint64) for t in thresholds])
                                   if len(thresholds) else np.zeros(1, np.uint64), dtype=np.uint64)
        ones = np.zeros(len(inst_tree), dtype=np.uint64)
        p = lambda a, t: a.ctypes.data_as(C.POINTER(t))
        _capi.check(self.lib.mcg_batch_run(self.h, len(inst_tree), p(inst_tree, C.c_uint32), p(offs, C.c_uint64),
                                           p(thr, C.c_uint64), thr.size, iteration, words_per_instance,
                                           p(ones, C.c_uint64)))
        return ones

    def info(self) -> dict:
        i = BatchInfo()
        _capi.check(self.lib.mcg_batch_info_get(self.h, C.byref(i)))
        return i.as_dict()

    def uncertainty(self, base_p: Sequence[np.ndarray], draws_per_tree: int = 16, error_factor: float = 3.0,
                    level: float = 0.95, parameterization: int = UA_MEDIAN, clip_max: float = 0.5, seed: int = 372,
                    words_per_instance: int = 1 << 16, iteration: int = 1, return_thresholds: bool = False):
        """Lognormal draws of every basic-event probability for every tree,
        all instances in one launch.  Returns (p_top [n_trees, draws],
        per-tree stats list, kernel ms[, thresholds])."""
        base = np.ascontiguousarray(np.concatenate([np.asarray(b, np.float64) for b in base_p]), dtype=np.float64)
        n_trees = len(self.trees)
        d = UaDesc(base_p=base.ctypes.data_as(_dp), draws_per_tree=draws_per_tree, error_factor=error_factor,
                   level=level, parameterization=parameterization, clip_max=clip_max, seed=seed,
                   words_per_instance=words_per_instance, iteration=iteration)
        p_top = np.zeros(n_trees * draws_per_tree, dtype=np.float64)
        stats = (UaStats * n_trees)()
        n_thr = sum(t.n_be for t in self.trees) * draws_per_tree
        thr = np.zeros(max(n_thr, 1), dtype=np.uint64) if return_thresholds else None
        ms = C.c_double()
        _capi.check(self.lib.mcg_ua_run(self.h, C.byref(d), p_top.ctypes.data_as(_dp), stats,
                                        thr.ctypes.data_as(_u64p) if thr is not None else None, C.byref(ms)))
        out = (p_top.reshape(n_trees, draws_per_tree), [s.as_dict() for s in stats], ms.value)
        if return_thresholds:
            out = out + (thr[:n_thr],)
        return out
