"""Monte Carlo importance factors (mcg_importance_factors in include/mcg_host.h).

One pass tallies the top event and, for every requested basic event x, the
conjunction "top and x"; the Birnbaum factor follows as
P(top | x=1) - P(top | x=0), and the critical, diagnosis, risk-achievement
and risk-reduction factors from it by the relations of the reference's exact
analysis (mcSCRAM src/importance_analysis.cc:50-56).
"""
from __future__ import annotations

import ctypes as C
from typing import List, Optional, Sequence

import numpy as np

from . import _capi
from .graph import FlatGraph


class ImportanceFactor(C.Structure):
    _fields_ = [("event", C.c_uint32), ("samples", C.c_uint64), ("p", C.c_double), ("p_top", C.c_double),
                ("p_joint", C.c_double), ("p_top_given_1", C.c_double), ("p_top_given_0", C.c_double),
                ("mif", C.c_double), ("cif", C.c_double), ("dif", C.c_double), ("raw", C.c_double),
                ("rrw", C.c_double)]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


_capi.register_signatures({
    "mcg_importance_factors": (C.c_int, [C.POINTER(_capi.GraphDesc), C.POINTER(C.c_uint32), C.c_uint32,
                                         C.POINTER(_capi.RunDesc), C.c_uint32, C.c_uint64,
                                         C.POINTER(ImportanceFactor)]),
    "mcg_importance_from_conditionals": (C.c_int, [C.c_double, C.c_double, C.c_double, C.c_double,
                                                   C.POINTER(ImportanceFactor)]),
})


def factors_from_conditionals(p: float, p_top: float, p_top_given_1: float, p_top_given_0: float) -> dict:
    """The factors of one event from exact (or externally estimated)
    conditionals, by the relations mcg_importance_factors applies; host only."""
    out = ImportanceFactor()
    _capi.check(_capi.load().mcg_importance_from_conditionals(p, p_top, p_top_given_1, p_top_given_0, C.byref(out)))
    return out.as_dict()


def importance_factors(g: FlatGraph, events: Optional[Sequence[int]] = None, words: int = 1 << 20,
                       iteration: int = 1, mode: int = _capi.MODE_STRIP, device: int = 0) -> List[dict]:
    """Factors of `events` (flattened basic-event ids; all when None) for the
    top event g.root from words * 64 samples."""
    lib = _capi.load()
    gt = g.with_tallies([g.root])
    view = _capi.GraphView(gt)
    ev = np.ascontiguousarray(np.arange(g.n_be) if events is None else events, dtype=np.uint32)
    out = (ImportanceFactor * max(len(ev), 1))()
    run = _capi.RunDesc(mode=mode, device=device)
    _capi.check(lib.mcg_importance_factors(C.byref(view.desc), ev.ctypes.data_as(C.POINTER(C.c_uint32)), len(ev),
                                           C.byref(run), iteration, words, out))
    return [out[i].as_dict() for i in range(len(ev))]
