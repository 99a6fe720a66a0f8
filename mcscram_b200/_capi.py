"""ctypes bindings of libmcg.so (include/mcg.h).

The shared library is loaded from this package directory.  If it is missing
or cannot be loaded, ``load()`` raises: there is no fallback implementation.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path
from typing import Optional

import numpy as np

from .graph import FlatGraph

LIB_PATH = Path(__file__).resolve().parent / "libmcg.so"

MCG_OK = 0
MCG_ERR_INVALID = 1
MCG_ERR_CUDA = 2
MCG_ERR_OOM = 3
MCG_ERR_TIMEOUT = 4
MCG_ERR_STATE = 5
MCG_ERR_NO_DEVICE = 6

MODE_AUTO = 0
MODE_LAYERED = 1
MODE_STAGED = 2
MODE_STRIP = 3
MODE_FUSED = 4
MODES = {"auto": MODE_AUTO, "fused": MODE_FUSED, "layered": MODE_LAYERED, "staged": MODE_STAGED,
         "strip": MODE_STRIP}
MODE_NAMES = {v: k for k, v in MODES.items()}

_u32p = C.POINTER(C.c_uint32)
_i32p = C.POINTER(C.c_int32)
_u64p = C.POINTER(C.c_uint64)
_u8p = C.POINTER(C.c_uint8)


class GraphDesc(C.Structure):
    _fields_ = [
        ("n_be", C.c_uint32),
        ("n_gates", C.c_uint32),
        ("be_pdag_idx", _i32p),
        ("be_event_idx", _u32p),
        ("be_threshold", _u64p),
        ("gate_pdag_idx", _i32p),
        ("gate_op", _u8p),
        ("gate_k", _u32p),
        ("gate_in_begin", _u32p),
        ("gate_in_count", _u32p),
        ("gate_neg_count", _u32p),
        ("inputs", _u32p),
        ("n_inputs", C.c_uint64),
        ("n_tally", C.c_uint32),
        ("tally_nodes", _u32p),
    ]


class RunDesc(C.Structure):
    _fields_ = [
        ("mode", C.c_uint32),
        ("device", C.c_int32),
        ("stream", C.c_void_p),
        ("block_threads", C.c_uint32),
        ("smem_slots", C.c_uint32),
        ("ctas_per_sm", C.c_uint32),
        ("chunk_words", C.c_uint64),
        ("layered_max_words", C.c_uint64),
        ("sampler_blocks_per_sm", C.c_uint32),
        ("tune_pass_words", C.c_uint64),
    ]


class ProgramInfo(C.Structure):
    _fields_ = [
        ("n_ops", C.c_uint64),
        ("smem_slots", C.c_uint32),
        ("global_slots", C.c_uint32),
        ("max_live", C.c_uint32),
        ("block_threads", C.c_uint32),
        ("grid_ctas", C.c_uint32),
        ("scratch_bytes", C.c_uint64),
        ("smem_bytes", C.c_uint32),
        ("n_inline_be", C.c_uint32),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class TuneChoice(C.Structure):
    _fields_ = [
        ("mode", C.c_uint32),
        ("ctas_per_sm", C.c_uint32),
        ("layered_max_words", C.c_uint64),
        ("words_per_second", C.c_double),
        ("probe_words", C.c_uint64),
        ("key", C.c_uint64),
        ("from_cache", C.c_uint32),
        ("candidates", C.c_uint32),
    ]

    def as_dict(self) -> dict:
        d = {name: getattr(self, name) for name, _ in self._fields_}
        d["mode_name"] = MODE_NAMES.get(self.mode, str(self.mode))
        return d


# double probe(void *user, const mcg_graph_desc *graph, const mcg_run_desc *candidate, uint64_t probe_words)
TUNE_PROBE = C.CFUNCTYPE(C.c_double, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64)


class McgError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"mcg error {code}: {msg}")
        self.code = code


_lib: Optional[C.CDLL] = None

_SIGNATURES = {
    "mcg_create": (C.c_int, [C.POINTER(GraphDesc), C.POINTER(RunDesc), C.POINTER(C.c_void_p)]),
    "mcg_destroy": (C.c_int, [C.c_void_p]),
    "mcg_run": (C.c_int, [C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint64, C.c_uint64]),
    "mcg_synchronize": (C.c_int, [C.c_void_p]),
    "mcg_trim_memory": (C.c_int, [C.c_int]),
    "mcg_read_tallies": (C.c_int, [C.c_void_p, _u64p, _u64p]),
    "mcg_tally_device_ptr": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "mcg_set_tallies": (C.c_int, [C.c_void_p, _u64p, C.c_uint64]),
    "mcg_reset_tallies": (C.c_int, [C.c_void_p]),
    "mcg_dump_words": (C.c_int, [C.c_void_p, C.c_uint32, C.c_uint64, C.c_uint64, _u64p]),
    "mcg_program_info_get": (C.c_int, [C.c_void_p, C.POINTER(ProgramInfo)]),
    "mcg_compile": (C.c_int, [C.POINTER(GraphDesc), C.c_uint32, C.c_uint32, C.POINTER(ProgramInfo), _u32p,
                              C.c_uint64]),
    "mcg_launch_count": (C.c_int, [C.c_void_p, _u64p]),
    "mcg_time_runs": (C.c_int, [C.c_void_p, C.c_uint32, C.c_uint64, C.c_uint64, C.c_uint32, C.POINTER(C.c_double)]),
    "mcg_sampler_peak": (C.c_int, [C.c_int32, C.c_uint64, C.c_uint64, C.c_uint32, C.POINTER(C.c_double)]),
    "mcg_sampler_peak_shared": (C.c_int, [C.c_int32, C.c_uint64, C.c_uint64, C.c_uint32, C.c_uint32,
                                          C.POINTER(C.c_double)]),
    "mcg_profile_sampler": (C.c_int, [C.c_void_p, C.c_int32]),
    "mcg_profile_sampler_read": (C.c_int, [C.c_void_p, _u64p, C.POINTER(C.c_double)]),
    "mcg_tune": (C.c_int, [C.POINTER(GraphDesc), C.POINTER(RunDesc), C.c_uint64, C.c_void_p, C.c_void_p,
                           C.POINTER(TuneChoice)]),
    "mcg_tune_set_cache_file": (C.c_int, [C.c_char_p]),
    "mcg_tune_forget": (C.c_int, []),
    "mcg_engine_launch_shape": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]),
    "mcg_last_error": (C.c_char_p, []),
    "mcg_version": (C.c_char_p, []),
}


def load() -> C.CDLL:
    """Loads libmcg.so (building it first if the toolkit is here and it is absent)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        from . import build as _build
        _build.build()
    lib = C.CDLL(str(LIB_PATH))
    for name, (res, args) in _SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    for name, (res, args) in _EXTRA_SIGNATURES.items():
        if hasattr(lib, name):
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
    _lib = lib
    return lib


_EXTRA_SIGNATURES: dict = {}


def register_signatures(sigs: dict) -> None:
    """Lets other binding modules add their entry points before or after load()."""
    _EXTRA_SIGNATURES.update(sigs)
    if _lib is not None:
        for name, (res, args) in sigs.items():
            fn = getattr(_lib, name)
            fn.restype = res
            fn.argtypes = args


def check(status: int) -> None:
    if status != MCG_OK:
        msg = load().mcg_last_error().decode(errors="replace")
        raise McgError(status, msg)


def _ptr(a: np.ndarray, ctype):
    return a.ctypes.data_as(C.POINTER(ctype))


class GraphView:
    """Keeps the numpy arrays of a FlatGraph alive while a GraphDesc points at them."""

    def __init__(self, g: FlatGraph):
        g.validate()
        self.g = g
        self._keep = [g.be_pdag_idx, g.be_event_idx, g.be_threshold, g.gate_pdag_idx, g.gate_op, g.gate_k,
                      g.gate_in_begin, g.gate_in_count, g.gate_neg_count, g.inputs, g.tally_nodes]
        self.desc = GraphDesc(
            n_be=g.n_be, n_gates=g.n_gates,
            be_pdag_idx=_ptr(g.be_pdag_idx, C.c_int32), be_event_idx=_ptr(g.be_event_idx, C.c_uint32),
            be_threshold=_ptr(g.be_threshold, C.c_uint64), gate_pdag_idx=_ptr(g.gate_pdag_idx, C.c_int32),
            gate_op=_ptr(g.gate_op, C.c_uint8), gate_k=_ptr(g.gate_k, C.c_uint32),
            gate_in_begin=_ptr(g.gate_in_begin, C.c_uint32), gate_in_count=_ptr(g.gate_in_count, C.c_uint32),
            gate_neg_count=_ptr(g.gate_neg_count, C.c_uint32), inputs=_ptr(g.inputs, C.c_uint32),
            n_inputs=int(g.inputs.size), n_tally=int(g.tally_nodes.size),
            tally_nodes=_ptr(g.tally_nodes, C.c_uint32))


def compile_program(g: FlatGraph, smem_slot_budget: int = 64, variable_thresholds: bool = False):
    """Host-only compilation of the fused program: (info dict, ops array [n_ops, 4] uint32)."""
    lib = load()
    view = GraphView(g)
    info = ProgramInfo()
    flags = 1 if variable_thresholds else 0
    check(lib.mcg_compile(C.byref(view.desc), smem_slot_budget, flags, C.byref(info), None, 0))
    ops = np.zeros((info.n_ops, 4), dtype=np.uint32)
    check(lib.mcg_compile(C.byref(view.desc), smem_slot_budget, flags, C.byref(info), _ptr(ops, C.c_uint32),
                          info.n_ops))
    return info.as_dict(), ops


class Engine:
    """One device engine over a flattened PDAG (wraps mcg_create ... mcg_destroy)."""

    def __init__(self, g: FlatGraph, mode: int = MODE_FUSED, device: int = 0, stream: Optional[int] = None,
                 smem_slots: int = 0, ctas_per_sm: int = 0, chunk_words: int = 0, layered_max_words: int = 0,
                 sampler_blocks_per_sm: int = 0, tune_pass_words: int = 0):
        self.lib = load()
        self.graph = g
        self._view = GraphView(g)
        run = RunDesc(mode=mode, device=device, stream=C.c_void_p(stream) if stream else None, block_threads=0,
                      smem_slots=smem_slots, ctas_per_sm=ctas_per_sm, chunk_words=chunk_words,
                      layered_max_words=layered_max_words, sampler_blocks_per_sm=sampler_blocks_per_sm,
                      tune_pass_words=tune_pass_words)
        h = C.c_void_p()
        check(self.lib.mcg_create(C.byref(self._view.desc), C.byref(run), C.byref(h)))
        self.handle = h

    def close(self):
        if getattr(self, "handle", None):
            self.lib.mcg_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def n_tally(self) -> int:
        return int(self.graph.tally_nodes.size)

    def run(self, iteration_first: int, n_iterations: int, word_begin: int, word_count: int) -> None:
        check(self.lib.mcg_run(self.handle, iteration_first, n_iterations, word_begin, word_count))

    def synchronize(self) -> None:
        check(self.lib.mcg_synchronize(self.handle))

    def tallies(self):
        ones = np.zeros(max(self.n_tally, 1), dtype=np.uint64)
        total = C.c_uint64()
        check(self.lib.mcg_read_tallies(self.handle, _ptr(ones, C.c_uint64), C.byref(total)))
        return ones[: self.n_tally], int(total.value)

    def set_tallies(self, ones: np.ndarray, total_bits: int) -> None:
        ones = np.ascontiguousarray(ones, dtype=np.uint64)
        check(self.lib.mcg_set_tallies(self.handle, _ptr(ones, C.c_uint64), total_bits))

    def tally_device_ptr(self) -> int:
        p = C.c_void_p()
        check(self.lib.mcg_tally_device_ptr(self.handle, C.byref(p)))
        return int(p.value or 0)

    def reset_tallies(self) -> None:
        check(self.lib.mcg_reset_tallies(self.handle))

    def dump_words(self, iteration: int, word_begin: int, n_words: int) -> np.ndarray:
        out = np.zeros((self.graph.n_nodes, n_words), dtype=np.uint64)
        check(self.lib.mcg_dump_words(self.handle, iteration, word_begin, n_words, _ptr(out, C.c_uint64)))
        return out

    def program_info(self) -> dict:
        info = ProgramInfo()
        check(self.lib.mcg_program_info_get(self.handle, C.byref(info)))
        return info.as_dict()

    def launch_count(self) -> int:
        n = C.c_uint64()
        check(self.lib.mcg_launch_count(self.handle, C.byref(n)))
        return int(n.value)

    def profile_sampler(self, enable: bool = True) -> None:
        check(self.lib.mcg_profile_sampler(self.handle, 1 if enable else 0))

    def profile_sampler_read(self):
        n = C.c_uint64()
        ms = C.c_double()
        check(self.lib.mcg_profile_sampler_read(self.handle, C.byref(n), C.byref(ms)))
        return int(n.value), float(ms.value)

    def launch_shape(self):
        """(mode, CTAs per SM) the engine runs with (the tuner's choice under MODE_AUTO)."""
        mode, ctas = C.c_uint32(), C.c_uint32()
        check(self.lib.mcg_engine_launch_shape(self.handle, C.byref(mode), C.byref(ctas)))
        return int(mode.value), int(ctas.value)

    def time_runs(self, iteration_first: int, word_begin: int, word_count: int, repeats: int) -> float:
        ms = C.c_double()
        check(self.lib.mcg_time_runs(self.handle, iteration_first, word_begin, word_count, repeats, C.byref(ms)))
        return float(ms.value)


def tune(g: FlatGraph, pass_words: int = 0, device: int = 0, probe=None) -> dict:
    """The launch shape mcg_tune picks for g's shape on `device` (cached per
    shape and device).  `probe`, when given, is called as
    probe(mode, ctas_per_sm, probe_words) -> basic-event words per second
    instead of timing passes on the GPU."""
    lib = load()
    view = GraphView(g)
    run = RunDesc(mode=MODE_AUTO, device=device)
    out = TuneChoice()
    cb = None
    if probe is not None:
        def _probe(user, graph, cand, words):
            c = C.cast(cand, C.POINTER(RunDesc)).contents
            return float(probe(int(c.mode), int(c.ctas_per_sm), int(words)))
        cb = TUNE_PROBE(_probe)
    check(lib.mcg_tune(C.byref(view.desc), C.byref(run), pass_words, C.cast(cb, C.c_void_p) if cb else None, None,
                       C.byref(out)))
    return out.as_dict()


def tune_set_cache_file(path: str) -> None:
    """Cache file of the tuner for later calls ("" = memory only)."""
    check(load().mcg_tune_set_cache_file(str(path).encode()))


def tune_forget() -> None:
    """Drops the tuner's in-memory entries (its file stays)."""
    check(load().mcg_tune_forget())


def trim_memory(device: int = 0) -> None:
    """Frees the work buffers destroyed engines left on `device` for the next
    engine (mcg_trim_memory)."""
    check(load().mcg_trim_memory(device))


def sampler_peak(n_events: int = 256, n_words: int = 1 << 21, repeats: int = 5, device: int = 0) -> float:
    """Basic-event words per second of the register-only sampler kernel."""
    lib = load()
    r = C.c_double()
    check(lib.mcg_sampler_peak(device, n_events, n_words, repeats, C.byref(r)))
    return float(r.value)


def sampler_peak_shared(instances: int, n_events: int = 256, n_words: int = 1 << 21, repeats: int = 5,
                        device: int = 0) -> float:
    """Instance words per second of the register-only sampler of batches that
    evaluate `instances` (1 or 4) instances per Philox evaluation."""
    lib = load()
    r = C.c_double()
    check(lib.mcg_sampler_peak_shared(device, n_events, n_words, repeats, instances, C.byref(r)))
    return float(r.value)


def version() -> str:
    return load().mcg_version().decode()
