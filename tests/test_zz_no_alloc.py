"""The fused pass that allocates no device memory (mcg_run_fused_noalloc).

Callers that cannot call cudaMalloc -- work enqueued while a CUDA graph is
being captured, processes whose device memory comes from their own pool or a
fixed budget, services that cannot take the implicit synchronisation of
cudaMalloc/cudaFree -- compile a program with mcg_compile, keep it in device
memory they already own, and call this entry point; the values the program
keeps outside shared memory go to a static device array instead of an
allocation.  This file checks, on the GPU and through the C ABI, that two
calls in a row give exactly the counts of the allocating entry point
(mcg_create / mcg_run), and that a program needing more scratch than the
static array holds is refused with a clear error.  It runs last so that a
failure here does not hide any other test's result."""
import ctypes as C

import numpy as np
import pytest

from mcscram_b200 import synth

pytestmark = pytest.mark.gpu


def _lib(capi):
    lib = capi.load()
    fn = lib.mcg_run_fused_noalloc
    fn.restype = C.c_int
    fn.argtypes = [C.c_void_p, C.c_uint64, C.c_uint32, C.c_uint32, C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32,
                   C.c_uint64, C.c_uint64, C.c_void_p]
    return lib


def _engine_ones(capi, g, it, n_it, wb, wc):
    with capi.Engine(g) as e:
        e.run(it, n_it, wb, wc)
        return e.tallies()[0]


def test_noalloc_matches_allocating_entry_point(capi, gpu):
    import torch
    lib = _lib(capi)
    g = synth.config1()
    info, ops = capi.compile_program(g, 16)
    assert info["global_slots"] > 0  # some values live in the static scratch
    # inputs and outputs in device memory the caller owns
    d_ops = torch.from_numpy(ops.view(np.int32).copy()).cuda()
    d_ones = torch.zeros(int(g.tally_nodes.size), dtype=torch.int64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    for it, n_it, wb, wc in [(1, 1, 0, 16384), (3, 2, 777, 70001)]:
        d_ones.zero_()
        rc = lib.mcg_run_fused_noalloc(d_ops.data_ptr(), int(info["n_ops"]), info["smem_slots"],
                                       info["global_slots"], d_ones.data_ptr(), int(g.tally_nodes.size), it, n_it,
                                       wb, wc, stream)
        assert rc == capi.MCG_OK, lib.mcg_last_error()
        torch.cuda.synchronize()
        got = d_ones.cpu().numpy().astype(np.uint64)
        expect = _engine_ones(capi, g, it, n_it, wb, wc)
        assert np.array_equal(got, expect), (it, n_it, wb, wc)


def _wide_graph(n_gates: int):
    """n_gates two-input gates over their own basic events, every gate tallied:
    a program with few live values and more tallies than shared memory holds."""
    from mcscram_b200.graph import AND, OR, FlatGraph, probability_threshold
    n_be = 2 * n_gates
    rng = np.random.default_rng(7)
    return FlatGraph(
        be_pdag_idx=np.arange(n_be) + 2, be_event_idx=np.arange(n_be),
        be_threshold=probability_threshold(rng.uniform(0.05, 0.6, n_be)),
        gate_op=np.where(np.arange(n_gates) % 2 == 0, AND, OR), gate_k=np.zeros(n_gates),
        gate_in_begin=2 * np.arange(n_gates), gate_in_count=np.full(n_gates, 2),
        gate_neg_count=(np.arange(n_gates) % 3 == 0).astype(np.uint32), inputs=np.arange(n_be),
        tally_nodes=n_be + np.arange(n_gates))


def _noalloc_ones(capi, lib, g, budget, runs):
    import torch
    info, ops = capi.compile_program(g, budget)
    d_ops = torch.from_numpy(ops.view(np.int32).copy()).cuda()
    d_ones = torch.zeros(int(g.tally_nodes.size), dtype=torch.int64, device="cuda")
    out = []
    for it, n_it, wb, wc in runs:
        d_ones.zero_()
        rc = lib.mcg_run_fused_noalloc(d_ops.data_ptr(), int(info["n_ops"]), info["smem_slots"],
                                       info["global_slots"], d_ones.data_ptr(), int(g.tally_nodes.size), it, n_it,
                                       wb, wc, torch.cuda.current_stream().cuda_stream)
        assert rc == capi.MCG_OK, lib.mcg_last_error()
        torch.cuda.synchronize()
        out.append(d_ones.cpu().numpy().astype(np.uint64))
    return info, out


def test_noalloc_several_launch_chunks(capi, gpu):
    """More words than one launch chunk (2^21), from an odd first word."""
    lib = _lib(capi)
    g = synth.config1()
    runs = [(2, 1, 12345, (1 << 21) + 54321), (5, 1, (1 << 22) + 3, (1 << 21) * 2 + 1)]
    info, got = _noalloc_ones(capi, lib, g, 16, runs)
    assert info["global_slots"] > 0
    for (it, n_it, wb, wc), ones in zip(runs, got):
        assert np.array_equal(ones, _engine_ones(capi, g, it, n_it, wb, wc)), (it, wb, wc)


def test_noalloc_tallies_outside_shared_memory(capi, gpu):
    """16,000 tallied gates (128 KB of counters) do not fit next to the value
    slots in a CTA's shared memory, so the kernel adds them in global memory."""
    lib = _lib(capi)
    g = _wide_graph(16000)
    runs = [(1, 1, 0, 9000), (4, 3, 100, 5000)]
    _, got = _noalloc_ones(capi, lib, g, 64, runs)
    for (it, n_it, wb, wc), ones in zip(runs, got):
        assert np.array_equal(ones, _engine_ones(capi, g, it, n_it, wb, wc)), (it, wb, wc)
        assert int(ones.sum()) > 0


def test_noalloc_after_an_engine_with_a_smaller_program(capi, gpu):
    """An engine of the same kernel (two CTAs per SM) created with a small
    program before the call must not lower the kernel's shared-memory limit
    below what the call's program needs."""
    lib = _lib(capi)
    small = synth.small_tree(5, n_be=12, n_gates=6)
    small = small.with_tallies([small.root])
    with capi.Engine(small, ctas_per_sm=2) as e:
        e.run(1, 1, 0, 4096)
        e.tallies()
    g = synth.config1()
    runs = [(1, 1, 0, 16384), (2, 1, 5, 3000)]
    info, got = _noalloc_ones(capi, lib, g, 40, runs)
    assert info["smem_slots"] > 16
    for (it, n_it, wb, wc), ones in zip(runs, got):
        assert np.array_equal(ones, _engine_ones(capi, g, it, n_it, wb, wc)), (it, wb, wc)


def test_noalloc_refuses_oversized_scratch(capi, gpu):
    import torch
    lib = _lib(capi)
    g = synth.config2()
    info, ops = capi.compile_program(g, 0)  # every value in global scratch
    d_ops = torch.from_numpy(ops.view(np.int32).copy()).cuda()
    d_ones = torch.zeros(int(g.tally_nodes.size), dtype=torch.int64, device="cuda")
    rc = lib.mcg_run_fused_noalloc(d_ops.data_ptr(), int(info["n_ops"]), info["smem_slots"], info["global_slots"],
                                   d_ones.data_ptr(), int(g.tally_nodes.size), 1, 1, 0, 4096, None)
    assert rc == capi.MCG_ERR_INVALID
    assert "static scratch" in lib.mcg_last_error().decode()
    torch.cuda.synchronize()
    assert int(d_ones.sum()) == 0  # nothing was launched
