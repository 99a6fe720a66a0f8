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
