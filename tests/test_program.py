"""The fused program compiler checked on the CPU: the compiled program,
executed by a plain emulator over oracle words, must reproduce every tallied
node word exactly, for any shared-memory slot budget (including none, which
moves every value to global scratch)."""
import numpy as np
import pytest

from mcscram_b200 import synth
from mcscram_b200.graph import ATLEAST, NOT, NULL, OR, FlatGraph, probability_threshold
from tests.program_emulator import emulate


def check_program(capi, oracle_mod, g, budget, W=64, iteration=1, word_begin=0):
    info, ops = capi.compile_program(g, budget)
    assert info["smem_slots"] <= max(budget, 0)
    words = oracle_mod.eval_words(g, iteration, word_begin, W)
    vals, ones = emulate(ops, g, words, int(g.tally_nodes.size))
    for i, node in enumerate(g.tally_nodes):
        assert vals[i] is not None, f"tally {i} never counted"
        assert np.array_equal(vals[i], words[node]), f"tally {i} (node {node}) differs, budget {budget}"
    return info


@pytest.mark.parametrize("budget", [0, 1, 2, 3, 5, 64])
@pytest.mark.parametrize("seed", range(5))
def test_small_dags(capi, oracle_mod, seed, budget):
    g = synth.small_tree(seed, n_be=40, n_gates=24, n_layers=5, p_range=(0.05, 0.6))
    g.gate_neg_count = np.array([1 if (gi % 3 == 0 and g.gate_in_count[gi] > 1) else 0
                                 for gi in range(g.n_gates)], dtype=np.uint32)
    info = check_program(capi, oracle_mod, g, budget)
    if budget == 0:
        assert info["smem_slots"] == 0


@pytest.mark.parametrize("budget", [0, 4, 48])
def test_config1(capi, oracle_mod, budget):
    info = check_program(capi, oracle_mod, synth.config1(), budget)
    assert info["n_inline_be"] > 0


def test_config2_program_shape(capi):
    g = synth.config2()
    info, ops = capi.compile_program(g, 44)
    # every basic event is sampled exactly once per word column
    codes = ops[:, 0] & 0xF
    assert int(((codes == 1) | (codes == 2)).sum()) == g.n_be
    assert int((codes == 8).sum()) == g.n_gates  # one tally per gate
    assert info["max_live"] >= info["smem_slots"]


def test_config2_subset_emulated(capi, oracle_mod):
    g = synth.config2()
    check_program(capi, oracle_mod, g, 44, W=8, iteration=1, word_begin=(1 << 24) - 8)


def test_edge_connectives(capi, oracle_mod):
    # thresholds 0 and 2^32, NOT/NULL with several inputs (last wins), a gate
    # without inputs, ATLEAST with k = 0 and k > n, duplicate inputs, a
    # tallied basic event and a tally listed twice.
    thr = probability_threshold([0.3, 0.0, 1.0, 0.7, 0.5])
    g = FlatGraph(
        be_pdag_idx=np.arange(5) + 2, be_event_idx=np.arange(5), be_threshold=thr,
        gate_op=[OR, NOT, NULL, ATLEAST, ATLEAST, OR, NOT, ATLEAST],
        gate_k=[0, 0, 0, 0, 9, 0, 0, 2],
        gate_in_begin=[0, 3, 6, 8, 8, 11, 13, 13],
        gate_in_count=[3, 3, 2, 3, 3, 2, 0, 3],
        gate_neg_count=[1, 1, 0, 0, 0, 0, 0, 1],
        inputs=[0, 1, 2, 0, 3, 4, 4, 0, 0, 1, 3, 5, 5, 9, 10, 11],
        tally_nodes=[5, 6, 7, 8, 9, 10, 11, 12, 0, 12, 2])
    for budget in (0, 1, 8):
        check_program(capi, oracle_mod, g, budget)
