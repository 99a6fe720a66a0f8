"""Host layer without a GPU: PDAG layering (event_idx assignment), flattening,
sample shaping, statistics and error behaviour of the reference-shaped API."""
import numpy as np
import pytest
import scipy.stats

from mcscram_b200 import host, synth
from mcscram_b200._capi import MCG_ERR_INVALID, McgError
from mcscram_b200.graph import AND, ATLEAST, NOT, OR, XOR


def test_event_order_follows_gather_order_small():
    # root = OR(G1, x9), G1 = AND(x7, x3): the depth-first gather visits
    # root, G1, x7, x3, x9; small sorts are stable, so event_idx follows it.
    p = host.Pdag()
    for i, pr in [(3, 0.1), (7, 0.2), (9, 0.3)]:
        p.add_variable(i, pr)
    p.add_gate(20, AND, [7, 3])
    p.add_gate(21, OR, [20, 9])
    p.set_root(21)
    assert p.event_order() == [7, 3, 9]
    g = p.flatten([21, 20])
    assert list(g.be_pdag_idx) == [7, 3, 9]
    assert list(g.be_event_idx) == [0, 1, 2]
    assert list(g.gate_pdag_idx) == [20, 21]  # layer 1, then layer 2


def test_gate_args_before_variable_args_in_gather():
    # root = AND(x2, G1, x5), G1 = OR(x4, x3): gate args are gathered first.
    p = host.Pdag()
    for i in (2, 3, 4, 5):
        p.add_variable(i, 0.1 * i)
    p.add_gate(10, OR, [4, 3])
    p.add_gate(11, AND, [2, 10, 5])
    p.set_root(11)
    assert p.event_order() == [4, 3, 2, 5]


def test_flat_inputs_layout_matches_kernel_builder():
    # variables first then gates; complemented ones moved to the tail
    p = host.Pdag()
    for i in (2, 3, 4):
        p.add_variable(i, 0.5)
    p.add_gate(10, OR, [2, -3])
    p.add_gate(11, AND, [-10, 4, 2])
    p.set_root(11)
    g = p.flatten([11])
    be = {int(v): k for k, v in enumerate(g.be_pdag_idx)}
    g10 = g.n_be + list(g.gate_pdag_idx).index(10)
    gi = list(g.gate_pdag_idx).index(11)
    assert list(g.gate_inputs(gi)) == [be[4], be[2], g10]
    assert int(g.gate_neg_count[gi]) == 1
    gi10 = list(g.gate_pdag_idx).index(10)
    assert list(g.gate_inputs(gi10)) == [be[2], be[3]] and int(g.gate_neg_count[gi10]) == 1


def test_large_layering_invariants():
    g0 = synth.config2()
    p = host.Pdag.from_flat(g0)
    order = p.event_order()
    assert sorted(order) == sorted(map(int, g0.be_pdag_idx))
    g = p.flatten([int(g0.gate_pdag_idx[-1])])
    assert g.n_be == g0.n_be and g.n_gates == g0.n_gates
    layers = g.layers()[g.n_be:]
    assert np.all(np.diff(layers) >= 0)
    # within a layer, gates sorted by connective
    for L in np.unique(layers):
        ops = g.gate_op[layers == L]
        assert np.all(np.diff(ops.astype(int)) >= 0)


def test_flattened_pdag_is_the_same_function(oracle_mod):
    g0 = synth.small_tree(2, n_be=14, n_gates=9, n_layers=3)
    p = host.Pdag.from_flat(g0)
    g = p.flatten([int(g0.gate_pdag_idx[-1])])
    g.root = int(g.tally_nodes[0])
    assert oracle_mod.bdd_probability(g) == pytest.approx(oracle_mod.bdd_probability(g0), rel=1e-12)


def test_pdag_errors():
    p = host.Pdag()
    p.add_variable(2, 0.5)
    with pytest.raises(McgError) as e:
        p.add_variable(2, 0.1)
    assert e.value.code == MCG_ERR_INVALID
    with pytest.raises(McgError):
        p.add_variable(1, 0.1)
    with pytest.raises(McgError):
        p.add_variable(3, 1.5)
    p.add_gate(10, AND, [2, 99])
    with pytest.raises(McgError):
        p.set_root(2)
    p.set_root(10)
    with pytest.raises(McgError) as e:
        p.event_order()
    assert "unknown argument" in str(e.value)


def test_manager_rejects_unknown_tally_before_device():
    p = host.Pdag()
    p.add_variable(2, 0.5)
    p.add_variable(3, 0.5)
    p.add_gate(10, AND, [2, 3])
    p.set_root(10)
    with pytest.raises(McgError) as e:
        host.LayerManager(p, 1 << 20, [10, 77])
    assert e.value.code == MCG_ERR_INVALID
    assert "Attempting to build tally for unknown event 77" in str(e.value)


@pytest.mark.parametrize("trials,words,iters,rounded", [
    (1 << 20, 16384, 1, 1 << 20),          # config 1: one pass of 16,384 words
    (1 << 30, 1 << 24, 1, 1 << 30),        # config 2 with the 2^24-word pass cap
    (1 << 32, 1 << 24, 4, 1 << 32),
    (1_000_000, 16384, 1, 1_000_000),      # 15,625 words -> closest power of two
    (100, 2, 1, 128),                      # remainder 36 > 32 rounds up
    (96 + 32, 2, 1, 128),
    (64 + 32, 1, 1, 64),                   # remainder 32 rounds down
    (0, 1 << 20, 0, 1 << 26),              # no request: 2^26 trials, no pass limit
])
def test_sample_shape(trials, words, iters, rounded):
    s = host.sample_shape(trials)
    assert s == {"words_per_iteration": words, "total_iterations": iters, "num_trials": rounded}


def test_normal_quantile_matches_reference_constants():
    assert host.normal_quantile_two_sided(0.95) == pytest.approx(1.959963984540054, rel=2e-9)
    assert host.normal_quantile_two_sided(0.99) == pytest.approx(2.5758293035489004, rel=2e-9)
    for c in (0.5, 0.8, 0.999, 0.999999):
        assert host.normal_quantile_two_sided(c) == pytest.approx(scipy.stats.norm.ppf(0.5 + c / 2), rel=2e-9)


@pytest.mark.parametrize("a,b", [(0.5, 0.5), (3.5, 1000.5), (0.5, 1e6 + 0.5), (50.5, 1e9), (2e3, 5e3),
                                 (1e6, 1e9), (5e5, 5e5), (1e9, 20.5)])
def test_beta_quantile_vs_scipy(a, b):
    for q in (0.005, 0.025, 0.5, 0.975, 0.995):
        ref = scipy.stats.beta.ppf(q, a, b)
        got = host.beta_quantile(a, b, q)
        sd = np.sqrt(a * b / ((a + b) ** 2 * (a + b + 1)))
        # accurate to a small fraction of the posterior spread (stopping rule only)
        assert abs(got - ref) <= max(1e-3 * sd, 1e-14), (a, b, q, got, ref)
