"""The oracle pinned to the reference: golden vectors from the reference's own
Philox build, closed-form and exhaustive checks of the BDD, and the MC
estimate against the BDD.  CPU only."""
import itertools
import json
from pathlib import Path

import numpy as np
import pytest

from mcscram_b200 import synth
from mcscram_b200.graph import AND, ATLEAST, NAND, NOR, NOT, NULL, OR, XOR, FlatGraph, probability_threshold

GOLDEN = Path(__file__).resolve().parent / "golden"


def load_graph(npz, prefix=""):
    return FlatGraph(**{k: npz[prefix + k] for k in (
        "be_pdag_idx", "be_event_idx", "be_threshold", "gate_op", "gate_k", "gate_in_begin", "gate_in_count",
        "gate_neg_count", "inputs", "tally_nodes")})


def test_survey_probe_vector(oracle_mod):
    # counter {3, 1, 1, 128}, p = 0.5: the vector probed on the reference header
    assert oracle_mod.word(3, 1, 1, 128, 1 << 31) == 0xDDA69A821AE43090


def test_packed_golden_vectors(oracle_mod):
    data = json.loads((GOLDEN / "philox_vectors.json").read_text())
    for v in data["packed"]:
        assert oracle_mod.word(*v["counter"], v["threshold"]) == v["word"], v
    for v in data["basic_event"]:
        got = oracle_mod.be_word(v["pdag_idx"], v["event_idx"], v["sample_idx"], v["iteration"], v["threshold"])
        assert got == v["word"], v


def test_threshold_edges(oracle_mod):
    for c in [(3, 1, 1, 128), (7, 9, 11, 13 << 6)]:
        assert oracle_mod.word(*c, 0) == 0
        assert oracle_mod.word(*c, 1 << 32) == (1 << 64) - 1


def test_restated_matches_reference_build(oracle_mod):
    if not oracle_mod.has_reference_build():
        pytest.skip("reference Philox build absent")
    rng = np.random.default_rng(5)
    for _ in range(2000):
        c = [int(x) for x in rng.integers(0, 1 << 32, size=4, dtype=np.uint64)]
        thr = int(rng.integers(0, (1 << 32) + 1))
        assert oracle_mod.word(*c, thr) == oracle_mod.word(*c, thr, reference=True)


def test_small_tree_words_golden(oracle_mod):
    npz = np.load(GOLDEN / "small_trees.npz")
    for name in npz["names"]:
        g = load_graph(npz, str(name))
        got = oracle_mod.eval_words(g, 1, 0, 96)
        assert np.array_equal(got, npz[str(name) + "words_it1_w0"])
        got = oracle_mod.eval_words(g, 3, (1 << 32) - 64, 64)
        assert np.array_equal(got, npz[str(name) + "words_it3_whigh"])


def test_config1_tallies_golden(oracle_mod):
    npz = np.load(GOLDEN / "config1_tallies.npz")
    g = load_graph(npz)
    ones = oracle_mod.tallies(g, 1, 1, 0, int(npz["words"]))
    assert np.array_equal(ones, npz["ones"])
    # the committed graph is the generator's config 1
    g1 = synth.config1()
    assert np.array_equal(g1.inputs, g.inputs) and np.array_equal(g1.be_threshold, g.be_threshold)


def _one_gate(op, n, k=0, neg=0, p=None):
    p = np.array(p if p is not None else [0.1 * (i + 1) for i in range(n)])
    return FlatGraph(be_pdag_idx=np.arange(n) + 2, be_event_idx=np.arange(n), be_threshold=probability_threshold(p),
                     gate_op=[op], gate_k=[k], gate_in_begin=[0], gate_in_count=[n], gate_neg_count=[neg],
                     inputs=np.arange(n), tally_nodes=[n]), p


def test_bdd_closed_forms(oracle_mod):
    q = lambda g: g.quantised_probabilities()
    g, _ = _one_gate(AND, 3)
    assert oracle_mod.bdd_probability(g) == pytest.approx(np.prod(q(g)), rel=1e-12)
    g, _ = _one_gate(OR, 3)
    assert oracle_mod.bdd_probability(g) == pytest.approx(1 - np.prod(1 - q(g)), rel=1e-12)
    g, _ = _one_gate(NAND, 2)
    assert oracle_mod.bdd_probability(g) == pytest.approx(1 - np.prod(q(g)), rel=1e-12)
    g, _ = _one_gate(NOR, 2)
    assert oracle_mod.bdd_probability(g) == pytest.approx(np.prod(1 - q(g)), rel=1e-12)
    g, _ = _one_gate(XOR, 2)
    a, b = q(g)
    assert oracle_mod.bdd_probability(g) == pytest.approx(a * (1 - b) + b * (1 - a), rel=1e-12)
    g, _ = _one_gate(NOT, 1)
    assert oracle_mod.bdd_probability(g) == pytest.approx(1 - q(g)[0], rel=1e-12)
    g, _ = _one_gate(ATLEAST, 3, k=2)
    a, b, c = q(g)
    assert oracle_mod.bdd_probability(g) == pytest.approx(a * b + a * c + b * c - 2 * a * b * c, rel=1e-12)
    g, _ = _one_gate(AND, 2, neg=1)  # A and not B
    a, b = q(g)
    assert oracle_mod.bdd_probability(g) == pytest.approx(a * (1 - b), rel=1e-12)


def _exhaustive(g):
    """P(root) by enumerating every basic-event assignment (small graphs)."""
    p = g.quantised_probabilities()
    total = 0.0
    for bits in itertools.product([0, 1], repeat=g.n_be):
        val = list(bits)
        for gi in range(g.n_gates):
            ins = g.gate_inputs(gi)
            off = int(g.gate_in_count[gi] - g.gate_neg_count[gi])
            xs = [val[c] if i < off else 1 - val[c] for i, c in enumerate(ins)]
            op = int(g.gate_op[gi])
            if op in (AND, NAND):
                r = int(all(xs))
            elif op in (OR, NOR):
                r = int(any(xs))
            elif op == XOR:
                r = sum(xs) % 2
            elif op == ATLEAST:
                r = int(sum(xs) % 256 >= int(g.gate_k[gi]) % 256)
            else:
                r = xs[-1] if xs else 0
            if op in (NAND, NOR, NOT):
                r = 1 - r
            val.append(r)
        w = np.prod([p[i] if bits[i] else 1 - p[i] for i in range(g.n_be)])
        total += w * val[g.root]
    return total


@pytest.mark.parametrize("seed", range(4))
def test_bdd_vs_exhaustive(oracle_mod, seed):
    g = synth.small_tree(seed, n_be=11, n_gates=8, n_layers=3, p_range=(0.05, 0.7))
    g.gate_neg_count = np.array([1 if (gi % 2 and g.gate_in_count[gi] > 1) else 0 for gi in range(g.n_gates)],
                                dtype=np.uint32)
    assert oracle_mod.bdd_probability(g) == pytest.approx(_exhaustive(g), rel=1e-10, abs=1e-15)


def test_oracle_atleast_uint8_wrap(oracle_mod):
    # 257 always-true inputs: the reference's uint8 count wraps to 1 < k = 2
    n = 257
    g = FlatGraph(be_pdag_idx=np.arange(n) + 2, be_event_idx=np.arange(n), be_threshold=np.full(n, 1 << 32),
                  gate_op=[ATLEAST, ATLEAST], gate_k=[2, 1], gate_in_begin=[0, 0], gate_in_count=[n, n],
                  gate_neg_count=[0, 0], inputs=np.arange(n), tally_nodes=[n, n + 1])
    w = oracle_mod.eval_words(g, 1, 0, 4)
    assert np.all(w[n] == 0) and np.all(w[n + 1] == np.uint64(0xFFFFFFFFFFFFFFFF))


def test_config1_estimate_within_3sigma_of_bdd(oracle_mod):
    g = synth.config1()
    exact = oracle_mod.bdd_probability(g)
    ones = oracle_mod.tallies(g.with_tallies([g.root]), 1, 1, 0, 16384)
    n = 16384 * 64
    phat = float(ones[0]) / n
    sigma = np.sqrt(exact * (1 - exact) / n)
    assert abs(phat - exact) <= 3 * sigma, (phat, exact, sigma)
