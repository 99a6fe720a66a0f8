"""Batched instances and uncertainty analysis.  CPU: the variable-threshold
program form; GPU: every instance bit-exact against the oracle with its own
thresholds, and the uncertainty statistics."""
import numpy as np
import pytest

from mcscram_b200 import mef, synth
from mcscram_b200.graph import probability_threshold
from tests.program_emulator import emulate


def test_variable_threshold_program_emulated(capi, oracle_mod):
    """The program form the batch engine compiles (thresholds by table index)
    gives the oracle's words for the instance's thresholds."""
    lib = capi.load()
    for seed in range(3):
        g = synth.small_tree(seed, n_be=30, n_gates=18, n_layers=4)
        g = g.with_tallies(np.arange(g.n_be, g.n_nodes))
        thr = g.be_threshold.copy()
        thr[0] = 0
        thr[1] = 1 << 32
        g = g.with_thresholds(thr)
        info, ops = capi.compile_program(g, 3, variable_thresholds=True)
        words = oracle_mod.eval_words(g, 1, 0, 64)
        vals, _ = emulate(ops, g, words, int(g.tally_nodes.size), variable_thresholds=True)
        for i, node in enumerate(g.tally_nodes):
            assert np.array_equal(vals[i], words[node])


def _instances(trees, n_draws, rng):
    inst_tree, thr = [], []
    for t, g in enumerate(trees):
        for d in range(n_draws):
            p = rng.uniform(0.01, 0.6, g.n_be)
            th = probability_threshold(p)
            if d == 1:
                th[0] = 0
                th[-1] = 1 << 32
            inst_tree.append(t)
            thr.append(th)
    return inst_tree, thr


@pytest.mark.gpu
def test_batch_instances_bit_exact(oracle_mod, gpu):
    from mcscram_b200.uncertainty import Batch
    rng = np.random.default_rng(7)
    trees = [synth.small_tree(s, n_be=40, n_gates=25, n_layers=5) for s in range(4)]
    trees = [t.with_tallies([t.root]) for t in trees]
    inst_tree, thr = _instances(trees, 3, rng)
    W = 3000
    with Batch(trees) as b:
        ones = b.run(inst_tree, thr, iteration=1, words_per_instance=W)
        ones2 = b.run(inst_tree, thr, iteration=1, words_per_instance=W)  # graph replay
        ones3 = b.run(inst_tree, thr, iteration=2, words_per_instance=W)  # re-capture
    for i, (t, th) in enumerate(zip(inst_tree, thr)):
        g = trees[t].with_thresholds(th)
        assert int(ones[i]) == int(oracle_mod.tallies(g, 1, 1, 0, W)[0]), i
        assert int(ones3[i]) == int(oracle_mod.tallies(g, 2, 1, 0, W)[0]), i
    assert np.array_equal(ones, ones2)


# negated event and gate inputs, NAND, NOR and XOR, no ATLEAST
_NEGATIONS = """<opsa-mef><define-fault-tree name="n">
<define-gate name="top"><or><gate name="a"/><gate name="b"/><not><basic-event name="e5"/></not></or></define-gate>
<define-gate name="a"><nand><basic-event name="e1"/><not><basic-event name="e2"/></not><basic-event name="e3"/>
</nand></define-gate>
<define-gate name="b"><and><gate name="b_nor"/><gate name="b_xor"/><basic-event name="e6"/></and></define-gate>
<define-gate name="b_nor"><nor><basic-event name="e3"/><basic-event name="e4"/></nor></define-gate>
<define-gate name="b_xor"><xor><basic-event name="e1"/><not><gate name="a"/></not></xor></define-gate>
</define-fault-tree><model-data>""" + "".join(
    f'<define-basic-event name="e{i}"><float value="0.{i}"/></define-basic-event>' for i in range(1, 7)) + \
    "</model-data></opsa-mef>"


@pytest.mark.gpu
@pytest.mark.parametrize("slots", [0xFFFFFFFF, 3, 0])
def test_shared_draws_bit_exact(oracle_mod, gpu, slots):
    """Trees without ATLEAST gates run up to four instances of one tree per
    work item, sharing their Philox calls: groups longer than four, groups of
    one, a tree coming back after another, thresholds 0 and 2^32 inside a
    group and an instance whose every threshold is constant -- every instance
    bit-exact against the oracle at its own thresholds."""
    from mcscram_b200.graph import AND, NOT, OR, XOR
    from mcscram_b200.uncertainty import Batch
    rng = np.random.default_rng(23)
    mix = {AND: 0.4, OR: 0.4, XOR: 0.1, NOT: 0.1}
    trees = [synth.small_tree(s, n_be=40, n_gates=25, n_layers=5, mix=mix) for s in (3, 4, 5)]
    trees = [t.with_tallies([t.root]) for t in trees] + [mef.load(_NEGATIONS)]
    order = [0] * 6 + [1] + [0] * 2 + [2] * 5 + [1] * 4 + [3] * 7
    inst_tree, thr = [], []
    for i, t in enumerate(order):
        th = probability_threshold(rng.uniform(0.02, 0.7, trees[t].n_be))
        if i % 3 == 1:
            th[0], th[5] = 0, 1 << 32
        if i == 7:
            th = np.where(rng.random(trees[t].n_be) < 0.5, 0, 1 << 32).astype(np.uint64)
        inst_tree.append(t)
        thr.append(th)
    W = 2500
    with Batch(trees, smem_slots=slots) as b:
        assert b.info()["instances_per_item"] == 4
        ones = b.run(inst_tree, thr, iteration=3, words_per_instance=W)
    for i, (t, th) in enumerate(zip(inst_tree, thr)):
        assert int(ones[i]) == int(oracle_mod.tallies(trees[t].with_thresholds(th), 3, 1, 0, W)[0]), i


# an ATLEAST gate of 16 inputs: wider than the shared kernel's four-slice counters
_WIDE_ATLEAST = ("<opsa-mef><define-fault-tree name='w'><define-gate name='top'><or>"
                 "<gate name='wide'/><basic-event name='y'/></or></define-gate><define-gate name='wide'>"
                 "<atleast min='3'>" + "".join(f"<basic-event name='x{i}'/>" for i in range(16)) + "</atleast>"
                 "</define-gate></define-fault-tree><model-data>" +
                 "".join(f"<define-basic-event name='x{i}'><float value='0.{i % 9 + 1}'/></define-basic-event>"
                         for i in range(16)) +
                 "<define-basic-event name='y'><float value='0.01'/></define-basic-event></model-data></opsa-mef>")


@pytest.mark.gpu
def test_atleast_widths_and_instances_per_item(oracle_mod, gpu):
    """ATLEAST gates of up to 15 inputs run four draws per work item (counted
    in four bit slices per draw); a wider one sends the batch back to one
    draw per item.  Both bit-exact against the oracle."""
    from mcscram_b200.uncertainty import Batch
    rng = np.random.default_rng(5)
    narrow = synth.small_tree(2, n_be=30, n_gates=18, n_layers=4)
    assert any(int(op) == 2 for op in narrow.gate_op)  # ATLEAST present, 3-5 inputs
    narrow = narrow.with_tallies([narrow.root])
    wide = mef.load(_WIDE_ATLEAST)
    for trees, per_item in (([narrow], 4), ([narrow, wide], 1)):
        inst_tree = [t for t in range(len(trees)) for _ in range(5)]
        thr = []
        for i, t in enumerate(inst_tree):
            th = probability_threshold(rng.uniform(0.05, 0.8, trees[t].n_be))
            if i == 2:
                th[0], th[-1] = 0, 1 << 32
            thr.append(th)
        with Batch(trees) as b:
            assert b.info()["instances_per_item"] == per_item
            ones = b.run(inst_tree, thr, iteration=2, words_per_instance=3000)
        for i, (t, th) in enumerate(zip(inst_tree, thr)):
            assert int(ones[i]) == int(oracle_mod.tallies(trees[t].with_thresholds(th), 2, 1, 0, 3000)[0]), (per_item, i)


@pytest.mark.gpu
@pytest.mark.parametrize("slots", [0xFFFFFFFF, 2, 0])
def test_batch_slot_budgets(oracle_mod, gpu, slots):
    from mcscram_b200.uncertainty import Batch
    rng = np.random.default_rng(11)
    trees = [synth.config1()] + [synth.small_tree(9, n_be=50, n_gates=30, n_layers=5)]
    trees = [t.with_tallies([t.root]) for t in trees]
    inst_tree, thr = _instances(trees, 2, rng)
    with Batch(trees, smem_slots=slots) as b:
        ones = b.run(inst_tree, thr, iteration=1, words_per_instance=1000)
    for i, (t, th) in enumerate(zip(inst_tree, thr)):
        assert int(ones[i]) == int(oracle_mod.tallies(trees[t].with_thresholds(th), 1, 1, 0, 1000)[0])


@pytest.mark.gpu
def test_uncertainty_small(oracle_mod, gpu):
    from mcscram_b200.uncertainty import Batch
    trees = [t.with_tallies([t.root]) for t in synth.config3(6, seed=5)]
    draws, W = 4, 4096
    with Batch(trees) as b:
        p_top, stats, ms, thr = b.uncertainty([t.be_prob for t in trees], draws_per_tree=draws,
                                              words_per_instance=W, seed=99, return_thresholds=True)
    off = 0
    for t, g in enumerate(trees):
        for d in range(draws):
            th = thr[off:off + g.n_be]
            off += g.n_be
            ones = oracle_mod.tallies(g.with_thresholds(th), 1, 1, 0, W)[0]
            assert p_top[t, d] == int(ones) / (W * 64)
            # sampled probabilities: lognormal around the base, clipped to 0.5
            p = th.astype(np.float64) / 2**32
            assert p.max() <= 0.5 + 1e-9
        v = p_top[t]
        assert stats[t]["mean"] == pytest.approx(v.mean())
        assert stats[t]["sigma"] == pytest.approx(v.std(ddof=1))
        assert stats[t]["p05"] == pytest.approx(np.percentile(v, 5))
        assert stats[t]["p95"] == pytest.approx(np.percentile(v, 95))
    assert ms > 0


@pytest.mark.gpu
def test_uncertainty_against_bdd(oracle_mod, gpu):
    from mcscram_b200.uncertainty import Batch
    trees = [t.with_tallies([t.root]) for t in synth.config3(4, seed=8) if t.n_gates <= 400][:3]
    draws, W = 3, 1 << 16
    with Batch(trees) as b:
        p_top, stats, ms, thr = b.uncertainty([t.be_prob for t in trees], draws_per_tree=draws,
                                              words_per_instance=W, return_thresholds=True)
    off = 0
    for t, g in enumerate(trees):
        for d in range(draws):
            th = thr[off:off + g.n_be]
            off += g.n_be
            exact = oracle_mod.bdd_probability(g.with_thresholds(th))
            n = W * 64
            sigma = np.sqrt(max(exact * (1 - exact), 1e-300) / n)
            assert abs(p_top[t, d] - exact) <= 4 * sigma + 1e-12, (t, d, p_top[t, d], exact)
