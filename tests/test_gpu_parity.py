"""Parity of the CUDA path with the oracle, through the C ABI (needs a GPU).

Bit-exact: basic-event and gate words (layered kernels, mcg_dump_words) and
tallies (fused and layered kernels) against the oracle and against the
golden fixtures drawn from the reference's own Philox build.  At full sizes:
fused vs layered kernels (two independent device paths) and tally
additivity over word ranges.  Statistical: config 1's top-event estimate
within 3 sigma of the exact BDD probability."""
from pathlib import Path

import numpy as np
import pytest

from mcscram_b200 import synth
from mcscram_b200.graph import ATLEAST, NOT, NULL, OR, XOR, AND, FlatGraph, probability_threshold
from tests.test_oracle import load_graph

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"


def engine(capi, g, **kw):
    return capi.Engine(g, **kw)


def test_words_match_golden_fixtures(capi, gpu):
    npz = np.load(GOLDEN / "small_trees.npz")
    for name in npz["names"]:
        g = load_graph(npz, str(name))
        with engine(capi, g, mode=capi.MODE_LAYERED) as e:
            assert np.array_equal(e.dump_words(1, 0, 96), npz[str(name) + "words_it1_w0"])
            assert np.array_equal(e.dump_words(3, (1 << 32) - 64, 64), npz[str(name) + "words_it3_whigh"])


@pytest.mark.parametrize("mode", ["fused", "layered", "staged", "strip"])
def test_small_tree_tallies_golden(capi, oracle_mod, gpu, mode):
    npz = np.load(GOLDEN / "small_trees.npz")
    m = capi.MODES[mode]
    for name in npz["names"]:
        g = load_graph(npz, str(name))
        g = g.with_tallies(np.arange(g.n_nodes))  # every node, basic events included
        words = npz[str(name) + "words_it1_w0"]
        expect = np.array([sum(bin(int(x)).count("1") for x in words[n]) for n in range(g.n_nodes)], np.uint64)
        with engine(capi, g, mode=m) as e:
            e.run(1, 1, 0, 96)
            ones, total = e.tallies()
            assert total == 96 * 64
            assert np.array_equal(ones, expect)


@pytest.mark.parametrize("mode", ["fused", "layered", "staged", "strip"])
def test_config1_golden_tallies(capi, gpu, mode):
    npz = np.load(GOLDEN / "config1_tallies.npz")
    g = load_graph(npz)
    m = capi.MODES[mode]
    with engine(capi, g, mode=m) as e:
        e.run(1, 1, 0, int(npz["words"]))
        ones, total = e.tallies()
    assert total == (1 << 20)
    assert np.array_equal(ones, npz["ones"])


@pytest.mark.parametrize("slots", [0xFFFFFFFF, 1, 2, 7, 0])
def test_fused_any_slot_budget(capi, oracle_mod, gpu, slots):
    g = synth.small_tree(3, n_be=60, n_gates=40, n_layers=6, p_range=(0.02, 0.5))
    g.gate_neg_count = np.array([1 if (gi % 4 == 1 and g.gate_in_count[gi] > 1) else 0 for gi in range(g.n_gates)],
                                dtype=np.uint32)
    g = g.with_tallies(np.arange(g.n_nodes))
    for (it, wb, n) in [(1, 0, 1), (1, 0, 33), (2, 1000, 1000), (5, (1 << 32) - 777, 777), (1, 12345, 70000)]:
        expect = oracle_mod.tallies(g, it, 1, wb, n)
        with engine(capi, g, smem_slots=slots) as e:
            e.run(it, 1, wb, n)
            ones, total = e.tallies()
        assert total == n * 64
        assert np.array_equal(ones, expect), (slots, it, wb, n)


@pytest.mark.parametrize("mode", ["fused", "staged", "strip"])
def test_multiple_passes_and_ranges(capi, oracle_mod, gpu, mode):
    g = synth.config1()
    expect = oracle_mod.tallies(g, 2, 3, 500, 3000)
    with engine(capi, g, mode=capi.MODES[mode], layered_max_words=1024) as e:
        e.run(2, 3, 500, 3000)
        ones, total = e.tallies()
        assert total == 3 * 3000 * 64
        assert np.array_equal(ones, expect)
        e.reset_tallies()
        # additivity: split ranges and passes give the same counts
        e.run(2, 1, 500, 1000)
        e.run(2, 1, 1500, 2000)
        e.run(3, 2, 500, 3000)
        ones2, total2 = e.tallies()
        assert total2 == total and np.array_equal(ones2, expect)


@pytest.mark.parametrize("mode", ["fused", "staged", "strip"])
def test_config2_windows_bit_exact(capi, oracle_mod, gpu, mode):
    g = synth.config2()
    with engine(capi, g, mode=capi.MODES[mode]) as e:
        for (wb, n) in [(0, 2048), ((1 << 24) - 2048, 2048), ((1 << 24) + 77, 513)]:
            expect = oracle_mod.tallies(g, 1, 1, wb, n)
            e.reset_tallies()
            e.run(1, 1, wb, n)
            ones, _ = e.tallies()
            assert np.array_equal(ones, expect), (wb, n)


def test_config2_headline_pass(capi, oracle_mod, gpu):
    """The benchmark's pass (pass 1 over words [0, 2^24) of the 5,000-event
    tree, strip mode) checked without a full CPU pass: its tallies equal the
    sum of the two half passes run by other engines (staged, fused), and
    windows drawn across the whole range equal the oracle's."""
    g = synth.config2()
    W = 1 << 24
    with engine(capi, g, mode=capi.MODE_STRIP) as e:
        e.run(1, 1, 0, W)
        full, total = e.tallies()
        rng = np.random.default_rng(24)
        for wb in sorted(int(x) for x in rng.integers(0, W - 512, 6)):
            e.reset_tallies()
            e.run(1, 1, wb, 512)
            ones, _ = e.tallies()
            assert np.array_equal(ones, oracle_mod.tallies(g, 1, 1, wb, 512)), wb
    assert total == W * 64
    with engine(capi, g, mode=capi.MODE_STAGED, layered_max_words=1 << 17) as st:
        st.run(1, 1, 0, W // 2)
        lo, _ = st.tallies()
    with engine(capi, g, mode=capi.MODE_FUSED) as f:
        f.run(1, 1, W // 2, W // 2)
        hi, _ = f.tallies()
    assert np.array_equal(full, lo + hi)
    assert int(full.sum()) > 0


def test_config2_fused_equals_layered_large(capi, gpu):
    g = synth.config2()
    W = 1 << 19
    with engine(capi, g) as f:
        f.run(1, 1, 0, W)
        a, ta = f.tallies()
    with engine(capi, g, mode=capi.MODE_LAYERED, layered_max_words=1 << 17) as l:
        l.run(1, 1, 0, W)
        b, tb = l.tallies()
    with engine(capi, g, mode=capi.MODE_STAGED, layered_max_words=1 << 17) as st:
        st.run(1, 1, 0, W)
        c, tc = st.tallies()
    with engine(capi, g, mode=capi.MODE_STRIP) as sp:
        sp.run(1, 1, 0, W)
        d, td = sp.tallies()
    assert ta == tb == tc == td == W * 64
    assert np.array_equal(a, b) and np.array_equal(a, c) and np.array_equal(a, d)
    assert a.sum() > 0


def test_edge_cases(capi, oracle_mod, gpu):
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
    expect = oracle_mod.tallies(g, 1, 1, 0, 4000)
    words = oracle_mod.eval_words(g, 1, 0, 64)
    for mode in (capi.MODE_FUSED, capi.MODE_LAYERED, capi.MODE_STAGED, capi.MODE_STRIP):
        with engine(capi, g, mode=mode) as e:
            e.run(1, 1, 0, 4000)
            ones, _ = e.tallies()
            assert np.array_equal(ones, expect)
            assert np.array_equal(e.dump_words(1, 0, 64), words)


def test_atleast_uint8_wrap(capi, oracle_mod, gpu):
    n = 300
    rng = np.random.default_rng(0)
    thr = probability_threshold(rng.uniform(0.3, 0.99, n))
    g = FlatGraph(be_pdag_idx=np.arange(n) + 2, be_event_idx=np.arange(n), be_threshold=thr,
                  gate_op=[ATLEAST, ATLEAST, ATLEAST], gate_k=[2, 200, 45], gate_in_begin=[0, 0, 0],
                  gate_in_count=[n, n, n], gate_neg_count=[0, 10, 0], inputs=np.arange(n),
                  tally_nodes=[n, n + 1, n + 2])
    expect = oracle_mod.tallies(g, 1, 1, 0, 2000)
    for mode in (capi.MODE_FUSED, capi.MODE_LAYERED, capi.MODE_STAGED, capi.MODE_STRIP):
        with engine(capi, g, mode=mode) as e:
            e.run(1, 1, 0, 2000)
            assert np.array_equal(e.tallies()[0], expect)


def test_config1_top_within_3sigma_of_bdd(capi, oracle_mod, gpu):
    g = synth.config1()
    exact = oracle_mod.bdd_probability(g)
    with engine(capi, g.with_tallies([g.root])) as e:
        e.run(1, 64, 0, 1 << 16)  # 2^28 samples
        ones, total = e.tallies()
    phat = float(ones[0]) / total
    sigma = np.sqrt(exact * (1 - exact) / total)
    assert abs(phat - exact) <= 3 * sigma, (phat, exact, sigma)


def test_sampler_peak_runs(capi, gpu):
    rate = capi.sampler_peak(n_events=64, n_words=1 << 18, repeats=2)
    assert rate > 1e9


def test_engines_reuse_kept_work_buffers(capi, oracle_mod, gpu):
    """Engines created one after another (every mode, and the strip engine
    again after mcg_trim_memory) take the work buffers a destroyed engine
    left behind: every one still gives the oracle's tallies."""
    g = synth.config1()
    words = 1 << 12
    want = oracle_mod.tallies(g, 2, 1, 0, words)
    for mode in ("strip", "fused", "staged", "strip", "fused"):
        with engine(capi, g, mode=capi.MODES[mode]) as e:
            e.run(2, 1, 0, words)
            ones, total = e.tallies()
        assert np.array_equal(ones, want) and total == words * 64, mode
    capi.trim_memory(0)
    with engine(capi, g, mode=capi.MODE_STRIP) as e:
        e.run(2, 1, 0, words)
        assert np.array_equal(e.tallies()[0], want)


@pytest.mark.parametrize("mode", ["fused", "staged", "strip"])
def test_engine_created_later_with_a_smaller_program(capi, oracle_mod, gpu, mode):
    """A kernel's shared-memory limit is shared by every engine that launches
    it: an engine created after another one, with a program that needs less
    shared memory, must leave the first engine's launches working."""
    big = synth.config1()
    small = synth.small_tree(5, n_be=12, n_gates=6)
    small = small.with_tallies([small.root])
    words = 1 << 12
    m = capi.MODES[mode]
    kw = dict(sampler_blocks_per_sm=2) if mode == "staged" else {}
    with engine(capi, big, mode=m, **kw) as a:
        with engine(capi, small, mode=m) as b:
            b.run(1, 1, 0, words)
            assert np.array_equal(b.tallies()[0], oracle_mod.tallies(small, 1, 1, 0, words))
        a.run(1, 1, 0, words)
        assert np.array_equal(a.tallies()[0], oracle_mod.tallies(big, 1, 1, 0, words))
