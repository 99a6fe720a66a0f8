"""The launch-shape tuner (include/mcg_tune.h): on CPU with a fake timer in
place of the probe passes (which candidates are measured, which one is kept,
cache hits in memory and from the file, which shapes share an entry); on the
GPU the tuned engine against the oracle."""
import numpy as np
import pytest

from mcscram_b200 import _capi as capi
from mcscram_b200 import synth

CANDIDATES = [(capi.MODE_STRIP, 6), (capi.MODE_STRIP, 5), (capi.MODE_STRIP, 4), (capi.MODE_STAGED, 0),
              (capi.MODE_FUSED, 4), (capi.MODE_FUSED, 2)]


class FakeTimer:
    """Rates by (mode, ctas); records every probe."""

    def __init__(self, rates):
        self.rates = rates
        self.calls = []

    def __call__(self, mode, ctas, words):
        self.calls.append((mode, ctas, words))
        return self.rates.get((mode, ctas), -1.0)


@pytest.fixture
def cache(tmp_path):
    path = tmp_path / "tune.txt"
    capi.tune_set_cache_file(str(path))
    capi.tune_forget()
    yield path
    capi.tune_set_cache_file("")
    capi.tune_forget()


def test_miss_probes_every_candidate_and_keeps_the_fastest(cache):
    g = synth.config1()
    t = FakeTimer({(capi.MODE_STRIP, 6): 2.0e10, (capi.MODE_STAGED, 0): 2.5e10, (capi.MODE_FUSED, 4): 1.0e10})
    c = capi.tune(g, pass_words=1 << 14, probe=t)
    assert [(m, k) for m, k, _ in t.calls] == CANDIDATES
    assert c["from_cache"] == 0 and c["candidates"] == len(CANDIDATES)
    assert (c["mode"], c["ctas_per_sm"]) == (capi.MODE_STAGED, 0) and c["words_per_second"] == 2.5e10
    assert all(w == c["probe_words"] for _, _, w in t.calls)
    assert c["probe_words"] == 1 << 14  # short passes are probed at their own length


def test_hit_in_memory_then_from_the_file(cache):
    g = synth.config1()
    t = FakeTimer({(capi.MODE_STRIP, 5): 3.0e10, (capi.MODE_FUSED, 2): 1.0e10})
    first = capi.tune(g, probe=t)
    assert (first["mode"], first["ctas_per_sm"]) == (capi.MODE_STRIP, 5)
    n = len(t.calls)
    again = capi.tune(g, probe=t)
    assert len(t.calls) == n and again["from_cache"] == 1 and again["key"] == first["key"]
    assert (again["mode"], again["ctas_per_sm"]) == (capi.MODE_STRIP, 5)
    assert cache.exists() and cache.read_text().startswith("mcg-tune-1")
    capi.tune_forget()  # a new process: memory empty, file kept
    reread = capi.tune(g, probe=t)
    assert len(t.calls) == n and reread["from_cache"] == 1
    assert (reread["mode"], reread["ctas_per_sm"], reread["words_per_second"]) == (capi.MODE_STRIP, 5, 3.0e10)


def test_key_follows_shape_and_pass_length_not_probabilities(cache):
    g = synth.config1()
    t = FakeTimer({(capi.MODE_STRIP, 6): 1.0})
    a = capi.tune(g, probe=t)
    # other probabilities, same structure: same entry
    rng = np.random.default_rng(3)
    other_p = g.with_thresholds((rng.uniform(0.01, 0.3, g.n_be) * 2 ** 32).astype(np.uint64))
    b = capi.tune(other_p, probe=t)
    assert b["key"] == a["key"] and b["from_cache"] == 1
    # another pass length bucket, another tree, another tally list: new entries
    c = capi.tune(g, pass_words=1 << 12, probe=t)
    d = capi.tune(synth.small_tree(4, n_be=30, n_gates=14), probe=t)
    e = capi.tune(g.with_tallies([g.root]), probe=t)
    assert len({a["key"], c["key"], d["key"], e["key"]}) == 4
    assert c["from_cache"] == d["from_cache"] == e["from_cache"] == 0


def test_no_runnable_candidate_is_an_error(cache):
    g = synth.config1()
    with pytest.raises(capi.McgError) as exc:
        capi.tune(g, probe=FakeTimer({}))
    assert "no candidate" in str(exc.value)


def test_large_tree_probes_shorter_passes(cache):
    g = synth.config2()
    t = FakeTimer({(capi.MODE_STRIP, 6): 1.0})
    c = capi.tune(g, pass_words=1 << 24, probe=t)
    assert c["probe_words"] == 1 << 20 and c["probe_words"] % 256 == 0


def test_memory_only_cache_writes_no_file(tmp_path):
    capi.tune_set_cache_file("")
    capi.tune_forget()
    try:
        t = FakeTimer({(capi.MODE_FUSED, 4): 1.0})
        capi.tune(synth.config1(), probe=t)
        assert not any(tmp_path.iterdir())
    finally:
        capi.tune_forget()


@pytest.mark.gpu
def test_tuned_engine_matches_oracle(oracle_mod, gpu, tmp_path):
    """A zero-initialised run description (MCG_MODE_AUTO) tunes on the GPU,
    builds the chosen engine, and its tallies are the oracle's; a second
    engine of the same shape takes the cached choice."""
    capi.tune_set_cache_file(str(tmp_path / "tune.txt"))
    capi.tune_forget()
    try:
        for g, words in ((synth.config1(), 1 << 14), (synth.small_tree(9, n_be=40, n_gates=20), 3000)):
            c = capi.tune(g, pass_words=words)
            assert c["from_cache"] == 0 and c["words_per_second"] > 0
            with capi.Engine(g, mode=capi.MODE_AUTO, tune_pass_words=words) as e:
                assert e.launch_shape() == (c["mode"], c["ctas_per_sm"])
                e.run(3, 1, 11, words)
                ones, total = e.tallies()
            assert total == words * 64
            assert np.array_equal(ones, oracle_mod.tallies(g, 3, 1, 11, words))
            assert capi.tune(g, pass_words=words)["from_cache"] == 1
    finally:
        capi.tune_set_cache_file("")
        capi.tune_forget()


@pytest.mark.gpu
def test_tuned_compute_tallies_close_to_strip_on_the_large_tree(gpu, tmp_path):
    """On the 5,000-event tree at 2^24-word passes the tuner's choice runs
    within 3 % of the strip kernel (the fastest measured engine there)."""
    capi.tune_set_cache_file(str(tmp_path / "tune.txt"))
    capi.tune_forget()
    try:
        g = synth.config2()
        c = capi.tune(g, pass_words=1 << 24)
        words = 1 << 21
        rates = {}
        for name, kw in (("strip", dict(mode=capi.MODE_STRIP)),
                         ("tuned", dict(mode=capi.MODE_AUTO, tune_pass_words=1 << 24))):
            with capi.Engine(g, **kw) as e:
                e.run(1, 1, 0, words)
                e.synchronize()
                rates[name] = 1.0 / e.time_runs(2, 0, words, 2)
        assert rates["tuned"] >= 0.97 * rates["strip"], (c, rates)
    finally:
        capi.tune_set_cache_file("")
        capi.tune_forget()
