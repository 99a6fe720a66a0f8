"""The reference-shaped host API on the GPU: layer_manager passes and tallies
bit-exact against the oracle (using the event_idx the layering assigns), the
convergence loop with both policies, and ComputeTallies."""
import numpy as np
import pytest

from mcscram_b200 import host, synth

pytestmark = pytest.mark.gpu


def c1_pdag():
    g0 = synth.config1()
    return g0, host.Pdag.from_flat(g0)


def test_manager_passes_match_oracle(oracle_mod, gpu):
    g0, p = c1_pdag()
    tally = [int(x) for x in g0.gate_pdag_idx]
    with host.LayerManager(p, 1 << 20, tally) as m:
        assert m.shape() == {"batch_size": 1, "bitpacks_per_batch": 16384, "total_iterations": 1}
        assert m.node_count() == g0.n_nodes
        got = m.pass_wait_collect(3, 2)
    flat = p.flatten(tally)
    expect = oracle_mod.tallies(flat, 1, 3, 0, 16384)
    for i, idx in enumerate(tally):
        assert got[idx]["num_one_bits"] == int(expect[i])
        assert got[idx]["total_bits"] == 3 * 16384 * 64


def test_single_pass_and_tally(oracle_mod, gpu):
    g0, p = c1_pdag()
    root = int(g0.gate_pdag_idx[-1])
    with host.LayerManager(p, 1 << 20, [root]) as m:
        t1 = m.single_pass_and_tally(root)
        t2 = m.single_pass_and_tally(root)
    flat = p.flatten([root])
    e1 = oracle_mod.tallies(flat, 1, 1, 0, 16384)[0]
    e2 = oracle_mod.tallies(flat, 1, 2, 0, 16384)[0]
    assert t1["num_one_bits"] == int(e1) and t1["total_bits"] == 16384 * 64
    assert t2["num_one_bits"] == int(e2) and t2["total_bits"] == 2 * 16384 * 64
    assert t2["mean"] == pytest.approx(int(e2) / (2 * 16384 * 64))


@pytest.mark.parametrize("policy", [host.POLICY_WALD, host.POLICY_BAYES])
def test_run_to_convergence(oracle_mod, gpu, policy):
    g0, p = c1_pdag()
    exact = oracle_mod.bdd_probability(g0)
    root = int(g0.gate_pdag_idx[-1])
    s = host.Settings.default(policy=policy, ci_rel_margin_error=0.01, ci_confidence=0.99,
                              ci_burnin_trials=float(1 << 20))
    with host.LayerManager(p, 0, [root], max_words_per_iteration=1 << 16) as m:
        tallies, rep = m.run_to_convergence(s)
    t = tallies[root]
    assert rep["epsilon_converged"] and rep["log10_converged"]
    assert rep["epsilon"] <= rep["target_epsilon"] * (1 + 1e-12)
    # stopped with a relative half-width <= 1%: the estimate is within it (plus slack) of the exact value
    assert abs(t["mean"] - exact) <= 3 * t["std_err"] + 1e-12
    assert rep["trials"] == t["total_bits"]


def test_fixed_trial_budget_stops(oracle_mod, gpu):
    g0, p = c1_pdag()
    root = int(g0.gate_pdag_idx[-1])
    s = host.Settings.default(num_trials=4 << 20, early_stop=0, ci_rel_margin_error=1e-6,
                              ci_burnin_trials=float(1 << 20))
    with host.LayerManager(p, 4 << 20, [root], max_words_per_iteration=1 << 14) as m:
        tallies, rep = m.run_to_convergence(s)
    assert rep["iteration_limit_reached"] == 1
    assert tallies[root]["total_bits"] == 4 << 20


def test_compute_tallies_root_first(oracle_mod, gpu):
    g0, p = c1_pdag()
    watch = [int(g0.gate_pdag_idx[5]), int(g0.gate_pdag_idx[17])]
    s = host.Settings.default(ci_rel_margin_error=0.05, ci_burnin_trials=float(1 << 20))
    out, rep = host.compute_tallies(p, s, watch)
    assert out[0]["index"] == int(g0.gate_pdag_idx[-1])
    assert [o["index"] for o in out[1:]] == watch
    exact = oracle_mod.bdd_probability(g0)
    assert abs(out[0]["mean"] - exact) <= 3 * out[0]["std_err"] + 1e-12


@pytest.mark.parametrize("case", ["bayes", "wald", "fixed"])
def test_pipelined_loop_equals_waiting_loop(gpu, case):
    """Judging pass k while pass k + 1 runs gives the waiting loop's tallies,
    statistics and stopping point."""
    g0, p = c1_pdag()
    root = int(g0.gate_pdag_idx[-1])
    kw = dict(policy=host.POLICY_WALD if case == "wald" else host.POLICY_BAYES, ci_rel_margin_error=0.01,
              ci_burnin_trials=float(1 << 20))
    budget = 0
    if case == "fixed":
        kw.update(num_trials=3 << 20, early_stop=0, ci_rel_margin_error=1e-6)
        budget = 3 << 20
    out = []
    for pipelined in (0, 1):
        s = host.Settings.default(pipelined=pipelined, **kw)
        with host.LayerManager(p, budget, [root], max_words_per_iteration=1 << 14) as m:
            tallies, rep = m.run_to_convergence(s)
            out.append((tallies, {k: v for k, v in rep.items() if k != "seconds"}))
    assert out[0][0] == out[1][0]
    assert out[0][1] == out[1][1]
    assert out[1][1]["steps"] + out[1][1]["burn_in_steps"] >= 2
