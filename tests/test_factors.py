"""Monte Carlo importance factors: the tallies behind them are exact counts
of the oracle's words, and the factors agree with the exact ones computed
from BDD conditionals (P(top | x=1), P(top | x=0)) within their sampling
error, using the reference's relations between the factors."""
import numpy as np
import pytest

from mcscram_b200 import synth

pytestmark = pytest.mark.gpu


def test_joint_counts_match_oracle_words(oracle_mod, gpu):
    from mcscram_b200.factors import importance_factors
    g = synth.config1()
    W = 3000
    f = importance_factors(g, words=W, iteration=2)
    words = oracle_mod.eval_words(g, 2, 0, W)
    top = words[g.root]
    n = W * 64
    assert f[0]["p_top"] * n == pytest.approx(sum(bin(int(x)).count("1") for x in top), abs=1e-6)
    for i in range(0, g.n_be, 17):
        joint = sum(bin(int(a) & int(b)).count("1") for a, b in zip(top, words[i]))
        assert f[i]["p_joint"] * n == pytest.approx(joint, abs=1e-6)
        assert f[i]["samples"] == n and f[i]["event"] == i


def test_factors_match_exact_conditionals(oracle_mod, gpu):
    from mcscram_b200.factors import importance_factors
    g = synth.small_tree(1, n_be=24, n_gates=12, n_layers=4, p_range=(0.05, 0.4))
    p = g.quantised_probabilities()
    P = oracle_mod.bdd_probability(g)
    events = list(range(0, g.n_be, 3))
    W = 1 << 22
    f = importance_factors(g, events=events, words=W)
    n = W * 64
    for r, i in zip(f, events):
        q1, q0 = p.copy(), p.copy()
        q1[i], q0[i] = 1.0, 0.0
        P1, P0 = oracle_mod.bdd_probability(g, p=q1), oracle_mod.bdd_probability(g, p=q0)
        mif = P1 - P0
        # mif = T/p - U/(1-p) with T = P(top, x=1), U = P(top, x=0): multinomial counts
        # of disjoint outcomes of the same samples, so Cov(T, U) = -T U / n
        T, U = p[i] * P1, (1 - p[i]) * P0
        se = np.sqrt((T * (1 - T) / p[i] ** 2 + U * (1 - U) / (1 - p[i]) ** 2 + 2 * T * U / (p[i] * (1 - p[i]))) / n)
        assert abs(r["mif"] - mif) <= 5 * se + 1e-12, (i, r["mif"], mif, se)
        assert r["p"] == pytest.approx(p[i], rel=1e-15)
        assert r["p_top"] == pytest.approx(P, abs=5 * np.sqrt(P * (1 - P) / n))
        # the reference's relations, applied to the exact values
        raw = 1 + (1 - p[i]) * mif / P
        assert r["raw"] == pytest.approx(raw, abs=6 * (1 - p[i]) * se / P + 1e-9)
        assert r["dif"] == pytest.approx(p[i] * raw, abs=6 * p[i] * (1 - p[i]) * se / P + 1e-9)
        assert r["cif"] == pytest.approx(p[i] * mif / P, abs=6 * p[i] * se / P + 1e-9)
