"""Learned importance sampling: the FP64 likelihood-ratio estimator, the
proposal MLP against an FP64 oracle, and the cross-entropy-trained proposal
on the rare-event tree against the exact BDD probability."""
import numpy as np
import pytest

from mcscram_b200 import synth
from mcscram_b200.graph import probability_threshold
from oracle import mlp_oracle

TWO32 = float(1 << 32)


def test_mlp_oracle_gradient_by_finite_differences():
    rng = np.random.default_rng(0)
    p = rng.normal(0, 0.3, mlp_oracle.IN * mlp_oracle.HID + 2 * mlp_oracle.HID + mlp_oracle.HID ** 2 +
                   mlp_oracle.HID + 1)
    X = rng.normal(0, 1, (20, 16))
    t = rng.uniform(0, 1, 20)
    w = rng.uniform(0.5, 2, 20)
    loss, g = mlp_oracle.loss_and_grad(p, X, t, w)
    for idx in rng.choice(p.size, 25, replace=False):
        h = 1e-6
        pp, pm = p.copy(), p.copy()
        pp[idx] += h
        pm[idx] -= h
        fd = (mlp_oracle.loss_and_grad(pp, X, t, w)[0] - mlp_oracle.loss_and_grad(pm, X, t, w)[0]) / (2 * h)
        assert fd == pytest.approx(g[idx], rel=1e-4, abs=1e-8)


def test_event_features_shape():
    from mcscram_b200.importance import event_features
    g = synth.config4()
    f = event_features(g)
    assert f.shape == (g.n_be, 16) and f.dtype == np.float32
    assert np.all(np.isfinite(f)) and np.all(f[:, 15] == 1.0)


def _words_and_weights(oracle_mod, g, q, it, W):
    """CPU log-weights for every top failure of the words drawn with q."""
    gq = g.with_thresholds(q)
    words = oracle_mod.eval_words(gq, it, 0, W)
    p = g.quantised_probabilities()
    qq = q.astype(np.float64) / TWO32
    a = np.log(p) - np.log(qq) - (np.log1p(-p) - np.log1p(-qq))
    C = float((np.log1p(-p) - np.log1p(-qq)).sum())
    bits = ((words[: g.n_be, :, None] >> np.arange(64, dtype=np.uint64)) & np.uint64(1)).astype(np.float64)
    top = ((words[g.root][:, None] >> np.arange(64, dtype=np.uint64)) & np.uint64(1)).astype(bool)
    logw = C + np.einsum("i,iwb->wb", a, bits)
    wgt = np.where(top, np.exp(logw), 0.0)
    return wgt, bits, top


@pytest.mark.gpu
def test_unbiased_proposal_reproduces_plain_tally(capi, oracle_mod, gpu):
    from mcscram_b200.importance import ImportanceSampler
    g = synth.config1()
    with ImportanceSampler(g) as s:
        r = s.run(g.be_threshold, iteration=1, word_count=16384)
    plain = int(oracle_mod.tallies(g.with_tallies([g.root]), 1, 1, 0, 16384)[0])
    assert r["hits"] == plain
    assert r["sum_w"] == pytest.approx(plain, rel=1e-12)
    assert r["estimate"] == pytest.approx(plain / (16384 * 64), rel=1e-12)


@pytest.mark.gpu
def test_weights_match_cpu(oracle_mod, gpu):
    from mcscram_b200.importance import ImportanceSampler
    g = synth.small_tree(4, n_be=40, n_gates=24, n_layers=5, p_range=(1e-3, 0.05))
    rng = np.random.default_rng(3)
    q = probability_threshold(np.minimum(g.quantised_probabilities() * rng.uniform(2, 20, g.n_be), 0.5))
    W = 700
    with ImportanceSampler(g, chunk_words=256) as s:
        r = s.run(q, iteration=3, word_count=W, ce=True)
    wgt, bits, top = _words_and_weights(oracle_mod, g, q, 3, W)
    assert r["hits"] == int(top.sum())
    assert r["sum_w"] == pytest.approx(wgt.sum(), rel=1e-10)
    assert r["sum_w2"] == pytest.approx((wgt ** 2).sum(), rel=1e-10)
    ce = np.einsum("wb,iwb->i", wgt, bits)
    np.testing.assert_allclose(r["ce_num"], ce, rtol=1e-10, atol=1e-300)


def _rand_params(seed):
    rng = np.random.default_rng(seed)
    p = np.zeros(16 * 64 + 64 + 64 * 64 + 64 + 64 + 1)
    p[:1024] = rng.normal(0, np.sqrt(2 / 16), 1024)
    p[1024:1088] = rng.normal(0, 0.05, 64)
    p[1088:5184] = rng.normal(0, np.sqrt(2 / 64), 4096)
    p[5184:5248] = rng.normal(0, 0.05, 64)
    p[5248:5312] = rng.normal(0, np.sqrt(1 / 64), 64)
    p[5312] = -1.0
    return p.astype(np.float32)


@pytest.mark.gpu
def test_mlp_forward_and_gradient_match_oracle(gpu):
    from mcscram_b200.importance import ProposalMLP
    rng = np.random.default_rng(1)
    n = 1000  # not a multiple of the 64-row tiles
    X = rng.normal(0, 1, (n, 16)).astype(np.float32)
    t = rng.uniform(0, 0.5, n).astype(np.float32)
    w = rng.uniform(0.1, 3, n).astype(np.float32)
    params = _rand_params(5)
    m = ProposalMLP()
    m.set_params(params)
    q = m.forward(X)
    q_ref, _ = mlp_oracle.forward(params, X, bf=True)
    np.testing.assert_allclose(q, q_ref, atol=2e-3)
    q_exact, _ = mlp_oracle.forward(params, X, bf=False)
    np.testing.assert_allclose(q, q_exact, atol=3e-2)
    g, loss = m.grad(X, t, w)
    loss_ref, g_ref = mlp_oracle.loss_and_grad(params, X, t, w, bf=True)
    assert loss == pytest.approx(loss_ref, rel=1e-3)
    assert np.linalg.norm(g - g_ref) <= 1e-2 * np.linalg.norm(g_ref)
    _, g_exact = mlp_oracle.loss_and_grad(params, X, t, w, bf=False)
    cos = float(g @ g_exact / (np.linalg.norm(g) * np.linalg.norm(g_exact)))
    assert cos > 0.995
    m.close()


@pytest.mark.gpu
def test_mlp_training_reduces_loss(gpu):
    from mcscram_b200.importance import ProposalMLP
    rng = np.random.default_rng(2)
    X = rng.normal(0, 1, (2000, 16)).astype(np.float32)
    t = (1 / (1 + np.exp(-(X[:, 0] - 2 * X[:, 3])))).astype(np.float32)
    m = ProposalMLP(seed=3)
    _, l0 = m.grad(X, t)
    l1 = m.train(X, t, steps=400, lr=3e-3)
    assert l1 < 0.97 * l0
    m.close()


@pytest.mark.gpu
def test_cross_entropy_proposal_on_rare_tree(oracle_mod, gpu):
    from mcscram_b200.importance import ImportanceSampler, cross_entropy, estimate, initial_proposal
    g = synth.config4()
    exact = oracle_mod.bdd_probability(g)
    assert 5e-9 < exact < 2e-8
    with ImportanceSampler(g) as s:
        q, mlp, hist = cross_entropy(g, rounds=4, words_per_round=1 << 18, sampler=s)
        res = estimate(s, q, target_rel_err=0.05, words_per_batch=1 << 18, max_words=1 << 24)
        assert not res["fallback"]
        assert abs(res["estimate"] - exact) <= 3 * res["std_err"] + 1e-15, (res, exact)
        # the trained proposal against the untrained (uniformly inflated) one at equal samples
        q0, _, _ = initial_proposal(s, g.quantised_probabilities())
        base = s.run(s.proposal_thresholds(q0), iteration=500, word_count=1 << 18)
        trained = s.run(s.proposal_thresholds(q), iteration=501, word_count=1 << 18)
        assert trained["rel_err"] < base["rel_err"]
    mlp.close()
