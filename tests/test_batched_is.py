"""Batched learned importance sampling over many rare-event trees.

CPU: the joined graph evaluates every tree exactly as the tree alone (same
counters), the vectorised features and exact read-once probabilities agree
with their direct definitions, the rare-event instance generator meets its
ranges, and the row gather that feeds the shared network works across two
gloo ranks.  GPU: per-tree FP64 sums and cross-entropy numerators against
the CPU, the unbiased proposal against plain tallies, and the whole batched
pipeline against the exact probabilities."""
import os
import socket

import numpy as np
import pytest

from mcscram_b200 import graph as G
from mcscram_b200 import synth
from mcscram_b200.graph import AND, ATLEAST, OR, XOR, probability_threshold

TWO32 = float(1 << 32)


def _small_rare(seed, n_be=60, n_gates=30, p_range=(1e-3, 0.05)):
    return synth.generate(synth.TreeSpec(n_be=n_be, n_gates=n_gates, mix={AND: 0.5, OR: 0.3, ATLEAST: 0.2},
                                         p_range=p_range, seed=seed, atleast_n=(3, 4), n_layers=5))


def _trees():
    return [_small_rare(1), synth.small_tree(4, n_be=40, n_gates=24, n_layers=5, p_range=(1e-3, 0.05)),
            _small_rare(7, n_be=37, n_gates=18)]


def test_concat_evaluates_each_tree_as_alone(oracle_mod):
    trees = _trees()
    u, bb, roots = G.concat(trees)
    u.validate()
    assert u.n_be == sum(t.n_be for t in trees) and u.n_gates == sum(t.n_gates for t in trees)
    assert list(bb) == [0] + list(np.cumsum([t.n_be for t in trees]))
    W = 300
    wu = oracle_mod.eval_words(u, 2, 5, W)
    g0 = u.n_be
    for k, t in enumerate(trees):
        # the same tree with the counters its events have in the union
        tk = t.with_tallies(t.tally_nodes)
        tk.be_pdag_idx = u.be_pdag_idx[bb[k]:bb[k + 1]].copy()
        tk.be_event_idx = u.be_event_idx[bb[k]:bb[k + 1]].copy()
        wk = oracle_mod.eval_words(tk, 2, 5, W)
        assert np.array_equal(wk[: t.n_be], wu[bb[k]:bb[k + 1]])
        assert np.array_equal(wk[t.n_be:], wu[g0:g0 + t.n_gates])
        assert np.array_equal(wk[t.root], wu[roots[k]])
        g0 += t.n_gates


def _event_features_direct(g):
    """The features by their definition, one event at a time."""
    from mcscram_b200.importance import N_FEATURES
    nb, ng = g.n_be, g.n_gates
    depth = g.layers()
    L = max(int(depth.max()), 1)
    parents = [[] for _ in range(g.n_nodes)]
    for gi in range(ng):
        for c in g.gate_inputs(gi):
            parents[int(c)].append(gi)
    logp = np.log10(np.clip(g.quantised_probabilities(), 1e-12, 1.0))
    up = np.zeros((ng, 3))
    for gi in range(ng - 1, -1, -1):
        ps = parents[nb + gi]
        if ps:
            q = ps[0]
            up[gi] = up[q] + [g.gate_op[q] == AND, g.gate_op[q] == OR, 1]
    f = np.zeros((nb, N_FEATURES), dtype=np.float32)
    for e in range(nb):
        ps = parents[e]
        f[e, 0] = (logp[e] + 4.0) / 2.0
        f[e, 1] = len(ps) / 4.0
        f[e, 15] = 1.0
        if not ps:
            continue
        d = [depth[nb + q] for q in ps]
        ops = [int(g.gate_op[q]) for q in ps]
        f[e, 2], f[e, 3] = min(d) / L, max(d) / L
        f[e, 4:7] = [np.mean([o == x for o in ops]) for x in (AND, OR, ATLEAST)]
        f[e, 7] = np.mean([int(g.gate_in_count[q]) for q in ps]) / 8.0
        kn = [int(g.gate_k[q]) / max(int(g.gate_in_count[q]), 1) for q in ps if g.gate_op[q] == ATLEAST]
        f[e, 8] = np.mean(kn) if kn else 0.0
        sib = [int(c) for c in g.gate_inputs(ps[0]) if int(c) != e]
        f[e, 9] = len(sib) / 8.0
        sb = [logp[c] for c in sib if c < nb]
        f[e, 10] = (np.mean(sb) + 4.0) / 2.0 if sb else 0.0
        f[e, 11] = np.mean([c >= nb for c in sib]) if sib else 0.0
        f[e, 12] = float(max(d) == L)
        f[e, 13] = up[ps[0], 0] / max(up[ps[0], 2] + 1, 1)
        f[e, 14] = up[ps[0], 1] / max(up[ps[0], 2] + 1, 1)
    return f


@pytest.mark.parametrize("make", [synth.config1, lambda: synth.small_tree(3), lambda: synth.config5(1, first=3)[0]])
def test_event_features_match_definition(make):
    from mcscram_b200.importance import event_features
    g = make()
    np.testing.assert_allclose(event_features(g), _event_features_direct(g), rtol=0, atol=1e-6)
    f = event_features(g, instance_scale=1e3)
    assert np.all(f[:, 15] == np.float32(0.5))


def _cond_by_definition(g, node):
    """P(x_i = 1 | node fails) of a read-once tree, one event at a time."""
    p = g.quantised_probabilities()
    P = synth.read_once_probability(g, p)[node]
    out = np.empty(g.n_be)
    for i in range(g.n_be):
        pp = p.copy()
        pp[i] = 1.0
        out[i] = p[i] * synth.read_once_probability(g, pp)[node] / P
    return out


@pytest.mark.parametrize("seed", range(4))
def test_approximate_importance_is_exact_on_trees(seed):
    from mcscram_b200.importance import approximate_importance
    g = synth.generate(synth.TreeSpec(n_be=40, n_gates=20, mix={AND: 0.3, OR: 0.3, ATLEAST: 0.2, XOR: 0.1,
                                                               synth.NOT: 0.1},
                                      p_range=(1e-4, 0.5), seed=seed, atleast_n=(3, 5)))
    pr, cond = approximate_importance(g)
    np.testing.assert_allclose(pr, synth.read_once_probability(g), rtol=1e-12)
    np.testing.assert_allclose(cond, _cond_by_definition(g, g.root), rtol=1e-9, atol=1e-14)
    child = int(g.gate_inputs(g.root - g.n_be)[0])
    if child >= g.n_be:
        _, cond_c = approximate_importance(g, root=child)
        np.testing.assert_allclose(cond_c, _cond_by_definition(g, child), rtol=1e-9, atol=1e-14)


@pytest.mark.parametrize("n_be,n_gates,seed", [(40, 20, 7), (24, 12, 0), (24, 12, 1)])
def test_approximate_importance_sensitivities_match_finite_differences(n_be, n_gates, seed):
    """On DAGs with shared nodes and wide ATLEAST gates the independence pass
    is an approximation, but its reverse-mode sensitivities must still be
    the derivatives of its own P~_top: cond_i = p_i + p_i (1 - p_i) d log P~ / d p_i."""
    from mcscram_b200.importance import approximate_importance
    g = synth.small_tree(seed, n_be=n_be, n_gates=n_gates, n_layers=4, share_node_frac=0.3, atleast_n=(3, 6),
                         p_range=(0.05, 0.6))
    assert int((np.bincount(g.inputs, minlength=g.n_nodes) > 1).sum()) > 0  # a DAG, not a tree
    assert int(((g.gate_op == ATLEAST) & (g.gate_in_count >= 5)).sum()) > 0
    pr, cond = approximate_importance(g)
    p = g.quantised_probabilities()
    top = pr[g.root]
    h = 1e-6
    for i in range(g.n_be):
        if not 0.0 < p[i] < 1.0:
            continue
        up, dn = p.copy(), p.copy()
        up[i] += h
        dn[i] -= h
        pu = approximate_importance(_with_probabilities(g, up))[0][g.root]
        pd = approximate_importance(_with_probabilities(g, dn))[0][g.root]
        dlog = (pu - pd) / (2 * h) / top
        assert cond[i] == pytest.approx(np.clip(p[i] + p[i] * (1 - p[i]) * dlog, 0, 1), rel=1e-5, abs=1e-8), i


def _with_probabilities(g, p):
    """The graph with basic-event probabilities p taken exactly (thresholds
    p * 2^32 represent them to the precision the check needs)."""
    out = g.with_thresholds(probability_threshold(p))
    out.quantised_probabilities = lambda p=p: np.asarray(p, dtype=np.float64)
    return out


def test_prepare_trees_on_an_executor_equals_serial():
    from concurrent.futures import ThreadPoolExecutor

    from mcscram_b200.importance import prepare_trees
    trees = [synth.config5_instance(i) for i in range(3)] + [synth.config5_dag_instance(5)]
    serial = prepare_trees(trees, 4, True, 0)
    with ThreadPoolExecutor(max_workers=2) as ex:
        pooled = prepare_trees(trees, 4, True, ex)
        made = synth.config5_instances([1, 3], workers=ex)
    for (f0, m0, z0, s0), (f1, m1, z1, s1) in zip(serial, pooled):
        assert np.array_equal(f0, f1) and np.array_equal(m0, m1)
        assert (z0 is None) == (z1 is None) and (z0 is None or np.array_equal(z0, z1))
        assert (s0 is None) == (s1 is None) and (s0 is None or np.array_equal(s0, s1))
    assert serial[0][2] is None and serial[3][2] is not None  # shared-event posteriors for the DAG only
    assert serial[3][3] is None  # the heuristic seed only where the posteriors cannot be computed
    assert np.array_equal(made[1].be_threshold, synth.config5_instance(3).be_threshold)


def test_prepare_trees_async_keeps_the_order_of_the_trees():
    """The pipeline submits the trees largest first and collects them back in
    the caller's order: the same inputs as the serial path, tree for tree."""
    from concurrent.futures import ThreadPoolExecutor

    from mcscram_b200.importance import prepare_trees, prepare_trees_async
    trees = [synth.config5_dag_instance(i) for i in (5, 0, 3)] + [synth.config5_instance(2)]
    assert len({t.n_be for t in trees}) == len(trees)  # distinct sizes: the submission order differs
    serial = prepare_trees(trees, 4, True, 0)
    with ThreadPoolExecutor(max_workers=3) as ex:
        collect = prepare_trees_async(trees, 4, True, ex)
        pooled = collect()
    assert len(pooled) == len(trees)
    for a, b in zip(serial, pooled):
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
        for x, y in zip(a[2:], b[2:]):
            assert (x is None) == (y is None) and (x is None or np.array_equal(x, y))


def test_mode_proposals_condition_on_top_children():
    from mcscram_b200.importance import approximate_importance, mode_proposals
    g = synth.config5_instance(0)
    kids = [int(c) for c in g.gate_inputs(g.root - g.n_be)]
    m = mode_proposals(g, 4, 0.5)
    assert m.shape == (4, g.n_be) and np.all((m >= 1e-7) & (m <= 0.5))
    pr, _ = approximate_importance(g)
    heaviest = max(kids, key=lambda c: pr[c])
    np.testing.assert_allclose(m[0], np.clip(approximate_importance(g, root=heaviest)[1], 1e-7, 0.5))


def test_layers_match_definition():
    for g in (synth.config1(), synth.small_tree(5, n_be=48, n_gates=24, n_layers=5)):
        ref = np.zeros(g.n_nodes, dtype=np.int64)
        for j in range(g.n_gates):
            ins = g.gate_inputs(j)
            ref[g.n_be + j] = 1 + (int(ref[ins].max()) if ins.size else 0)
        assert np.array_equal(g.layers(), ref)


@pytest.mark.parametrize("seed", range(5))
def test_read_once_probability_matches_bdd(oracle_mod, seed):
    g = synth.generate(synth.TreeSpec(n_be=40, n_gates=20, mix={AND: 0.3, OR: 0.3, ATLEAST: 0.2, XOR: 0.1,
                                                               synth.NOT: 0.1},
                                      p_range=(1e-4, 0.5), seed=seed, atleast_n=(3, 5)))
    pr = synth.read_once_probability(g)
    assert pr[g.root] == pytest.approx(oracle_mod.bdd_probability(g), rel=1e-12)


def test_config5_instances_meet_their_ranges(oracle_mod):
    gs = synth.config5(6, first=0)
    for i, g in enumerate(gs):
        assert 50 <= g.n_be <= 10000
        t = g.meta["target_p_top"]
        assert 1e-10 <= t <= 1e-5
        assert abs(np.log(g.meta["exact_p_top"] / t)) < 0.011
        ops = np.bincount(g.gate_op, minlength=8) / g.n_gates
        assert (ops[AND] > 0.5) if i % 2 == 0 else (ops[ATLEAST] > 0.3)
        assert np.all(np.bincount(g.inputs, minlength=g.n_nodes) <= 1)  # read-once
        if g.n_be <= 1500:
            assert g.meta["exact_p_top"] == pytest.approx(oracle_mod.bdd_probability(g), rel=1e-9)
    # an instance does not depend on the others built with it
    assert np.array_equal(synth.config5(1, first=4)[0].be_threshold, gs[4].be_threshold)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _gather_main(rank, world, port, queue):
    import torch.distributed as dist
    from mcscram_b200 import parallel
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    n = 3 + 4 * rank  # uneven row counts
    f = np.full((n, 16), rank, dtype=np.float32) + np.arange(n, dtype=np.float32)[:, None]
    t = np.full(n, 10 + rank, dtype=np.float32)
    F, T = parallel.allgather_rows(f, t)
    params = parallel.broadcast_params(np.full(5, rank + 1.0, dtype=np.float32))
    queue.put((rank, F, T, params))
    dist.barrier()
    dist.destroy_process_group()


def test_gloo_row_gather_and_param_broadcast():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_gather_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, F, T, params in got:
        assert F.shape == (3 + 7, 16) and T.shape == (10,)
        assert np.array_equal(T, [10] * 3 + [11] * 7)
        assert np.array_equal(F[:3, 0], [0, 1, 2]) and np.array_equal(F[3:, 0], 1 + np.arange(7))
        assert np.array_equal(params, np.ones(5, dtype=np.float32))


# ----------------------------------------------------------------------------- GPU

def _log_ratio(p, thr, bits, s):
    q = thr.astype(np.float64) / TWO32
    l1 = np.log1p(-p) - np.log1p(-q)
    a = np.log(p) - np.log(q) - l1
    return l1[s].sum() + np.einsum("i,iwb->wb", a[s], bits[s])


def _union_weights(oracle_mod, u, bb, roots, comps, it):
    """Per-tree CPU sums and per-event CE numerators of the joined graph.
    comps = [(thresholds, words), ...] in drawing order; with more than one
    component every sample gets the balance-heuristic weight."""
    W = sum(wc for _, wc in comps)
    parts, pos = [], 0
    for thr, wc in comps:
        if wc:
            parts.append(oracle_mod.eval_words(u.with_thresholds(thr), it, pos, wc))
        pos += wc
    words = np.concatenate(parts, axis=1)
    p = u.quantised_probabilities()
    bits = ((words[: u.n_be, :, None] >> np.arange(64, dtype=np.uint64)) & np.uint64(1)).astype(np.float64)
    live = [(thr, wc) for thr, wc in comps if wc]
    sums, ce = [], np.zeros(u.n_be)
    for k in range(len(roots)):
        s = slice(int(bb[k]), int(bb[k + 1]))
        top = ((words[roots[k]][:, None] >> np.arange(64, dtype=np.uint64)) & np.uint64(1)).astype(bool)
        lws = [_log_ratio(p, thr, bits, s) for thr, _ in live]
        if len(live) == 1:
            logw = lws[0]
        else:
            logw = -np.logaddexp.reduce([np.log(wc / W) - lw for (_, wc), lw in zip(live, lws)], axis=0)
        w = np.where(top, np.exp(logw), 0.0)
        sums.append((w.sum(), (w ** 2).sum(), int(top.sum()), logw[top].max() if top.any() else -np.inf))
        ce[s] = np.einsum("wb,iwb->i", w, bits[s])
    return sums, ce


@pytest.mark.gpu
@pytest.mark.parametrize("wdef", [(), (300,), (120, 0, 250)])
def test_batched_sums_match_cpu(oracle_mod, gpu, wdef):
    from mcscram_b200.importance import BatchedImportanceSampler
    trees = _trees()
    rng = np.random.default_rng(5)
    with BatchedImportanceSampler(trees, chunk_words=256) as s:
        p = s.union.quantised_probabilities()
        q = probability_threshold(np.minimum(p * rng.uniform(2, 30, p.size), 0.5))
        qdef = np.stack([probability_threshold(np.minimum(p * f, 0.5)) for f in (8.0, 3.0, 20.0)])[: len(wdef)]
        W = 700  # chunks of 256 words, the last one short
        r = s.run(q, iteration=4, word_count=W, ce=True, q_defensive=qdef if wdef else None,
                  words_defensive=list(wdef))
        comps = [(q, W - sum(wdef))] + [(qdef[c], wdef[c]) for c in range(len(wdef))]
        sums, ce = _union_weights(oracle_mod, s.union, s.be_begin, s.roots, comps, 4)
    for k, (sw, sw2, h, mx) in enumerate(sums):
        assert r["hits"][k] == h
        assert r["sum_w"][k] == pytest.approx(sw, rel=1e-10)
        assert r["sum_w2"][k] == pytest.approx(sw2, rel=1e-10)
        assert r["max_log_w"][k] == pytest.approx(mx, rel=1e-12)
    np.testing.assert_allclose(r["ce_num"], ce, rtol=1e-10, atol=1e-300)
    assert r["samples"] == W * 64


@pytest.mark.gpu
def test_batched_nominal_proposal_counts_plain_tallies(oracle_mod, gpu):
    from mcscram_b200.importance import BatchedImportanceSampler
    trees = _trees()
    with BatchedImportanceSampler(trees) as s:
        r = s.run(s.union.be_threshold, iteration=1, word_count=5000)
        plain = oracle_mod.tallies(s.union, 1, 1, 0, 5000)  # the union tallies its roots
    assert np.array_equal(r["hits"], plain.astype(np.int64))
    np.testing.assert_allclose(r["sum_w"], plain.astype(np.float64), rtol=1e-12)


@pytest.mark.gpu
def test_batched_create_rejects_bad_partitions(capi, gpu):
    import ctypes as C
    from mcscram_b200 import _capi
    trees = _trees()
    u, bb, roots = G.concat(trees)
    lib = _capi.load()
    import mcscram_b200.importance  # registers the signatures  # noqa: F401
    view = _capi.GraphView(u)
    h = C.c_void_p()
    bad = np.ascontiguousarray([0, int(bb[1]) + 3, int(bb[2]), int(bb[3])], dtype=np.uint32)
    rc = lib.mcg_is_batch_create(C.byref(view.desc), 3, bad.ctypes.data_as(C.POINTER(C.c_uint32)), None, C.byref(h))
    assert rc == _capi.MCG_ERR_INVALID and b"two trees" in lib.mcg_last_error()
    swapped = u.with_tallies(roots[[1, 0, 2]])
    view2 = _capi.GraphView(swapped)
    good = np.ascontiguousarray(bb, dtype=np.uint32)
    rc = lib.mcg_is_batch_create(C.byref(view2.desc), 3, good.ctypes.data_as(C.POINTER(C.c_uint32)), None,
                                 C.byref(h))
    assert rc == _capi.MCG_ERR_INVALID and b"not a node of tree" in lib.mcg_last_error()


def _small_config5(n):
    """The first n instances of the batched rare-event set with at most 600 events."""
    out, i = [], 0
    while len(out) < n:
        g = synth.config5_instance(i)
        if g.n_be <= 600:
            out.append(g)
        i += 1
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("defensive_proposal", ["modes", "cutsets"])
def test_batched_learned_is_reaches_exact(gpu, defensive_proposal):
    from mcscram_b200.importance import BatchedImportanceSampler, batched_learned_is
    trees = _small_config5(6)
    exact = np.array([g.meta["exact_p_top"] for g in trees])
    res = batched_learned_is(trees, target_rel_err=0.05, ce_rounds=6, ce_words=1 << 14, max_est_words=1 << 22,
                             defensive_proposal=defensive_proposal)
    assert res.converged.all() and not res.fallback.any(), [r for r in res.rounds if r["phase"] != "probe"]
    se = res.estimate * res.rel_err95 / 1.96
    assert np.all(np.abs(res.estimate - exact) <= 4 * se), (res.estimate, exact, se)
    assert np.all(res.rel_err95 <= 0.05)
    # what the network adds: at equal samples, its proposal against the probe's uniform inflation
    with BatchedImportanceSampler(trees) as s:
        p = s.union.quantised_probabilities()
        tree_of = np.repeat(np.arange(len(trees)), np.diff(s.be_begin))
        q0 = np.minimum(p * res.scale[tree_of], 0.5)
        W = 1 << 14
        base = s.run(s.proposal_thresholds(q0), iteration=9000, word_count=W)
        learned = s.run(s.proposal_thresholds(res.q), iteration=9001, word_count=W)

    def rel(r):
        n = r["samples"]
        est = r["sum_w"] / n
        var = np.maximum(r["sum_w2"] / n - est ** 2, 0)
        return np.sqrt(var / (n - 1)) / np.where(est > 0, est, np.nan)

    assert np.nanmedian(rel(learned)) < np.nanmedian(rel(base))


# ----------------------------------------------------------------------------- cut-set component

M64 = (1 << 64) - 1


def _mix64(z):
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
    return z ^ (z >> 31)


def _cut_tables(u):
    """S per node, OR cumulative shares, ATLEAST suffix sums E[j][r] (same order of operations as the library)."""
    nb = u.n_be
    S = [0.0] * u.n_nodes
    for i in range(nb):
        t = int(u.be_threshold[i])
        S[i] = 1.0 if t >= (1 << 32) else t / 4294967296.0
    tab = {}
    for j in range(u.n_gates):
        op, n, k = int(u.gate_op[j]), int(u.gate_in_count[j]), int(u.gate_k[j]) & 0xFF
        ins = [int(x) for x in u.gate_inputs(j)]
        if op == AND:
            v = 1.0
            for c in ins:
                v *= S[c]
        elif op == OR:
            v = 0.0
            for c in ins:
                v += S[c]
            cum, t = 0.0, []
            for c in ins:
                cum += S[c]
                t.append(cum / v if v > 0 else 1.0)
            tab[j] = t
        else:  # ATLEAST
            E = [[0.0] * (k + 1) for _ in range(n + 1)]
            E[n][0] = 1.0
            for c in range(n - 1, -1, -1):
                for r in range(k + 1):
                    e = E[c + 1][r]
                    if r > 0:
                        e += S[ins[c]] * E[c + 1][r - 1]
                    E[c][r] = e
            v = E[0][k]
            tab[j] = E
        S[nb + j] = v
    return S, tab


def _descend(u, S, tab, root, base):
    """Events forced for one sample (the library's stack order and draws)."""
    nb = u.n_be
    forced, stack, draw = [], [root], 0

    def unif():
        nonlocal draw
        draw += 1
        return (_mix64((base + draw * 0x9E3779B97F4A7C15) & M64) >> 11) * 2.0 ** -53

    while stack:
        node = stack.pop()
        if node < nb:
            forced.append(node)
            continue
        j = node - nb
        op, n, k = int(u.gate_op[j]), int(u.gate_in_count[j]), int(u.gate_k[j]) & 0xFF
        ins = [int(x) for x in u.gate_inputs(j)]
        if op == OR:
            x = unif()
            c = 0
            while c + 1 < n and x >= tab[j][c]:
                c += 1
            stack.append(ins[c])
        elif op == ATLEAST:
            r = k
            E = tab[j]
            for c in range(n):
                if r == 0:
                    break
                take = n - c == r
                if not take:
                    take = unif() * E[c][r] < S[ins[c]] * E[c + 1][r - 1]
                if take:
                    stack.append(ins[c])
                    r -= 1
        else:
            stack.extend(ins)
    return forced


def _count(u, bits, node):
    """N(x): minimal cut sets inside the sample x (bits[node] = fired)."""
    nb = u.n_be
    if node < nb:
        return 1.0 if bits[node] else 0.0
    if not bits[node]:
        return 0.0
    j = node - nb
    op, k = int(u.gate_op[j]), int(u.gate_k[j]) & 0xFF
    vals = [(_count(u, bits, int(c)) if bits[int(c)] else 0.0) for c in u.gate_inputs(j)]
    if op == AND:
        return float(np.prod(vals))
    if op == ATLEAST:
        dp = [1.0] + [0.0] * k
        for v in vals:
            for r in range(k, 0, -1):
                dp[r] += dp[r - 1] * v
        return dp[k]
    return float(sum(vals))


def _gate_words(u, be_words):
    """All node words from the basic-event words (AND/OR/ATLEAST trees)."""
    W = be_words.shape[1]
    bits = np.zeros((u.n_nodes, W, 64), dtype=bool)
    bits[: u.n_be] = ((be_words[:, :, None] >> np.arange(64, dtype=np.uint64)) & np.uint64(1)).astype(bool)
    for j in range(u.n_gates):
        ins = [int(c) for c in u.gate_inputs(j)]
        op = int(u.gate_op[j])
        v = bits[ins]
        if op == AND:
            r = v.all(axis=0)
        elif op == OR:
            r = v.any(axis=0)
        else:
            r = v.sum(axis=0) >= (int(u.gate_k[j]) & 0xFF)
        bits[u.n_be + j] = r
    return bits


def _cut_trees():
    out = []
    for seed in range(40):
        try:
            g = synth.generate(synth.TreeSpec(n_be=30, n_gates=14, mix={AND: 0.4, OR: 0.3, ATLEAST: 0.3},
                                              p_range=(0.01, 0.2), seed=seed, atleast_n=(3, 4), n_layers=4))
        except ValueError:
            continue
        if np.all(np.bincount(g.inputs, minlength=g.n_nodes) <= 1):
            out.append(g)
        if len(out) == 3:
            return out
    raise AssertionError("no read-once trees generated")


@pytest.mark.gpu
@pytest.mark.parametrize("w_main,w_cut", [(0, 256), (300, 300)])
def test_cut_set_component_matches_cpu(oracle_mod, gpu, w_main, w_cut):
    from mcscram_b200.importance import BatchedImportanceSampler
    trees = _cut_trees()
    it = 7
    with BatchedImportanceSampler(trees, chunk_words=256) as s:
        u, bb, roots = s.union, s.be_begin, s.roots
        p = u.quantised_probabilities()
        q = probability_threshold(np.minimum(p * 6.0, 0.5))
        W = w_main + w_cut
        r = s.run(q, iteration=it, word_count=W, ce=True, words_cutset=w_cut)
    # CPU: main words with q, cut-set words with the nominal thresholds plus forced cut sets
    parts = []
    if w_main:
        parts.append(oracle_mod.eval_words(u.with_thresholds(q), it, 0, w_main)[: u.n_be])
    nom = oracle_mod.eval_words(u, it, w_main, w_cut)[: u.n_be].copy()
    S, tab = _cut_tables(u)
    seed = _mix64(((it << 32) ^ 0x5bd1e995) & M64)
    for k, root in enumerate(roots):
        b0 = _mix64(seed ^ (k << 32))
        for w in range(w_cut):
            b1 = _mix64(b0 ^ (w_main + w))
            for b in range(64):
                for e in _descend(u, S, tab, int(root), _mix64(b1 ^ b)):
                    nom[e, w] |= np.uint64(1) << np.uint64(b)
    parts.append(nom)
    be = np.concatenate(parts, axis=1)
    bits = _gate_words(u, be)
    ql = q.astype(np.float64) / TWO32
    l1 = np.log1p(-p) - np.log1p(-ql)
    a = np.log(p) - np.log(ql) - l1
    ce = np.zeros(u.n_be)
    for k, root in enumerate(roots):
        sl = slice(int(bb[k]), int(bb[k + 1]))
        top = bits[int(root)]
        lw_main = l1[sl].sum() + np.einsum("i,iwb->wb", a[sl], bits[sl].astype(np.float64))
        sw = sw2 = 0.0
        hits = 0
        wgt = np.zeros((W, 64))
        logS = np.log(S[int(root)])
        for w in range(W):
            for b in range(64):
                if not top[w, b]:
                    continue
                n_cut = _count(u, bits[:, w, b], int(root))
                lw_cut = logS - np.log(n_cut)
                if w_main:
                    lw = -np.logaddexp(np.log(w_main / W) - lw_main[w, b], np.log(w_cut / W) - lw_cut)
                else:
                    lw = lw_cut
                wgt[w, b] = np.exp(lw)
                hits += 1
        assert r["hits"][k] == hits
        assert r["sum_w"][k] == pytest.approx(wgt.sum(), rel=1e-10)
        assert r["sum_w2"][k] == pytest.approx((wgt ** 2).sum(), rel=1e-10)
        ce[sl] = np.einsum("wb,iwb->i", wgt, bits[sl].astype(np.float64))
    np.testing.assert_allclose(r["ce_num"], ce, rtol=1e-10, atol=1e-300)


@pytest.mark.gpu
def test_cut_set_estimates_rare_trees(gpu):
    """The cut-set component alone: every tree's estimate within 4 sigma of
    its exact probability, with far fewer samples than a product proposal."""
    from mcscram_b200.importance import BatchedImportanceSampler
    trees = _small_config5(8)
    exact = np.array([g.meta["exact_p_top"] for g in trees])
    W = 1 << 12
    with BatchedImportanceSampler(trees) as s:
        r = s.run(s.union.be_threshold, iteration=11, word_count=W, words_cutset=W)
    n = W * 64
    est = r["sum_w"] / n
    se = np.sqrt(np.maximum(r["sum_w2"] / n - est ** 2, 0) / (n - 1))
    # When almost every sample holds a single cut set (N(x) = 1) the weights are all S(top) and the
    # variance estimate is ~0; the estimator stays unbiased, but its error then comes from the rare
    # samples with N > 1, which carry the difference S - P (of order P^2 for rare events) and which
    # the sample variance does not see until they occur: a floor of 10 P^2 (+ 1e-6 P) covers them.
    assert np.all(np.abs(est - exact) <= 4 * se + 1e-6 * exact + 10 * exact ** 2), (est / exact, se / exact)
    assert np.all(1.96 * se / est < 0.05)  # 5 % reached with 2.6e5 samples per tree


@pytest.mark.gpu
def test_cut_set_component_rejects_shared_gates(gpu):
    from mcscram_b200 import _capi
    from mcscram_b200.importance import BatchedImportanceSampler, cut_set_eligible
    g = synth.generate(synth.TreeSpec(n_be=40, n_gates=20, mix={AND: 0.5, OR: 0.5}, p_range=(0.01, 0.2), seed=3,
                                      n_layers=5, share_node_frac=0.3))
    assert np.any(np.bincount(g.inputs, minlength=g.n_nodes)[g.n_be:] > 1) and not cut_set_eligible(g)
    with BatchedImportanceSampler([g]) as s:
        with pytest.raises(_capi.McgError, match="read by several gates"):
            s.run(s.union.be_threshold, iteration=1, word_count=64, words_cutset=64)


# ------------------------------------------- cut-set component with shared basic events

Z_OCC = 32  # occurrences a sample keeps for pruning (the kernel's kZOcc)


def _occurrences(u, roots, shared):
    nb = u.n_be
    occ_range, occ_of, pos = {}, {}, 0
    for root in roots:
        stack = [(int(root), 0)]
        occ_range[int(root) - nb] = [pos, pos]
        while stack:
            node, i = stack[-1]
            j = node - nb
            ins = [int(x) for x in u.gate_inputs(j)]
            if i < len(ins):
                stack[-1] = (node, i + 1)
                x = ins[i]
                if x < nb:
                    if shared[x]:
                        occ_of.setdefault(x, []).append(pos)
                        pos += 1
                else:
                    occ_range[x - nb] = [pos, pos]
                    stack.append((x, 0))
            else:
                occ_range[j][1] = pos
                stack.pop()
    return occ_range, occ_of


def _eval(u, node, leaf, enter, other):
    """The kernels' AND / OR / ATLEAST recursion (same order of operations)."""
    nb = u.n_be
    j = node - nb
    op, k = int(u.gate_op[j]), int(u.gate_k[j]) & 0xFF
    acc = 1.0 if op == AND else 0.0
    dp = [1.0] + [0.0] * 8
    for x in (int(c) for c in u.gate_inputs(j)):
        val = leaf(x) if x < nb else (_eval(u, x, leaf, enter, other) if enter(x) else other(x))
        if op == AND:
            acc *= val
        elif op == ATLEAST:
            for r in range(k, 0, -1):
                dp[r] += dp[r - 1] * val
        else:
            acc += val
    return dp[k] if op == ATLEAST else acc


def _descend_shared(u, S0, tab, shared, occ_range, zlist, zthr, root, base):
    """Shared events drawn and private events forced for one sample (the
    library's draws, pruning and arithmetic)."""
    nb = u.n_be
    zbase = _mix64(base ^ 0x2545F4914F6CDD1D)
    z = {}
    occ, prune = [], True
    for jj, (e, occs) in enumerate(zlist):
        z[e] = (_mix64((zbase + (jj + 1) * 0x9E3779B97F4A7C15) & M64) >> 32) < int(zthr[e])
        if not z[e]:
            continue
        for o in occs:
            if not prune:
                break
            if len(occ) == Z_OCC:
                prune = False
                break
            occ.append(o)
            occ.sort()

    def affected(x):
        lo, hi = occ_range.get(x - nb, (0, 0))
        if lo >= hi:
            return False
        if not prune:
            return True
        return any(lo <= o < hi for o in occ)

    leaf = lambda x: (1.0 if z[x] else 0.0) if shared[x] else S0[x]
    other = lambda x: S0[x]

    def sz(x):
        if x < nb:
            return leaf(x)
        return _eval(u, x, leaf, affected, other) if affected(x) else S0[x]

    draw = 0

    def unif():
        nonlocal draw
        draw += 1
        return (_mix64((base + draw * 0x9E3779B97F4A7C15) & M64) >> 11) * 2.0 ** -53

    forced = []
    if not sz(int(root)) > 0:
        return z, forced
    stack = [int(root)]
    while stack:
        node = stack.pop()
        if node < nb:
            if not shared[node]:
                forced.append(node)
            continue
        j = node - nb
        op, n, k = int(u.gate_op[j]), int(u.gate_in_count[j]), int(u.gate_k[j]) & 0xFF
        ins = [int(x) for x in u.gate_inputs(j)]
        cond = affected(node)
        if op == OR:
            x = unif()
            c = 0
            if not cond:
                while c + 1 < n and x >= tab[j][c]:
                    c += 1
            else:
                tot = 0.0
                for i in ins:
                    tot += sz(i)
                cum = 0.0
                while c + 1 < n:
                    cum += sz(ins[c])
                    if x * tot < cum:
                        break
                    c += 1
            stack.append(ins[c])
        elif op == ATLEAST:
            if cond:
                v = [sz(i) for i in ins]
                E = [[0.0] * (k + 1) for _ in range(n + 1)]
                E[n][0] = 1.0
                for c in range(n - 1, -1, -1):
                    for r in range(k + 1):
                        e = E[c + 1][r]
                        if r > 0:
                            e += v[c] * E[c + 1][r - 1]
                        E[c][r] = e
            else:
                v, E = [S0[i] for i in ins], tab[j]
            r = k
            for c in range(n):
                if r == 0:
                    break
                take = n - c == r
                if not take:
                    take = unif() * E[c][r] < v[c] * E[c + 1][r - 1]
                if take:
                    stack.append(ins[c])
                    r -= 1
        else:
            stack.extend(ins)
    return z, forced


def _dag_cut_trees(n=3, n_be=36, n_gates=16, share=0.3, seeds=range(60), n_layers=4):
    out = []
    for seed in seeds:
        try:
            g = synth.generate(synth.TreeSpec(n_be=n_be, n_gates=n_gates, mix={AND: 0.4, OR: 0.3, ATLEAST: 0.3},
                                              p_range=(0.01, 0.2), seed=seed, atleast_n=(3, 4), n_layers=n_layers,
                                              share_be_frac=share))
        except ValueError:
            continue
        fan = np.bincount(g.inputs, minlength=g.n_nodes)
        if np.all(fan[g.n_be:] <= 1) and np.any(fan[: g.n_be] > 1):
            out.append(g)
        if len(out) == n:
            return out
    raise AssertionError("no trees with shared events generated")


def _tree_with_shared_gates():
    g = synth.generate(synth.TreeSpec(n_be=30, n_gates=14, mix={AND: 0.5, OR: 0.5}, p_range=(0.01, 0.2), seed=3,
                                      n_layers=4, share_node_frac=0.3))
    assert np.any(np.bincount(g.inputs, minlength=g.n_nodes)[g.n_be:] > 1)
    return g


@pytest.mark.gpu
@pytest.mark.parametrize("w_main,w_cut,zscale,n_be,mixed", [(0, 256, 12.0, 36, False), (300, 300, 12.0, 36, False),
                                                            (0, 48, 1e6, 110, False), (200, 200, 12.0, 36, True)])
def test_cut_set_component_with_shared_events_matches_cpu(oracle_mod, gpu, w_main, w_cut, zscale, n_be, mixed):
    """Trees whose shared nodes are basic events: the words after forcing,
    the hits, sum w, sum w^2 and CE numerators equal a CPU restatement of
    the component (shared events drawn from their own proposal, the cut set
    on the conditioned tree).  zscale 1e6 puts many shared events at 0.5, so
    that samples exceed the pruning list and take the unpruned path.  mixed
    adds a tree with a gate read by two gates, which the component cannot
    draw: its samples there stay nominal (density p)."""
    from mcscram_b200.importance import BatchedImportanceSampler
    trees = _dag_cut_trees() if n_be < 100 else _dag_cut_trees(n=2, n_be=n_be, n_gates=n_be // 2, share=0.4, n_layers=5)
    if mixed:
        trees = trees[:2] + [_tree_with_shared_gates()] + trees[2:]
    it = 5
    with BatchedImportanceSampler(trees, chunk_words=256) as s:
        u, bb, roots = s.union, s.be_begin, s.roots
        p = u.quantised_probabilities()
        drawn = np.array([not (mixed and k == 2) for k in range(len(trees))])
        shared = (np.bincount(u.inputs, minlength=u.n_nodes)[: u.n_be] > 1) & np.repeat(drawn, np.diff(bb))
        q = probability_threshold(np.minimum(p * 6.0, 0.5))
        qz = probability_threshold(np.where(shared, np.minimum(p * zscale, 0.5), p))
        W = w_main + w_cut
        r = s.run(q, iteration=it, word_count=W, ce=True, words_cutset=w_cut, q_cutset=qz)
    parts = []
    if w_main:
        parts.append(oracle_mod.eval_words(u.with_thresholds(q), it, 0, w_main)[: u.n_be])
    nom = oracle_mod.eval_words(u, it, w_main, w_cut)[: u.n_be].copy()
    nom[shared] = 0  # the forcing kernel draws the shared events itself
    v0 = u.with_thresholds(np.where(shared, 0, u.be_threshold).astype(np.uint64))
    S0, tab = _cut_tables(v0)
    occ_range, occ_of = _occurrences(u, roots[drawn], shared)
    seed = _mix64(((it << 32) ^ 0x5bd1e995) & M64)
    for k, root in enumerate(roots):
        if not drawn[k]:
            continue
        zlist = [(e, occ_of.get(e, [])) for e in range(int(bb[k]), int(bb[k + 1])) if shared[e]]
        b0 = _mix64(seed ^ (k << 32))
        for w in range(w_cut):
            b1 = _mix64(b0 ^ (w_main + w))
            for b in range(64):
                z, forced = _descend_shared(u, S0, tab, shared, occ_range, zlist, qz, int(root), _mix64(b1 ^ b))
                for e in forced + [e for e, on in z.items() if on]:
                    nom[e, w] |= np.uint64(1) << np.uint64(b)
    parts.append(nom)
    be = np.concatenate(parts, axis=1)
    bits = _gate_words(u, be)
    ql = q.astype(np.float64) / TWO32
    l1 = np.log1p(-p) - np.log1p(-ql)
    a = np.log(p) - np.log(ql) - l1
    rz = qz.astype(np.float64) / TWO32
    lz1 = np.where(shared, np.log1p(-p) - np.log1p(-rz), 0.0)
    az = np.where(shared, np.log(p) - np.log(rz) - lz1, 0.0)
    ce = np.zeros(u.n_be)
    n_long = 0
    for k, root in enumerate(roots):
        sl = slice(int(bb[k]), int(bb[k + 1]))
        top = bits[int(root)]
        lw_main = l1[sl].sum() + np.einsum("i,iwb->wb", a[sl], bits[sl].astype(np.float64))
        lw_z = lz1[sl].sum() + np.einsum("i,iwb->wb", az[sl], bits[sl].astype(np.float64))
        wgt = np.zeros((W, 64))
        hits = 0
        for w in range(W):
            for b in range(64):
                if not top[w, b]:
                    continue
                x = bits[:, w, b]
                if drawn[k]:
                    leaf = lambda e: (1.0 if x[e] else 0.0) if shared[e] else S0[e]
                    s_z = _eval(u, int(root), leaf, lambda g: True, lambda g: S0[g])
                    n_cut = _count(u, x, int(root))
                    lw_cut = lw_z[w, b] + np.log(s_z) - np.log(n_cut)
                else:
                    lw_cut = 0.0  # nominal samples: density p
                if w_main:
                    lw = -np.logaddexp(np.log(w_main / W) - lw_main[w, b], np.log(w_cut / W) - lw_cut)
                else:
                    lw = lw_cut
                wgt[w, b] = np.exp(lw)
                hits += 1
                n_long += int(sum(len(occ_of.get(e, [])) for e in range(sl.start, sl.stop) if x[e] and shared[e])
                              > Z_OCC)
        assert r["hits"][k] == hits
        assert r["sum_w"][k] == pytest.approx(wgt.sum(), rel=1e-10)
        assert r["sum_w2"][k] == pytest.approx((wgt ** 2).sum(), rel=1e-10)
        ce[sl] = np.einsum("wb,iwb->i", wgt, bits[sl].astype(np.float64))
    np.testing.assert_allclose(r["ce_num"], ce, rtol=1e-10, atol=1e-300)
    if zscale > 1e3:
        assert n_long > 0  # the unpruned path ran


# ----------------------------------------- rare-event trees with shared basic events

def _small_dag_rare(n, max_events=600):
    """Instances of the rare-event set with shared events (20 % of the
    basic events read by two gates) with at most max_events events, and
    their exact top-event probabilities by BDD."""
    from oracle import oracle
    out, exact, i = [], [], 0
    while len(out) < n:
        g = synth.config5_dag_instance(i)
        i += 1
        if g.n_be > max_events:
            continue
        out.append(g)
        exact.append(oracle.bdd_probability(g))
    return out, np.array(exact)


@pytest.mark.gpu
def test_learned_is_on_rare_dags_with_shared_events(gpu):
    """The batched pipeline (cut-set component drawing the shared events
    first) on rare-event DAGs of at most 600 events whose shared events
    matter: every estimate within 3 sigma of the exact BDD value, with its
    reported 95 % relative error at most 5 %."""
    from mcscram_b200.importance import batched_learned_is, shared_events
    trees, exact = _small_dag_rare(8)
    assert all(shared_events(g).sum() >= 0.15 * g.n_be for g in trees)
    res = batched_learned_is(trees, target_rel_err=0.05, max_est_words=1 << 22)
    assert res.converged.all() and not res.fallback.any(), [r for r in res.rounds if r["phase"] != "probe"]
    se = res.estimate * res.rel_err95 / 1.96
    assert np.all(np.abs(res.estimate - exact) <= 3 * se + 1e-6 * exact + 10 * exact ** 2), \
        (res.estimate / exact, res.rel_err95)
    assert np.all(res.rel_err95 <= 0.05)


@pytest.mark.gpu
def test_learned_is_on_the_2000_event_dag_at_1e8(gpu):
    """The 2,000-event / 1,200-gate rare-event tree with 400 shared events
    (P_top ~ 1e-8): within 3 sigma of the exact value at 5 %."""
    from oracle import oracle
    from mcscram_b200.importance import batched_learned_is
    g = synth.config4_dag()
    exact = oracle.bdd_probability(g)
    res = batched_learned_is([g], target_rel_err=0.05)
    se = res.estimate[0] * res.rel_err95[0] / 1.96
    assert res.converged[0] and res.rel_err95[0] <= 0.05
    assert abs(res.estimate[0] - exact) <= 3 * se + 10 * exact ** 2, (res.estimate[0] / exact, res.rel_err95[0])


@pytest.mark.gpu
def test_network_against_the_pipeline_without_it(gpu):
    """What the trained network adds over the same pipeline without it (the
    smoothed cross-entropy targets as the proposal) on rare DAGs with shared
    events: both estimates unbiased against the BDD; the relative error of
    each at the same number of samples is recorded (the network's proposal
    is not required to win: on these trees the cut-set component carries most
    of the accuracy)."""
    from mcscram_b200.importance import batched_learned_is
    trees, exact = _small_dag_rare(6)
    out = {}
    for net in (True, False):
        res = batched_learned_is(trees, target_rel_err=0.0, est_words=1 << 13, max_est_words=1 << 13,
                                 use_network=net)
        se = res.estimate * res.rel_err95 / 1.96
        assert np.all(np.abs(res.estimate - exact) <= 4 * se + 10 * exact ** 2), (net, res.estimate / exact)
        out[net] = np.median(res.rel_err95)
    print(f"median 95% relative error at 2^19 samples per tree: network {out[True]:.4g}, without {out[False]:.4g}")


@pytest.mark.gpu
def test_mixed_batch_chooses_the_defensive_proposal_per_tree(gpu):
    """A batch of rare DAGs the cut-set component draws and rare trees with
    gates read by two gates (which it cannot draw): "auto" gives the first
    the cut-set component and the others mode proposals in the same passes,
    and every estimate lies within 4 sigma of the exact BDD value."""
    from oracle import oracle
    from mcscram_b200.importance import batched_learned_is, cut_set_eligible
    trees, exact = _small_dag_rare(3)
    for seed in (7, 8):
        g = synth.generate(synth.TreeSpec(n_be=120, n_gates=60, mix={AND: 0.5, OR: 0.4, ATLEAST: 0.1},
                                          p_range=(1e-4, 1e-2), seed=seed, n_layers=6, atleast_n=(3, 4),
                                          share_node_frac=0.15))
        g = synth.calibrate_rare_approx(g, 1e-6)
        assert not cut_set_eligible(g)
        trees.append(g)
        exact = np.append(exact, oracle.bdd_probability(g))
    res = batched_learned_is(trees, target_rel_err=0.05, max_est_words=1 << 22)
    se = res.estimate * res.rel_err95 / 1.96
    assert np.all(np.abs(res.estimate - exact) <= 4 * se + 10 * exact ** 2), (res.estimate / exact, res.rel_err95)
    assert res.converged.sum() >= len(trees) - 1
