"""Learned importance sampling for rare top events (include/mcg_is.h).

* ``event_features`` -- 16 structural features per basic event (log p,
  fan-out, depths, parent gate-type mix, ATLEAST tightness, path
  connectives, ...), the network's input.
* ``ImportanceSampler`` -- the bit-packed sampler with proposal thresholds
  and FP64 likelihood-ratio estimator (mcg_is_run).
* ``ProposalMLP`` -- 16 -> 64 -> 64 -> 1 network trained on the GPU
  (mcg_mlp_*), BF16 weights with FP32 accumulation.
* ``cross_entropy`` -- the cross-entropy method: sample with the current
  proposal, take the likelihood-weighted failure frequency of every event as
  the next target, fit the network to it, repeat.
* ``estimate`` -- the final IS estimate with an effective-sample-size check
  that falls back to the plain sampler when the weights collapse.
* ``BatchedImportanceSampler`` / ``batched_learned_is`` -- the same for many
  trees at once: the trees are joined into one graph and sampled in one
  staged pass per call, one network (with a per-tree input) gives every
  tree's proposal, and trees leave the batch as they reach the target
  error (or fall back to plain sampling).
"""
from __future__ import annotations

import ctypes as C
import time
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

from . import _capi
from .graph import AND, ATLEAST, OR, XOR, FlatGraph, concat, probability_threshold

N_FEATURES = 16
N_PARAMS = 16 * 64 + 64 + 64 * 64 + 64 + 64 + 1
TWO_32 = float(1 << 32)

_vp = C.c_void_p
_u64p = C.POINTER(C.c_uint64)
_fp = C.POINTER(C.c_float)
_dp = C.POINTER(C.c_double)


class IsResult(C.Structure):
    _fields_ = [("samples", C.c_uint64), ("hits", C.c_uint64), ("sum_w", C.c_double), ("sum_w2", C.c_double),
                ("estimate", C.c_double), ("std_err", C.c_double), ("rel_err", C.c_double), ("ess", C.c_double),
                ("max_log_w", C.c_double), ("kernel_ms", C.c_double)]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


_capi.register_signatures({
    "mcg_is_create": (C.c_int, [C.POINTER(_capi.GraphDesc), C.POINTER(_capi.RunDesc), C.POINTER(_vp)]),
    "mcg_is_destroy": (C.c_int, [_vp]),
    "mcg_is_run": (C.c_int, [_vp, _u64p, C.c_uint32, C.c_uint64, C.c_uint64, C.POINTER(IsResult), _dp]),
    "mcg_is_batch_create": (C.c_int, [C.POINTER(_capi.GraphDesc), C.c_uint32, C.POINTER(C.c_uint32),
                                      C.POINTER(_capi.RunDesc), C.POINTER(_vp)]),
    "mcg_is_batch_destroy": (C.c_int, [_vp]),
    "mcg_is_batch_run": (C.c_int, [_vp, _u64p, C.c_uint32, _u64p, _u64p, C.c_uint64, _u64p, C.c_uint32,
                                   C.c_uint64, C.c_uint64, _dp, _dp, _dp]),
    "mcg_mlp_create": (C.c_int, [C.c_int32, C.c_uint64, C.POINTER(_vp)]),
    "mcg_mlp_train_time": (C.c_int, [_vp, C.POINTER(C.c_double)]),
    "mcg_shared_posteriors": (C.c_int, [C.POINTER(_capi.GraphDesc), C.c_uint32, C.c_uint64, C.POINTER(C.c_double),
                                        C.POINTER(C.c_double)]),
    "mcg_mlp_destroy": (C.c_int, [_vp]),
    "mcg_mlp_set_params": (C.c_int, [_vp, _fp]),
    "mcg_mlp_get_params": (C.c_int, [_vp, _fp]),
    "mcg_mlp_forward": (C.c_int, [_vp, _fp, C.c_uint32, _fp]),
    "mcg_mlp_grad": (C.c_int, [_vp, _fp, _fp, _fp, C.c_uint32, _fp, _fp]),
    "mcg_mlp_train": (C.c_int, [_vp, _fp, _fp, _fp, C.c_uint32, C.c_uint32, C.c_float, _fp]),
})


def _p(a, t):
    return a.ctypes.data_as(C.POINTER(t))


def approximate_importance(g: FlatGraph, root=None):
    """Node probabilities and per-event conditional marginals under the
    independence approximation (every gate's inputs taken as independent):
    one bottom-up pass gives P~ of every node, one reverse-mode pass the
    sensitivity d log P~_top / d p_i, and
        P~(x_i = 1 | top) = p_i + p_i (1 - p_i) d log P~_top / d p_i,
    the approximate conditional marginal that the zero-variance product
    proposal needs (approximate zero-variance importance sampling).  Exact
    for trees where no node has two parents; an approximation, and still
    cheap, for DAGs.  With `root` (a node id) the marginals are conditioned on
    that node instead of the top event (events outside its cone keep p);
    with a list of node ids, on each of them (cond then [len(root), n_be]).
    Returns (node_prob [n_nodes], cond [n_be])."""
    from .graph import NAND, NOR, NOT, NULL
    nb, ng = g.n_be, g.n_gates
    pr = np.zeros(g.n_nodes)
    pr[:nb] = g.quantised_probabilities()
    if ng == 0 or nb == 0:
        roots = [g.root if root is None else int(root)] if np.ndim(root) == 0 else [int(r) for r in root]
        cond = _conditioned(pr, [], nb, g.n_nodes, roots)
        return pr, (cond[0] if np.ndim(root) == 0 else cond)
    depth = g.layers()[nb:]
    cnt = g.gate_in_count.astype(np.int64)
    pos_neg = cnt - g.gate_neg_count.astype(np.int64)
    ops = g.gate_op.astype(np.int64)
    kk = g.gate_k.astype(np.int64) & 0xFF
    ib = g.gate_in_begin.astype(np.int64)
    levels = [np.nonzero(depth == d)[0] for d in range(1, int(depth.max()) + 1)]
    cache = []
    for gs in levels:  # bottom-up
        c = cnt[gs]
        m = int(c.max())
        col = np.arange(m)
        valid = col[None, :] < c[:, None]
        src = g.inputs[np.where(valid, ib[gs][:, None] + col[None, :], 0)].astype(np.int64)
        neg = col[None, :] >= pos_neg[gs][:, None]
        v = np.where(valid, np.where(neg, 1.0 - pr[src], pr[src]), 0.0)
        op = ops[gs]
        r = np.zeros(gs.size)
        d = np.zeros((gs.size, m))  # d gate / d (input value), before the output complement
        s_and = (op == AND) | (op == NAND)
        if s_and.any():
            vv = np.where(valid[s_and], v[s_and], 1.0)
            r[s_and] = np.prod(vv, axis=1)
            for j in range(m):  # leave-one-out products
                d[s_and, j] = np.prod(np.where(col[None, :] == j, 1.0, vv), axis=1)
        s_or = (op == OR) | (op == NOR)
        if s_or.any():
            cv = np.where(valid[s_or], 1.0 - v[s_or], 1.0)
            with np.errstate(divide="ignore"):
                r[s_or] = -np.expm1(np.sum(np.log1p(-np.where(valid[s_or], v[s_or], 0.0)), axis=1))
            for j in range(m):
                d[s_or, j] = np.prod(np.where(col[None, :] == j, 1.0, cv), axis=1)
        s_x = op == XOR
        if s_x.any():
            vx = v[s_x]
            acc = np.zeros(vx.shape[0])
            for j in range(m):
                acc = acc * (1 - vx[:, j]) + (1 - acc) * vx[:, j]
            r[s_x] = acc
            for j in range(m):  # XOR of the others, then d/dv_j = 1 - 2 x_others
                o = np.zeros(vx.shape[0])
                for l in range(m):
                    if l != j:
                        o = o * (1 - vx[:, l]) + (1 - o) * vx[:, l]
                d[s_x, j] = 1.0 - 2.0 * o
        s_k = op == ATLEAST
        if s_k.any():
            vk = v[s_k]
            k = kk[gs][s_k]
            ck = c[s_k]
            nk = vk.shape[0]

            def count_dists(vals):
                # F[j][:, t] = P(t of columns 0 .. j-1 fire), j = 0 .. m (padded columns have p = 0)
                f = np.zeros((m + 1, nk, m + 1))
                f[0][:, 0] = 1.0
                for j in range(m):
                    x = vals[:, j][:, None]
                    f[j + 1] = f[j] * (1.0 - x)
                    f[j + 1][:, 1:] += f[j][:, :-1] * x
                return f

            fwd = count_dists(vk)
            bwd = count_dists(vk[:, ::-1])  # bwd[i]: the last i columns
            tail = np.cumsum(fwd[m][:, ::-1], axis=1)[:, ::-1]  # P(count >= t)
            r[s_k] = np.where(k <= ck, tail[np.arange(nk), np.clip(k, 0, m)], 0.0)
            # d P(count >= k) / d v_j = P(count of the others == k - 1): the
            # columns before j (fwd[j]) and after it (bwd[m - 1 - j]) combined
            a = np.arange(m + 1)
            idx = (k - 1)[None, :, None] - a[None, None, :]
            ok = (idx >= 0) & (idx <= m)
            after = bwd[m - 1 - np.arange(m)]
            picked = np.take_along_axis(after, np.broadcast_to(np.clip(idx, 0, m), after.shape), axis=2)
            others_eq = np.sum(fwd[:m] * np.where(ok, picked, 0.0), axis=2)  # [m, nk]
            d[s_k] = np.where((k <= ck)[:, None], others_eq.T, 0.0)
        s_l = (op == NOT) | (op == NULL)
        if s_l.any():
            last = np.maximum(c[s_l] - 1, 0)
            r[s_l] = v[s_l][np.arange(last.size), last]
            d[s_l] = np.where(col[None, :] == last[:, None], 1.0, 0.0)
        comp = (op == NAND) | (op == NOR) | (op == NOT)
        r[comp] = 1.0 - r[comp]
        d = np.where(comp[:, None], -d, d)
        d = np.where(neg, -d, d)
        d = np.where(valid, d, 0.0)
        pr[nb + gs] = r
        cache.append((gs, src, valid, d))
    roots = [g.root if root is None else int(root)] if np.ndim(root) == 0 else [int(r) for r in root]
    cond = _conditioned(pr, cache, nb, g.n_nodes, roots)
    return pr, (cond[0] if np.ndim(root) == 0 else cond)


def _conditioned(pr, cache, nb, n_nodes, roots):
    """Reverse mode for several conditioning nodes at once:
    adj[:, r] = d log P~_root_r / d P~_node, then the conditional marginals
    [len(roots), n_be]."""
    R = len(roots)
    adj = np.zeros((n_nodes, R))
    live = np.zeros(R, dtype=bool)
    for j, r0 in enumerate(roots):
        if pr[r0] > 1e-300:
            adj[r0, j] = 1.0 / pr[r0]
            live[j] = True
    for gs, src, valid, d in reversed(cache):
        contrib = adj[nb + gs][:, None, :] * d[:, :, None]
        np.add.at(adj, src[valid], contrib[valid])
    p = pr[:nb]
    cond = np.clip(p[None, :] + (p * (1.0 - p))[None, :] * adj[:nb].T, 0.0, 1.0)
    for j, r0 in enumerate(roots):
        if not live[j]:  # nothing to condition on
            cond[j] = p
        elif r0 < nb:  # conditioned on a basic event: it fires, the rest keep p
            cond[j] = p
            cond[j, r0] = 1.0
    return cond


def cut_set_eligible(g: FlatGraph) -> bool:
    """Whether the cut-set component (mcg_is_batch_run's words_cutset) takes
    this graph: AND/OR/ATLEAST (k <= 8)/pass-through gates, no complemented
    inputs, no gate read by two gates (basic events may be: they are drawn
    first, and the cut set on the tree conditioned on them)."""
    from .graph import NULL
    ok_ops = np.isin(g.gate_op, [AND, OR, ATLEAST, NULL])
    k_ok = np.where(g.gate_op == ATLEAST, (g.gate_k & 0xFF) <= 8, True)
    fan = np.bincount(g.inputs, minlength=g.n_nodes)
    return bool(np.all(ok_ops) and np.all(k_ok) and np.all(g.gate_neg_count == 0) and np.all(fan[g.n_be:] <= 1))


def shared_posteriors(g: FlatGraph, max_terms: int = 4096):
    """(S, posterior): the tree's cut-set sum with every shared event counted
    once per product, and P(x_e = 1 | top) ~ p_e S(top | x_e = 1) / S for the
    events read by several gates (-1 for the others), from
    mcg_shared_posteriors; None when a gate holds more than max_terms
    monomials (too many shared events open below it) or the graph does not
    qualify."""
    lib = _capi.load()
    view = _capi.GraphView(g)
    post = np.zeros(max(g.n_be, 1), dtype=np.float64)
    s = C.c_double()
    rc = lib.mcg_shared_posteriors(C.byref(view.desc), int(g.root), max_terms, C.byref(s), _p(post, C.c_double))
    if rc != _capi.MCG_OK:
        return None
    return float(s.value), post[: g.n_be]


def shared_seed(g: FlatGraph) -> np.ndarray:
    """A generous estimate of P(x_i = 1 | top) for the basic events read by
    several gates (others: their p): the largest of cut_inclusion (a shared
    event's m leaves at p^(1/m)), the same inclusion with the leaves at p,
    and the independence approximation's conditional marginal.  The first
    weighs right a cut set that uses all of a shared event's leaves and
    over-weighs one that uses fewer, the second the other way round."""
    from .graph import probability_threshold
    p = g.quantised_probabilities()
    fan = np.maximum(np.bincount(g.inputs, minlength=g.n_nodes)[: g.n_be], 1)
    plain = g.with_thresholds(probability_threshold(np.clip(p ** fan, 0.0, 1.0)))
    est = np.maximum(np.maximum(cut_inclusion(g), cut_inclusion(plain)), approximate_importance(g)[1])
    return np.where(fan > 1, est, p)


def cut_inclusion(g: FlatGraph) -> np.ndarray:
    """Expected number of times each basic event is picked by the cut-set
    descent on the graph read as a tree, every leaf of an event read by m
    gates at p^(1/m): S(node) bottom-up (leaf value; AND product, OR sum,
    ATLEAST k-th elementary symmetric sum), then the descent's visit
    probability top-down (OR: child share S(child)/S(OR); AND: every child;
    ATLEAST k: P(child in the k-subset) = S_c e_{k-1}(others) / e_k(all)).
    A cut set that uses all m leaves of a shared event then weighs p once, as
    it does in the graph, where read as a tree it would weigh p^m; one that
    uses fewer leaves weighs more than it should.  For events read by several
    gates the result is a generous estimate of how much of the union of cut
    sets goes through them: the seed of their proposal in the cut-set
    component."""
    nb, ng = g.n_be, g.n_gates
    S = np.zeros(g.n_nodes)
    p0 = g.quantised_probabilities()
    fan = np.maximum(np.bincount(g.inputs, minlength=g.n_nodes)[:nb], 1)
    S[:nb] = np.where(fan > 1, p0 ** (1.0 / fan), p0)
    ops = g.gate_op
    kk = g.gate_k & 0xFF

    def esym(v, k):
        e = np.zeros(k + 1)
        e[0] = 1.0
        for x in v:
            e[1:] = e[1:] + e[:-1] * x
        return e

    for j in range(ng):
        v = S[g.gate_inputs(j)]
        op = int(ops[j])
        if op == AND:
            S[nb + j] = float(np.prod(v))
        elif op == ATLEAST:
            S[nb + j] = esym(v, int(kk[j]))[int(kk[j])]
        elif op == OR:
            S[nb + j] = float(np.sum(v))
        else:
            S[nb + j] = float(v[-1]) if v.size else 0.0
    visit = np.zeros(g.n_nodes)
    visit[g.root] = 1.0
    for j in range(ng - 1, -1, -1):
        vg = visit[nb + j]
        if vg == 0.0:
            continue
        ins = g.gate_inputs(j).astype(np.int64)
        v = S[ins]
        op = int(ops[j])
        if op == OR:
            tot = v.sum()
            if tot > 0:
                np.add.at(visit, ins, vg * v / tot)
        elif op == ATLEAST:
            k = int(kk[j])
            ek = esym(v, k)[k]
            if ek > 0:
                share = np.array([v[c] * esym(np.delete(v, c), k - 1)[k - 1] / ek for c in range(v.size)])
                np.add.at(visit, ins, vg * share)
        else:
            np.add.at(visit, ins, vg)
    return visit[:nb]


def shared_events(g: FlatGraph) -> np.ndarray:
    """Basic events read by more than one gate."""
    return np.bincount(g.inputs, minlength=g.n_nodes)[: g.n_be] > 1


def _mode_kids(g: FlatGraph) -> List[int]:
    """Children of the top gate when it is an OR without complemented inputs
    (the modes of mode_proposals), else none."""
    from .graph import OR
    top = g.root - g.n_be
    if 0 <= top < g.n_gates and int(g.gate_op[top]) == OR and int(g.gate_neg_count[top]) == 0:
        return [int(c) for c in g.gate_inputs(top)]
    return []


def mode_proposals(g: FlatGraph, n_comp: int, cap: float, approx=None) -> np.ndarray:
    """Defensive proposals for the union-of-modes form of the top event
    ([n_comp, n_be]).  When the top gate is an OR, component j is the
    approximate zero-variance proposal conditioned on its child j failing
    (approximate_importance with that child as root; events outside the
    child keep p): sampling every child's failure region at a fixed share is
    the mixture form of importance sampling for a union of rare events.
    With more children than components the last component is the
    unconditioned proposal, and with fewer children (or a top gate that is
    not an OR) components repeat.  Clipped to [1e-7, cap].  `approx` may pass
    approximate_importance(g, root=[g.root] + _mode_kids(g)) computed already."""
    nb = g.n_be
    kids = _mode_kids(g)
    pr, cond = approx if approx is not None else approximate_importance(g, root=[g.root] + kids)
    cond = np.clip(cond, 1e-7, cap)
    whole = cond[0]
    if not kids:
        return np.repeat(whole[None, :], n_comp, axis=0)
    order = sorted(range(len(kids)), key=lambda j: -pr[kids[j]])  # heaviest modes first
    comps = [cond[1 + j] for j in order[:n_comp]]
    if len(kids) > n_comp:
        comps[-1] = whole
    out = np.empty((n_comp, nb))
    for j in range(n_comp):
        out[j] = comps[j % len(comps)]
    return out


def event_features(g: FlatGraph, instance_scale: Optional[float] = None, importance: bool = False,
                   approx=None) -> np.ndarray:
    """16 features per basic event, float32 [n_be, 16]:

    0 log10 p (shifted), 1 fan-out, 2-3 min/max depth of the parents, 4-6
    fraction of AND/OR/ATLEAST parents, 7 mean parent fan-in, 8 mean k/n of
    ATLEAST parents, 9 siblings under the first parent, 10 mean log10 p of
    the sibling events, 11 fraction of sibling gates, 12 parent at the top
    depth, 13-14 AND/OR share of the first-parent path to the top, 15 a
    per-instance input: 1 for a single tree, log10 of the instance's
    probe inflation / 6 when one network serves many trees.  "First parent"
    is the parent gate of lowest index.  Computed for all events at once.
    importance=True replaces 11 and 12 with the independence-approximation
    inputs of approximate_importance: log10 of the first parent's
    probability / 10 + 1 and log10 P~(x_i = 1 | top) / 4 + 1; `approx` may pass
    (node probabilities, conditional marginals given the top) computed already."""
    nb, ng = g.n_be, g.n_gates
    feats = np.zeros((nb, N_FEATURES), dtype=np.float32)
    feats[:, 15] = 1.0 if instance_scale is None else np.log10(max(instance_scale, 1.0)) / 6.0
    p = np.clip(g.quantised_probabilities(), 1e-12, 1.0)
    logp = np.log10(p)
    feats[:, 0] = (logp + 4.0) / 2.0
    if ng == 0 or nb == 0:
        return feats
    depth = g.layers()
    L = max(int(depth.max()), 1)
    gid, src, _ = g.edges()
    gnode = gid + nb
    op = g.gate_op.astype(np.int64)
    fin = g.gate_in_count.astype(np.int64)
    fanout = np.bincount(src, minlength=g.n_nodes)
    # first (lowest-index) parent of every node; ng marks "none"
    first = np.full(g.n_nodes, ng, dtype=np.int64)
    np.minimum.at(first, src, gid)
    # AND / OR counts along the first-parent chain from every gate to the top
    fp_g = first[nb:]
    has_fp = fp_g < ng
    fp_safe = np.where(has_fp, fp_g, 0)
    step_and = np.where(has_fp, (op[fp_safe] == AND).astype(np.float64), 0.0)
    step_or = np.where(has_fp, (op[fp_safe] == OR).astype(np.float64), 0.0)
    step_len = has_fp.astype(np.float64)
    up_and = np.zeros(ng)
    up_or = np.zeros(ng)
    up_len = np.zeros(ng)
    for _ in range(ng + 1):
        na = np.where(has_fp, up_and[fp_safe] + step_and, 0.0)
        no = np.where(has_fp, up_or[fp_safe] + step_or, 0.0)
        nl = np.where(has_fp, up_len[fp_safe] + step_len, 0.0)
        if np.array_equal(na, up_and) and np.array_equal(no, up_or) and np.array_equal(nl, up_len):
            break
        up_and, up_or, up_len = na, no, nl
    # per-event aggregates over parent edges (edges whose input is an event)
    ev = src < nb
    e_src, e_gate = src[ev], gid[ev]
    fo = fanout[:nb].astype(np.float64)
    has = fo > 0
    den = np.where(has, fo, 1.0)
    dmin = np.full(nb, np.iinfo(np.int64).max)
    dmax = np.zeros(nb, dtype=np.int64)
    np.minimum.at(dmin, e_src, depth[e_gate + nb])
    np.maximum.at(dmax, e_src, depth[e_gate + nb])
    cnt_of = lambda m: np.bincount(e_src, weights=m.astype(np.float64), minlength=nb)
    feats[:, 1] = fo / 4.0
    feats[has, 2] = dmin[has] / L
    feats[has, 3] = dmax[has] / L
    feats[has, 4] = (cnt_of(op[e_gate] == AND) / den)[has]
    feats[has, 5] = (cnt_of(op[e_gate] == OR) / den)[has]
    feats[has, 6] = (cnt_of(op[e_gate] == ATLEAST) / den)[has]
    feats[has, 7] = (np.bincount(e_src, weights=fin[e_gate].astype(np.float64), minlength=nb) / den / 8.0)[has]
    is_k = op[e_gate] == ATLEAST
    kn = (g.gate_k.astype(np.float64)[e_gate] / np.maximum(fin[e_gate], 1))
    n_k = np.bincount(e_src[is_k], minlength=nb).astype(np.float64)
    s_k = np.bincount(e_src[is_k], weights=kn[is_k], minlength=nb)
    feats[:, 8] = np.where(n_k > 0, s_k / np.maximum(n_k, 1.0), 0.0)
    # siblings under the first parent
    q0 = first[:nb]
    q0s = np.where(has, q0, 0)
    occ = np.bincount(e_src[e_gate == q0s[e_src]], minlength=nb).astype(np.float64)
    n_sib = np.where(has, fin[q0s] - occ, 0.0)
    feats[:, 9] = n_sib / 8.0
    in_be = src < nb
    g_be_cnt = np.bincount(gid[in_be], minlength=ng).astype(np.float64)
    g_be_sum = np.bincount(gid[in_be], weights=logp[src[in_be]], minlength=ng)
    g_gate_cnt = np.bincount(gid[~in_be], minlength=ng).astype(np.float64)
    sb_cnt = g_be_cnt[q0s] - occ
    sb_sum = g_be_sum[q0s] - occ * logp
    feats[:, 10] = np.where(has & (sb_cnt > 0), (sb_sum / np.maximum(sb_cnt, 1.0) + 4.0) / 2.0, 0.0)
    feats[:, 11] = np.where(has & (n_sib > 0), g_gate_cnt[q0s] / np.maximum(n_sib, 1.0), 0.0)
    feats[:, 12] = np.where(has, (dmax == L).astype(np.float64), 0.0)
    feats[:, 13] = np.where(has, up_and[q0s] / np.maximum(up_len[q0s] + 1, 1), 0.0)
    feats[:, 14] = np.where(has, up_or[q0s] / np.maximum(up_len[q0s] + 1, 1), 0.0)
    if importance:
        pr, cond = approx if approx is not None else approximate_importance(g)
        pp = np.where(has, pr[np.where(has, q0s + nb, 0)], 1.0)
        feats[:, 11] = np.log10(np.clip(pp, 1e-30, 1.0)) / 10.0 + 1.0
        feats[:, 12] = np.log10(np.clip(cond, 1e-12, 1.0)) / 4.0 + 1.0
    return feats


class ImportanceSampler:
    """Proposal sampling with FP64 likelihood ratios over one tree (root tallied)."""

    def __init__(self, g: FlatGraph, device: int = 0, chunk_words: int = 0):
        self.lib = _capi.load()
        self.graph = g.with_tallies([g.root])
        self._view = _capi.GraphView(self.graph)
        run = _capi.RunDesc(mode=_capi.MODE_STAGED, device=device, layered_max_words=chunk_words)
        self.h = _vp()
        _capi.check(self.lib.mcg_is_create(C.byref(self._view.desc), C.byref(run), C.byref(self.h)))

    def close(self):
        if getattr(self, "h", None):
            self.lib.mcg_is_destroy(self.h)
            self.h = None

    __del__ = close

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def proposal_thresholds(self, q: np.ndarray) -> np.ndarray:
        """Thresholds for proposal probabilities q; events with a constant
        nominal word (p = 0 or 1) keep their nominal threshold."""
        thr = probability_threshold(np.clip(q, 0.0, 1.0))
        thr = np.clip(thr, 1, (1 << 32) - 1).astype(np.uint64)
        fixed = (self.graph.be_threshold == 0) | (self.graph.be_threshold >= (1 << 32))
        thr[fixed] = self.graph.be_threshold[fixed]
        return np.ascontiguousarray(thr, dtype=np.uint64)

    def run(self, q_thresholds: np.ndarray, iteration: int = 1, word_begin: int = 0, word_count: int = 1 << 20,
            ce: bool = False):
        q_thresholds = np.ascontiguousarray(q_thresholds, dtype=np.uint64)
        res = IsResult()
        ce_num = np.zeros(max(self.graph.n_be, 1), dtype=np.float64) if ce else None
        _capi.check(self.lib.mcg_is_run(self.h, _p(q_thresholds, C.c_uint64), iteration, word_begin, word_count,
                                        C.byref(res), _p(ce_num, C.c_double) if ce else None))
        out = res.as_dict()
        if ce:
            out["ce_num"] = ce_num[: self.graph.n_be]
        return out


class ProposalMLP:
    """16 -> 64 -> 64 -> 1 sigmoid network on the GPU."""

    def __init__(self, device: int = 0, seed: int = 7):
        self.lib = _capi.load()
        self.h = _vp()
        _capi.check(self.lib.mcg_mlp_create(device, seed, C.byref(self.h)))

    def close(self):
        if getattr(self, "h", None):
            self.lib.mcg_mlp_destroy(self.h)
            self.h = None

    __del__ = close

    def params(self) -> np.ndarray:
        out = np.zeros(N_PARAMS, dtype=np.float32)
        _capi.check(self.lib.mcg_mlp_get_params(self.h, _p(out, C.c_float)))
        return out

    def set_params(self, params: np.ndarray) -> None:
        params = np.ascontiguousarray(params, dtype=np.float32)
        _capi.check(self.lib.mcg_mlp_set_params(self.h, _p(params, C.c_float)))

    def forward(self, feats: np.ndarray) -> np.ndarray:
        feats = np.ascontiguousarray(feats, dtype=np.float32)
        q = np.zeros(feats.shape[0], dtype=np.float32)
        _capi.check(self.lib.mcg_mlp_forward(self.h, _p(feats, C.c_float), feats.shape[0], _p(q, C.c_float)))
        return q

    def grad(self, feats, targets, weights=None):
        feats = np.ascontiguousarray(feats, dtype=np.float32)
        targets = np.ascontiguousarray(targets, dtype=np.float32)
        w = None if weights is None else np.ascontiguousarray(weights, dtype=np.float32)
        g = np.zeros(N_PARAMS, dtype=np.float32)
        loss = C.c_float()
        _capi.check(self.lib.mcg_mlp_grad(self.h, _p(feats, C.c_float), _p(targets, C.c_float),
                                          _p(w, C.c_float) if w is not None else None, feats.shape[0],
                                          _p(g, C.c_float), C.byref(loss)))
        return g, float(loss.value)

    def train(self, feats, targets, weights=None, steps: int = 200, lr: float = 3e-3) -> float:
        feats = np.ascontiguousarray(feats, dtype=np.float32)
        targets = np.ascontiguousarray(targets, dtype=np.float32)
        w = None if weights is None else np.ascontiguousarray(weights, dtype=np.float32)
        loss = C.c_float()
        _capi.check(self.lib.mcg_mlp_train(self.h, _p(feats, C.c_float), _p(targets, C.c_float),
                                           _p(w, C.c_float) if w is not None else None, feats.shape[0], steps, lr,
                                           C.byref(loss)))
        ms = C.c_double()
        _capi.check(self.lib.mcg_mlp_train_time(self.h, C.byref(ms)))
        self.last_train_ms = float(ms.value)
        return float(loss.value)


@dataclass
class CeHistory:
    rounds: List[dict] = field(default_factory=list)
    seconds: float = 0.0
    gpu_ms: float = 0.0


def initial_proposal(sampler: ImportanceSampler, p: np.ndarray, probe_words: int = 1 << 16,
                     min_hits: int = 200, max_scale: float = 1e6):
    """Uniform inflation q = min(p * s, 0.5), doubling s until a probe run of the
    plain (biased) sampler sees at least min_hits top-event failures."""
    s = 1.0
    gpu_ms = 0.0
    while True:
        q = np.minimum(p * s, 0.5)
        r = sampler.run(sampler.proposal_thresholds(q), iteration=1, word_begin=0, word_count=probe_words)
        gpu_ms += r["kernel_ms"]
        if r["hits"] >= min_hits or s >= max_scale:
            return q, s, gpu_ms
        s *= 2.0


def cross_entropy(g: FlatGraph, rounds: int = 5, words_per_round: int = 1 << 20, mlp: Optional[ProposalMLP] = None,
                  smoothing: float = 0.7, train_steps: int = 300, lr: float = 3e-3, q_max: float = 0.5,
                  device: int = 0, sampler: Optional[ImportanceSampler] = None):
    """Cross-entropy training of the proposal.  Each round samples
    words_per_round * 64 samples with the current proposal (passes 2, 3, ...,
    so rounds use fresh random numbers), sets the target of event i to the
    likelihood-weighted frequency of x_i = 1 among top-event failures,
    smooths it with the current proposal and fits the network to it.
    Returns (q, mlp, history)."""
    t0 = time.perf_counter()
    own = sampler is None
    sampler = sampler or ImportanceSampler(g, device=device)
    p = g.quantised_probabilities()
    feats = event_features(g)
    mlp = mlp or ProposalMLP(device=device)
    hist = CeHistory()
    q, scale, ms = initial_proposal(sampler, p)
    hist.gpu_ms += ms
    hist.rounds.append({"round": 0, "scale": scale})
    for r in range(rounds):
        res = sampler.run(sampler.proposal_thresholds(q), iteration=2 + r, word_begin=0,
                          word_count=words_per_round, ce=True)
        hist.gpu_ms += res["kernel_ms"]
        if res["sum_w"] <= 0 or res["hits"] == 0:
            hist.rounds.append({"round": r + 1, "hits": 0})
            break
        target = np.clip(res["ce_num"] / res["sum_w"], 1e-7, q_max)
        target = smoothing * target + (1.0 - smoothing) * q
        loss = mlp.train(feats, target.astype(np.float32), steps=train_steps, lr=lr)
        q = np.clip(mlp.forward(feats).astype(np.float64), 1e-7, q_max)
        hist.rounds.append({"round": r + 1, "hits": res["hits"], "estimate": res["estimate"],
                            "rel_err": res["rel_err"], "ess": res["ess"], "loss": loss})
    hist.seconds = time.perf_counter() - t0
    if own:
        sampler.close()
    return q, mlp, hist


def estimate(sampler: ImportanceSampler, q: np.ndarray, target_rel_err: float = 0.05, words_per_batch: int = 1 << 20,
             max_words: int = 1 << 28, iteration: int = 100, ess_floor: float = 50.0):
    """Runs batches until the relative standard error at 95% confidence
    (1.96 * std_err / estimate) is at most target_rel_err.  Returns the
    pooled result; 'fallback' is set when the effective sample size stays
    below ess_floor (the proposal is unreliable and the plain sampler should
    be used instead)."""
    thr = sampler.proposal_thresholds(q)
    n = sw = sw2 = 0.0
    hits = 0
    gpu_ms = 0.0
    used = 0
    b = 0
    while used < max_words:
        r = sampler.run(thr, iteration=iteration, word_begin=used, word_count=words_per_batch)
        gpu_ms += r["kernel_ms"]
        used += words_per_batch
        b += 1
        n += r["samples"]
        sw += r["sum_w"]
        sw2 += r["sum_w2"]
        hits += r["hits"]
        est = sw / n
        var = max(sw2 / n - est * est, 0.0)
        se = np.sqrt(var / max(n - 1, 1))
        rel95 = 1.96 * se / est if est > 0 else np.inf
        ess = sw * sw / sw2 if sw2 > 0 else 0.0
        if rel95 <= target_rel_err and ess >= ess_floor:
            break
    return {"estimate": est, "std_err": se, "rel_err95": rel95, "samples": int(n), "hits": hits, "ess": ess,
            "batches": b, "gpu_ms": gpu_ms, "fallback": bool(ess < ess_floor)}


# --- many trees at once -------------------------------------------------------

def _proposal_thr(nominal: np.ndarray, q: np.ndarray) -> np.ndarray:
    thr = probability_threshold(np.clip(q, 0.0, 1.0))
    thr = np.clip(thr, 1, (1 << 32) - 1).astype(np.uint64)
    fixed = (nominal == 0) | (nominal >= (1 << 32))
    thr[fixed] = nominal[fixed]
    return np.ascontiguousarray(thr, dtype=np.uint64)


class BatchedImportanceSampler:
    """Proposal sampling over many trees joined into one graph (mcg_is_batch_*).

    ``run`` returns per-tree FP64 sums over word_count * 64 samples of every
    tree; tree k's events are ``slice(be_begin[k], be_begin[k + 1])`` of the
    joined graph."""

    def __init__(self, graphs, device: int = 0, chunk_words: int = 0):
        self.lib = _capi.load()
        self.graphs = list(graphs)
        self.union, self.be_begin, self.roots = concat(self.graphs)
        self._view = _capi.GraphView(self.union)
        self._be_begin32 = np.ascontiguousarray(self.be_begin, dtype=np.uint32)
        run = _capi.RunDesc(mode=_capi.MODE_STAGED, device=device, layered_max_words=chunk_words)
        self.h = _vp()
        _capi.check(self.lib.mcg_is_batch_create(C.byref(self._view.desc), len(self.graphs),
                                                 _p(self._be_begin32, C.c_uint32), C.byref(run), C.byref(self.h)))

    @property
    def n_trees(self) -> int:
        return len(self.graphs)

    def close(self):
        if getattr(self, "h", None):
            self.lib.mcg_is_batch_destroy(self.h)
            self.h = None

    __del__ = close

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def proposal_thresholds(self, q: np.ndarray) -> np.ndarray:
        """Thresholds for proposal probabilities q over all events of the joined
        graph (events with a constant nominal word keep it)."""
        return _proposal_thr(self.union.be_threshold, q)

    def run(self, q_thresholds: np.ndarray, iteration: int = 1, word_begin: int = 0, word_count: int = 1 << 14,
            ce: bool = False, q_defensive: Optional[np.ndarray] = None, words_defensive=0,
            words_cutset: int = 0, q_cutset: Optional[np.ndarray] = None) -> dict:
        """Per-tree sums of one pass.  q_defensive ([n_be] or [n_comp, n_be]
        thresholds) with words_defensive (an int or one per component): the
        main proposal draws the first words, each defensive proposal the next
        words_defensive[c], the cut-set component the last words_cutset, and
        samples carry the balance-heuristic weight.  q_cutset ([n_be]
        thresholds): the cut-set component's proposal for the events read by
        several gates (default: their nominal thresholds)."""
        q_thresholds = np.ascontiguousarray(q_thresholds, dtype=np.uint64)
        nb = self.union.n_be
        if q_thresholds.shape != (nb,):
            raise ValueError("one proposal threshold per event of the joined graph")
        qd, wd, n_def = None, None, 0
        if q_defensive is not None:
            qd = np.ascontiguousarray(np.atleast_2d(q_defensive), dtype=np.uint64)
            if qd.shape[1] != nb:
                raise ValueError("one defensive threshold per event of the joined graph")
            n_def = qd.shape[0]
            wd = np.ascontiguousarray(np.broadcast_to(np.asarray(words_defensive, dtype=np.uint64), (n_def,)))
        sums = np.zeros((self.n_trees, 4), dtype=np.float64)
        ce_num = np.zeros(max(nb, 1), dtype=np.float64) if ce else None
        ms = C.c_double()
        qc = None
        if q_cutset is not None:
            qc = np.ascontiguousarray(q_cutset, dtype=np.uint64)
            if qc.shape != (nb,):
                raise ValueError("one cut-set proposal threshold per event of the joined graph")
        _capi.check(self.lib.mcg_is_batch_run(self.h, _p(q_thresholds, C.c_uint64), n_def,
                                              _p(qd, C.c_uint64) if n_def else None,
                                              _p(wd, C.c_uint64) if n_def else None, int(words_cutset),
                                              _p(qc, C.c_uint64) if qc is not None else None,
                                              iteration, word_begin, word_count, _p(sums, C.c_double),
                                              _p(ce_num, C.c_double) if ce else None, C.byref(ms)))
        out = {"sum_w": sums[:, 0].copy(), "sum_w2": sums[:, 1].copy(), "hits": sums[:, 2].astype(np.int64),
               "max_log_w": sums[:, 3].copy(), "samples": int(word_count) * 64, "kernel_ms": float(ms.value)}
        if ce:
            out["ce_num"] = ce_num[: self.union.n_be]
        return out


@dataclass
class BatchedIsResult:
    estimate: np.ndarray          # per tree
    rel_err95: np.ndarray         # 1.96 * std_err / estimate
    samples: np.ndarray
    hits: np.ndarray
    ess: np.ndarray
    converged: np.ndarray         # reached the target error
    fallback: np.ndarray          # sampled with the nominal probabilities (weights collapsed)
    scale: np.ndarray             # probe inflation per tree
    gpu_ms: dict                  # device time per phase (CUDA events)
    seconds: dict                 # wall time per phase
    q: np.ndarray = None          # final proposal of every event (trees concatenated)
    be_begin: np.ndarray = None   # tree k's events: q[be_begin[k]:be_begin[k + 1]]
    rounds: List[dict] = field(default_factory=list)


def _prepare_one(g: FlatGraph, n_modes: int, importance: bool):
    """Per-tree host inputs of the batched driver: features (the per-tree
    input 15 filled in later) and the uncapped mode proposals, from one
    independence-approximation pass conditioned on the top and on each mode;
    and for a tree with events read by several gates whose gates are each read
    once, their conditional probabilities given the top (shared_posteriors;
    None when the tree has no shared event or they cannot be computed), and
    where they cannot be computed the heuristic seed (shared_seed; else None)."""
    pr, cond = approximate_importance(g, root=[g.root] + _mode_kids(g))
    post = seed = None
    if cut_set_eligible(g) and shared_events(g).any():
        r = shared_posteriors(g)
        post = None if r is None else r[1]
        if post is None:
            seed = shared_seed(g)
    return (event_features(g, instance_scale=1.0, importance=importance, approx=(pr, cond[0])),
            mode_proposals(g, n_modes, 1.0, approx=(pr, cond)), post, seed)


def prepare_trees_async(graphs, n_modes: int, importance: bool, executor):
    """Starts _prepare_one for every tree on an executor (the tasks are
    submitted now, one tree each, the largest first so that no worker is left
    with several of them at the end) and returns a function that waits for
    the results, in the order of `graphs`."""
    order = sorted(range(len(graphs)), key=lambda k: -graphs[k].n_be)
    futures = [executor.submit(_prepare_one, graphs[k], n_modes, importance) for k in order]

    def collect():
        out = [None] * len(graphs)
        for k, f in zip(order, futures):
            out[k] = f.result()
        return out
    return collect


def prepare_trees(graphs, n_modes: int = 4, importance: bool = True, workers=0):
    """_prepare_one for every tree, in `workers` spawned processes when > 1,
    or on `workers` itself when it is an executor (a process pool kept across
    calls, whose start-up is then not paid again)."""
    if hasattr(workers, "map"):
        n = getattr(workers, "_max_workers", 1) or 1
        return list(workers.map(_prepare_one, graphs, [n_modes] * len(graphs), [importance] * len(graphs),
                                chunksize=max(1, len(graphs) // (4 * n))))
    if workers and workers > 1 and len(graphs) > 1:
        import multiprocessing as mp
        from concurrent.futures import ProcessPoolExecutor
        with ProcessPoolExecutor(max_workers=workers, mp_context=mp.get_context("spawn")) as ex:
            return list(ex.map(_prepare_one, graphs, [n_modes] * len(graphs), [importance] * len(graphs),
                               chunksize=max(1, len(graphs) // (4 * workers))))
    return [_prepare_one(g, n_modes, importance) for g in graphs]


def _rel95(n, sw, sw2):
    est = np.where(n > 0, sw / np.maximum(n, 1), 0.0)
    var = np.maximum(sw2 / np.maximum(n, 1) - est * est, 0.0)
    se = np.sqrt(var / np.maximum(n - 1, 1))
    with np.errstate(divide="ignore", invalid="ignore"):
        rel = np.where(est > 0, 1.96 * se / np.where(est > 0, est, 1.0), np.inf)
    return est, rel


def _train_shared(mlp: "ProposalMLP", feats, targets, steps, lr, weights=None, group=None):
    """Fits the shared network to the rows of every rank: the rows are
    gathered to all ranks, rank 0's trained parameters are broadcast."""
    if group is None:
        import torch.distributed as dist
        if not (dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1):
            return mlp.train(feats, targets, weights, steps=steps, lr=lr)
    from . import parallel
    if weights is not None:
        feats = np.concatenate([feats, np.asarray(weights, dtype=np.float32)[:, None]], axis=1)
    feats, targets = parallel.allgather_rows(feats, targets, group=group)
    if weights is not None:
        feats, weights = np.ascontiguousarray(feats[:, :-1]), np.ascontiguousarray(feats[:, -1])
    loss = mlp.train(feats, targets, weights, steps=steps, lr=lr)
    mlp.set_params(parallel.broadcast_params(mlp.params(), group=group))
    return loss


def batched_learned_is(graphs, target_rel_err: float = 0.05, mlp: Optional[ProposalMLP] = None, device: int = 0,
                       probe_words: int = 1 << 10, min_hits: int = 200, max_probe_rounds: int = 24,
                       ce_rounds: Optional[int] = None, ce_words: int = 1 << 13, smoothing: float = 0.7,
                       train_steps: int = 150,
                       lr: float = 3e-3, q_max: float = 0.5, est_words: int = 1 << 12, max_est_words: int = 1 << 22,
                       ess_floor: float = 50.0, collapse_ratio: float = 1e-3, plain_words: int = 1 << 16,
                       defensive: float = 0.3, chunk_words: int = 0, use_network: bool = True,
                       importance_features: bool = True, tree_weighting: bool = True, fallback_after: int = 2,
                       cap_levels=(0.75, 0.9, 0.97, 0.99), confirm_rounds: int = 1,
                       defensive_proposal: str = "auto", n_modes: int = 4, min_words: int = 0,
                       mode_cap: float = 0.5, workers=0, prepared=None, log=None) -> BatchedIsResult:
    """Learned importance sampling for a batch of rare-event trees.

    1. Probe: q = min(p * s_k, c_k) per tree, s_k x4 per round (x8 without
       a hit) until the probe sees min_hits top-event failures (the plain
       sampler fed the inflated thresholds).  The cap c_k starts at q_max and
       is raised through cap_levels only for a tree whose every event already
       sits at the cap (a top event that needs many near-certain failures);
       the tree's proposals stay below c_k from then on.
    From here on a share `defensive` of every pass's words is drawn from a
    defensive proposal q_d and every sample carries the balance-heuristic
    weight p / (defensive * q_d + (1 - defensive) * q) (mcg_is_batch_run):
    a failure region the learned proposal under-samples is still reached
    through q_d's share, so the estimate stays unbiased with a bounded
    variance instead of silently missing that region.  q_d is, with
    defensive_proposal="cutsets" ("auto" picks it when every tree qualifies),
    the cut-set component of mcg_is_batch_run
    (each sample forces a minimal cut set drawn with probability prod p / S:
    the mixture over all failure modes of the tree, which bounds every
    weight by S / defensive; trees only), with "modes" a mixture of n_modes proposals each
    conditioned on one child of the top OR gate failing (mode_proposals;
    a product proposal cannot follow failure modes of very different order
    at once, a mixture over the top gate's children can), with "approx" the
    single approximate zero-variance proposal P~(x_i = 1 | top), with
    "probe" the probe's inflation; all clipped to the tree's cap (the mode
    proposals to max(cap, mode_cap): a child's failure that needs all of
    its events is only reached often when they may come close to 1).  The
    first cross-entropy round samples q_d alone.
    2. Cross-entropy rounds over all trees at once (ce_rounds: 1 with the
       cut-set component, whose samples already follow the failure region,
       5 otherwise): per-event targets are the
       likelihood-weighted failure frequencies, smoothed with the current
       proposal; one network, whose 16th input is the tree's log10 s_k / 6,
       is fitted to the rows of all trees (each tree weighing the same in the
       loss with tree_weighting) and gives every tree's next q.
    3. Estimate rounds with doubling words; a tree leaves the batch once
       1.96 * std_err / estimate <= target_rel_err with ESS >= ess_floor
       at the end of confirm_rounds consecutive rounds and after at least
       min_words words (a product-form proposal can leave a failure mode
       almost unsampled; a sample that has not met it yet shows a small
       error around a low estimate, so a floor on the sample count guards
       the error estimate),
       and the joined graph is rebuilt from the trees left.  A tree whose
       ESS / hits falls below collapse_ratio after its first estimate round
       is re-run with its nominal probabilities (plain Monte Carlo, weights 1)
       and reported as a fallback.
    Every round draws fresh Philox counters (its own pass number).  The
    per-tree host inputs (features, mode proposals) are computed by
    prepare_trees, in `workers` processes, unless given as `prepared`; when
    `workers` is an executor they are computed while the probe runs.
    use_network=False takes the smoothed cross-entropy targets themselves as
    the next proposal (the method without the network, for comparison);
    importance_features=False leaves the independence-approximation inputs
    out of the features (event_features)."""
    say = log or (lambda *a: None)
    n = len(graphs)
    t_all = time.perf_counter()
    gpu = {"probe": 0.0, "ce": 0.0, "estimate": 0.0}
    wall = {"features": 0.0, "probe": 0.0, "ce": 0.0, "train": 0.0, "estimate": 0.0, "rebuild": 0.0}
    rounds = []
    t0 = time.perf_counter()
    collect = None
    if prepared is None:
        if hasattr(workers, "map"):  # a kept pool: the host inputs are computed while the probe runs
            collect = prepare_trees_async(graphs, n_modes, importance_features, workers)
        else:
            prepared = prepare_trees(graphs, n_modes, importance_features, workers)
    wall["features"] = time.perf_counter() - t0
    t0 = time.perf_counter()
    full = BatchedImportanceSampler(graphs, device=device, chunk_words=chunk_words)
    wall["rebuild"] += time.perf_counter() - t0
    bb = full.be_begin
    p = full.union.quantised_probabilities()
    sl = [slice(int(bb[k]), int(bb[k + 1])) for k in range(n)]
    tree_of_event = np.repeat(np.arange(n), np.diff(bb))
    # 1. probe
    t0 = time.perf_counter()
    scale = np.ones(n)
    cap = np.full(n, float(q_max))
    ok = np.zeros(n, dtype=bool)
    p_min = np.array([float(p[sl[k]][p[sl[k]] > 0].min()) if np.any(p[sl[k]] > 0) else 1.0 for k in range(n)])
    it = 1
    probe, probing = full, np.arange(n)  # the joined graph of the trees still probed
    for r in range(max_probe_rounds):
        left = np.nonzero(~ok)[0]
        if left.size <= probing.size // 2:
            t1 = time.perf_counter()
            if probe is not full:
                probe.close()
            probe, probing = BatchedImportanceSampler([graphs[k] for k in left], device=device,
                                                      chunk_words=chunk_words), left
            wall["rebuild"] += time.perf_counter() - t1
        q = np.concatenate([np.minimum(p[sl[k]] * scale[k], cap[k]) for k in probing])
        res = probe.run(probe.proposal_thresholds(q), iteration=it, word_count=probe_words)
        it += 1
        gpu["probe"] += res["kernel_ms"]
        ok[probing] |= res["hits"] >= min_hits
        hits = np.zeros(n, dtype=np.int64)
        hits[probing] = res["hits"]
        rounds.append({"phase": "probe", "round": r, "trees_left": int((~ok).sum()), "ms": res["kernel_ms"]})
        if ok.all():
            break
        saturated = ~ok & (scale * p_min >= cap)
        for k in np.nonzero(saturated)[0]:
            higher = [c for c in cap_levels if c > cap[k]]
            if higher:
                cap[k] = higher[0]
        grow = ~ok & ~saturated
        scale = np.where(grow, scale * np.where(hits == 0, 8.0, 4.0), scale)
        scale = np.minimum(scale, cap / p_min)
    if probe is not full:
        probe.close()
    wall["probe"] = time.perf_counter() - t0
    if collect is not None:  # what the host inputs still take after the probe
        t0 = time.perf_counter()
        prepared = collect()
        wall["features"] += time.perf_counter() - t0
    # 2. cross-entropy rounds with the shared network
    feats = np.concatenate([pr[0] for pr in prepared])
    feats[:, 15] = (np.log10(np.maximum(scale, 1.0)) / 6.0)[tree_of_event]
    mlp = mlp or (ProposalMLP(device=device) if use_network else None)
    cap_e = cap[tree_of_event]
    eligible = np.array([cut_set_eligible(g) for g in graphs])
    if defensive_proposal == "auto":  # per tree: cut sets where it takes them, mode proposals where not
        defensive_proposal = "cutsets" if eligible.all() else ("modes" if not eligible.any() else "mixed")
    mixed = defensive_proposal == "mixed"
    cut = defensive_proposal in ("cutsets", "mixed")
    if ce_rounds is None:  # cut-set samples give near-ideal targets at once
        ce_rounds = 1 if defensive_proposal == "cutsets" else 5
    elig_e = eligible[tree_of_event]
    if defensive_proposal == "cutsets":
        bad = [k for k, g in enumerate(graphs) if not eligible[k]]
        if bad:
            raise ValueError(f"cut-set sampling needs trees of AND/OR/ATLEAST gates without negations and without "
                             f"gates read by several gates; trees {bad[:5]} are not")
        q_def = np.zeros((0, full.union.n_be))
    elif mixed:  # mode proposals for the trees the cut-set component cannot draw, the main proposal
        # again for the others (their rows follow it round by round)
        q_def = np.clip(np.concatenate([pr[1] for pr in prepared], axis=1), 1e-7,
                        np.maximum(cap_e, mode_cap)[None, :])
        q_def[:, elig_e] = np.minimum(p * scale[tree_of_event], cap_e)[elig_e][None, :]
    elif defensive_proposal == "modes":
        q_def = np.clip(np.concatenate([pr[1] for pr in prepared], axis=1), 1e-7,
                        np.maximum(cap_e, mode_cap)[None, :])
    elif defensive_proposal == "approx":
        q_def = np.concatenate([np.clip(approximate_importance(g)[1], 1e-7, cap[k])
                                for k, g in enumerate(graphs)])[None, :]
    elif defensive_proposal == "probe":
        q_def = np.minimum(p * scale[tree_of_event], cap_e)[None, :]
    else:
        raise ValueError("defensive_proposal must be 'auto', 'cutsets', 'mixed', 'modes', 'approx' or 'probe'")
    n_comp = q_def.shape[0]

    # Events read by several gates: the cut-set component draws them first,
    # from r = their conditional failure probability given the top (the
    # product proposal's cross-entropy optimum): the posterior of
    # shared_posteriors where it was computed, else the event's own
    # cross-entropy target above a floor of half of shared_seed's generous
    # estimate (so that a cut set of several shared events that the first
    # samples under-weigh is still drawn), at most 0.9; then the cut set on
    # the tree conditioned on them.
    shared_u = (np.concatenate([shared_events(g) for g in graphs]) & elig_e if cut
                else np.zeros(full.union.n_be, bool))
    has_shared = bool(shared_u.any())

    def z_thr(rv, smp=None):  # thresholds of the cut-set component: r (per event of the union) on the shared events
        if not has_shared:
            return None
        smp = full if smp is None else smp
        rs = rv if smp is full else np.concatenate([rv[sl[k]] for k in members])
        return smp.proposal_thresholds(np.where(shared_u_of(smp), rs, p_of(smp)))

    def r_now():  # the posterior where computed, else the event's own target above its floor
        return np.where(post_fixed, r0, np.minimum(np.maximum(np.maximum(p, r_floor), z_target), 0.9))

    def shared_u_of(smp):
        return shared_u if smp is full else np.concatenate([shared_u[sl[k]] for k in members])

    def p_of(smp):
        return p if smp is full else np.concatenate([p[sl[k]] for k in members])

    r0 = p.copy()
    r_floor = np.zeros(full.union.n_be)
    z_target = np.zeros(full.union.n_be)  # the shared events' own cross-entropy targets
    explore = np.zeros(full.union.n_be)
    # Shared events of the trees whose posteriors were computed keep r = the posterior in every
    # round: it is the cross-entropy optimum of their product proposal, and lifting the many
    # shared events that hardly matter (posterior ~ p) above p, as noisy targets do, spreads
    # log(p(z) / r(z)) over a range that grows with their number (sd ~ 11 over 1,665 such events
    # at r ~ 7 p), which leaves the estimate to a few samples with few of them drawn.
    post_fixed = np.zeros(full.union.n_be, dtype=bool)
    if has_shared:
        # seed: their conditional probabilities given the top (shared_posteriors), half of which
        # stays as a floor; for a tree where those cannot be computed, shared_seed and an
        # exploration round (every shared event at least at 2 / its count, so that pairs of them
        # the seeds miss are drawn together often enough for the first targets to see them)
        needs_exploration = False
        for k, g in enumerate(graphs):
            m = shared_u[sl[k]]
            if not m.any():
                continue
            post = prepared[k][2]
            inc = np.minimum((post if post is not None else prepared[k][3])[m], 0.9)
            r_floor[sl[k]][m] = 0.5 * inc
            r0[sl[k]][m] = np.clip(inc, p[sl[k]][m], 0.9)
            post_fixed[sl[k]] = m & (post is not None)
            if post is None:
                explore[sl[k]][m] = min(0.5, 2.0 / m.sum())
                needs_exploration = True
        if needs_exploration and (ce_rounds is None or ce_rounds < 2):
            ce_rounds = 2

    def def_words(w):  # words per defensive component
        return max(1, int(round(defensive * w / n_comp))) if defensive > 0 and n_comp else 0

    def cut_words(w):  # words of the cut-set component
        return max(1, int(round(defensive * w))) if cut and defensive > 0 else 0
    row_w = (1.0 / np.diff(bb).astype(np.float64))[tree_of_event].astype(np.float32) if tree_weighting else None
    thr_def = np.stack([full.proposal_thresholds(qc) for qc in q_def]) if n_comp else None
    q = None
    t0 = time.perf_counter()
    for r in range(ce_rounds):
        if q is None and cut and not mixed:  # first round: cut-set samples alone
            res = full.run(full.union.be_threshold, iteration=it, word_count=ce_words, ce=True,
                           words_cutset=ce_words, q_cutset=z_thr(np.maximum(r0, explore)) if has_shared else None)
            q = np.minimum(p * scale[tree_of_event], cap_e)
            if has_shared:
                q = np.where(shared_u, r0, q)
        elif q is None and mixed:  # first round: the mode proposals and the cut-set component, half each
            half = ce_words // 2
            res = full.run(thr_def[0], iteration=it, word_count=ce_words, ce=True, q_defensive=thr_def,
                           words_defensive=[half // n_comp + (c < half % n_comp) for c in range(n_comp)],
                           words_cutset=ce_words - half,
                           q_cutset=z_thr(np.maximum(r0, explore)) if has_shared else None)
            q = np.where(elig_e, np.minimum(p * scale[tree_of_event], cap_e), q_def.mean(axis=0))
            if has_shared:
                q = np.where(shared_u, r0, q)
        elif q is None:  # first round: the defensive mixture alone
            res = full.run(thr_def[0], iteration=it, word_count=ce_words, ce=True, q_defensive=thr_def,
                           words_defensive=[ce_words // n_comp + (c < ce_words % n_comp) for c in range(n_comp)])
            q = q_def.mean(axis=0)
        else:
            res = full.run(full.proposal_thresholds(q), iteration=it, word_count=ce_words, ce=True,
                           q_defensive=thr_def if def_words(ce_words) else None, words_defensive=def_words(ce_words),
                           words_cutset=cut_words(ce_words), q_cutset=z_thr(r_now()) if cut_words(ce_words) else None)
        it += 1
        gpu["ce"] += res["kernel_ms"]
        sw = res["sum_w"][tree_of_event]
        hit = sw > 0
        target = np.where(hit, res["ce_num"] / np.where(hit, sw, 1.0), q)
        target = np.clip(target, 1e-7, cap_e)
        if has_shared:  # the cut-set component's shared events follow their own targets (the network
            # smooths across events with alike features, which lifts the many that hardly matter
            # and can miss one tree's particular pair)
            z_target = np.where(shared_u, np.maximum(z_target, target) if r > 0 else target, z_target)
        target = smoothing * target + (1.0 - smoothing) * q
        t1 = time.perf_counter()
        if use_network:
            loss = _train_shared(mlp, feats, target.astype(np.float32), train_steps, lr, weights=row_w)
            q = np.clip(mlp.forward(feats).astype(np.float64), 1e-7, cap_e)
        else:
            loss, q = float("nan"), target
        wall["train"] += time.perf_counter() - t1
        if mixed:  # the cut-set trees' defensive rows follow their main proposal
            q_def[:, elig_e] = q[elig_e][None, :]
            thr_def = np.stack([full.proposal_thresholds(qc) for qc in q_def])
        est, rel = _rel95(res["samples"], res["sum_w"], res["sum_w2"])
        rounds.append({"phase": "ce", "round": r, "ms": res["kernel_ms"], "loss": loss,
                       "median_rel95": float(np.median(rel)), "trees_without_hits": int((res["hits"] == 0).sum())})
        say(rounds[-1])
    wall["ce"] = time.perf_counter() - t0
    # 3. estimate
    t0 = time.perf_counter()
    N = np.zeros(n)
    SW = np.zeros(n)
    SW2 = np.zeros(n)
    H = np.zeros(n, dtype=np.int64)
    converged = np.zeros(n, dtype=bool)
    fallback = np.zeros(n, dtype=bool)
    checked = np.zeros(n, dtype=bool)
    rounds_in = np.zeros(n, dtype=np.int64)
    streak = np.zeros(n, dtype=np.int64)
    q_use = q.copy()
    active = np.arange(n)
    sampler, members = full, active.copy()
    words = est_words
    used = 0
    while active.size and used < max_est_words:
        # the joined graph is rebuilt once the trees still running hold half
        # of its events or fewer; until then finished trees ride along and
        # their sums are left out
        n_ev = np.diff(bb)
        if not np.isin(active, members).all() or 2 * n_ev[active].sum() <= n_ev[members].sum():
            t1 = time.perf_counter()
            sampler.close()  # the joined graph of the trees left replaces it (and its device memory)
            sampler = BatchedImportanceSampler([graphs[k] for k in active], device=device, chunk_words=chunk_words)
            members = active.copy()
            wall["rebuild"] += time.perf_counter() - t1
        qa = np.concatenate([q_use[sl[k]] for k in members])
        qd = np.concatenate([q_def[:, sl[k]] if not fallback[k] else np.repeat(p[sl[k]][None, :], n_comp, axis=0)
                             for k in members], axis=1)
        res = sampler.run(sampler.proposal_thresholds(qa), iteration=it, word_begin=0, word_count=words,
                          q_defensive=np.stack([sampler.proposal_thresholds(qc) for qc in qd]) if def_words(words)
                          else None, words_defensive=def_words(words), words_cutset=cut_words(words),
                          q_cutset=z_thr(r_now(), sampler) if cut_words(words) else None)
        it += 1
        gpu["estimate"] += res["kernel_ms"]
        used += words
        live = np.isin(members, active)
        run_k = members[live]
        N[run_k] += res["samples"]
        SW[run_k] += res["sum_w"][live]
        SW2[run_k] += res["sum_w2"][live]
        H[run_k] += res["hits"][live]
        est, rel = _rel95(N, SW, SW2)
        ess = np.where(SW2 > 0, SW * SW / np.where(SW2 > 0, SW2, 1.0), 0.0)
        ok_now = (rel <= target_rel_err) & (ess >= ess_floor) & (N >= 64.0 * min_words)
        streak[run_k] = np.where(ok_now[run_k], streak[run_k] + 1, 0)
        done = streak >= confirm_rounds
        # weight collapse: few effective samples among many hits after
        # `fallback_after` rounds -> plain sampling
        rounds_in[run_k] += 1
        first = run_k[(~checked[run_k]) & (rounds_in[run_k] >= fallback_after)]
        checked[first] = True
        bad = first[(H[first] > 0) & (ess[first] < collapse_ratio * H[first]) & ~done[first]]
        if cut:  # its weights stay below S / pi: more samples, not plain sampling (hopeless at 1e-9)
            bad = bad[~eligible[bad]]
        for k in bad:
            fallback[k] = True
            q_use[sl[k]] = p[sl[k]]
            N[k] = SW[k] = SW2[k] = 0.0
            H[k] = 0
        converged |= done
        rounds.append({"phase": "estimate", "words": words, "trees": int(run_k.size), "ms": res["kernel_ms"],
                       "converged": int(converged.sum()), "fallback": int(fallback.sum()),
                       "tree_ids": [int(k) for k in run_k[:8]]})
        say(rounds[-1])
        active = np.nonzero(~converged & ~(fallback & (N >= plain_words * 64)))[0]
        words = min(words * 2, max(max_est_words - used, est_words))
    sampler.close()
    full.close()
    wall["estimate"] = time.perf_counter() - t0
    wall["total"] = time.perf_counter() - t_all
    est, rel = _rel95(N, SW, SW2)
    ess = np.where(SW2 > 0, SW * SW / np.where(SW2 > 0, SW2, 1.0), 0.0)
    return BatchedIsResult(estimate=est, rel_err95=rel, samples=N.astype(np.int64), hits=H, ess=ess,
                           converged=converged, fallback=fallback, scale=scale, gpu_ms=gpu, seconds=wall,
                           q=q_use, be_begin=bb, rounds=rounds)
