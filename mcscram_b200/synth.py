"""Seeded synthetic fault trees in the shapes of the benchmark configurations.

The reference measures on the Aralia fault-tree set; synthetic trees with
the benchmark's stated sizes, gate mixes and probability ranges stand in for
it here.  The generator builds a single-top DAG bottom-up in depth layers:

* gate layer sizes grow geometrically from the top (1 gate) downwards and
  level off, so every gate at depth d >= 2 gets one input from depth d - 1
  (fixing the number of layers) and every non-top gate has a parent;
* every basic event is used; a chosen fraction of basic events (or of all
  nodes) gets a second parent, which makes the graph a DAG;
* AND/OR fan-in is drawn uniformly from its range and then nudged, one input
  at a time and never outside the range, until the input slots match the
  edges needed to cover every node and the requested sharing;
* ATLEAST gates take n uniform in their range and k uniform in [2, n - 1];
  XOR gates have two inputs, NOT gates one;
* probabilities are log-uniform in the given range.

The top gate is an OR gate.  Basic events get PDAG indices 2, 3, ...
(core::Pdag::kVariableStartIndex, mcSCRAM src/pdag.h:804) and gates the
indices after them.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Dict, Optional, Tuple

import numpy as np

from .graph import AND, ATLEAST, NOT, OR, XOR, FlatGraph, probability_threshold


@dataclass
class TreeSpec:
    n_be: int
    n_gates: int
    mix: Dict[int, float]                      # connective -> fraction of gates
    p_range: Tuple[float, float]
    seed: int
    n_layers: Optional[int] = None
    fanin: Tuple[int, int] = (2, 4)            # AND/OR fan-in range
    atleast_n: Tuple[int, int] = (3, 8)
    atleast_k_max_offset: int = 1              # k in [2, n - offset]
    share_be_frac: float = 0.0                 # basic events given >= 2 parents
    share_node_frac: float = 0.0               # nodes (events and gates) given >= 2 parents
    share_scope: Optional[int] = None          # shared events' parents within the subtree of the first
                                               # parent's ancestor this many levels up (None: anywhere)
    name: str = "tree"
    extra: dict = field(default_factory=dict)


def _layer_sizes(n_gates: int, n_layers: int) -> np.ndarray:
    """Sizes for depths 1..n_layers (index 0 = depth 1); top (last) is 1,
    non-increasing with depth, growth at most x2 per layer."""
    if n_layers < 1:
        raise ValueError("n_layers must be >= 1")
    if n_gates < n_layers:
        raise ValueError("need at least one gate per layer")
    # ramp[i] for depth n_layers - i
    lo, hi = 1, n_gates
    while lo < hi:  # smallest cap with sum(min(2^i, cap)) >= n_gates
        cap = (lo + hi) // 2
        s = sum(min(1 << min(i, 40), cap) for i in range(n_layers))
        if s >= n_gates:
            hi = cap
        else:
            lo = cap + 1
    cap = lo
    ramp = [min(1 << min(i, 40), cap) for i in range(n_layers)]
    excess = sum(ramp) - n_gates
    i = n_layers - 1
    while excess > 0:  # trim the bottom layers, keep non-increasing towards the top
        floor_i = ramp[i - 1] if i > 0 else 1
        can = ramp[i] - floor_i
        take = min(can, excess)
        ramp[i] -= take
        excess -= take
        i -= 1
        if i < 0:
            i = n_layers - 1
    deficit = n_gates - sum(ramp)  # only when 2^n_layers - 1 < n_gates
    j = n_layers - 1
    while deficit > 0:  # widen the bottom layers
        ramp[j] += 1
        deficit -= 1
        j = j - 1 if j > max(0, n_layers - 3) else n_layers - 1
    sizes = np.array(ramp[::-1], dtype=np.int64)  # depth 1 first
    assert sizes.sum() == n_gates and sizes[-1] == 1
    return sizes


def _default_layers(n_gates: int, fanin_mean: float) -> int:
    # depth of a balanced tree of n_gates gates with the mean fan-in, plus a margin
    d = int(np.ceil(np.log(max(n_gates, 2)) / np.log(max(fanin_mean, 1.5)))) + 2
    return max(2, min(d, n_gates))


def _local_sharing(rng, children, be_req, slots, share_be, B, G, scope):
    """Slot assignment with every shared event's two occurrences in one
    neighbourhood: the subtree of the ancestor `scope` levels above the gate
    of its first occurrence (widened a level at a time when that subtree has
    no other gate with a free slot).  Gates must have one parent each.
    Returns (events, slots) in matching order; the other events fill the
    remaining slots at random."""
    parent = np.full(G, -1, dtype=np.int64)
    for g in range(G):
        for c in children[g]:
            if c >= B:
                parent[c - B] = g
    free_by_gate = {}
    for s in slots:
        free_by_gate[int(s)] = free_by_gate.get(int(s), 0) + 1

    def ancestor(g, h):
        for _ in range(h):
            if parent[g] < 0:
                break
            g = int(parent[g])
        return g

    def subtree_gates(a):
        out, todo = [], [a]
        while todo:
            g = todo.pop()
            out.append(g)
            todo.extend(int(c) - B for c in children[g] if c >= B)
        return out

    ev, sl = [], []
    for e in rng.permutation(np.nonzero(share_be)[0]):
        open_gates = [g for g, n in free_by_gate.items() if n > 0]
        if len(open_gates) < 2:
            raise ValueError("no slots left for a shared event")
        g1 = int(open_gates[rng.integers(len(open_gates))])
        h = scope
        while True:
            cand = [g for g in subtree_gates(ancestor(g1, h)) if g != g1 and free_by_gate.get(g, 0) > 0]
            if cand or ancestor(g1, h) == ancestor(g1, h + 1):
                break
            h += 1
        if not cand:
            raise ValueError("no second slot for a shared event")
        g2 = int(cand[rng.integers(len(cand))])
        for g in (g1, g2):
            free_by_gate[g] -= 1
            ev.append(int(e))
            sl.append(g)
    rest_slots = np.repeat(np.array(list(free_by_gate.keys()), dtype=np.int64),
                           np.array(list(free_by_gate.values()), dtype=np.int64))
    rng.shuffle(rest_slots)
    rest_ev = np.nonzero(~share_be)[0]
    rng.shuffle(rest_ev)
    if rest_slots.size != rest_ev.size:
        raise ValueError("slot/requirement mismatch after placing the shared events")
    return (np.concatenate([np.array(ev, dtype=np.int64), rest_ev]),
            np.concatenate([np.array(sl, dtype=np.int64), rest_slots]))


def generate(spec: TreeSpec) -> FlatGraph:
    rng = np.random.default_rng(spec.seed)
    G, B = spec.n_gates, spec.n_be
    if G < 1 or B < 1:
        raise ValueError("need at least one gate and one basic event")
    L = spec.n_layers or _default_layers(G, (spec.fanin[0] + spec.fanin[1]) / 2)
    sizes = _layer_sizes(G, L)
    depth = np.repeat(np.arange(1, L + 1), sizes)  # gate j (topological) -> depth

    # Connectives: the mix over all gates, top forced to OR.
    kinds = []
    for op, frac in sorted(spec.mix.items()):
        kinds += [op] * int(round(frac * G))
    while len(kinds) < G:
        kinds.append(max(spec.mix, key=spec.mix.get))
    kinds = np.array(kinds[:G], dtype=np.int64)
    rng.shuffle(kinds)
    top = G - 1
    if kinds[top] != OR:
        swap = np.nonzero(kinds == OR)[0]
        if swap.size:
            kinds[swap[0]] = kinds[top]
        kinds[top] = OR
    # NOT gates at depth >= 2 take their one input from depth - 1, which is fine;
    # a NOT at depth 1 takes a basic event.

    # Fan-in.
    fanin = np.zeros(G, dtype=np.int64)
    kvals = np.zeros(G, dtype=np.int64)
    flexible = np.zeros(G, dtype=bool)
    for j in range(G):
        op = kinds[j]
        if op in (AND, OR):
            fanin[j] = rng.integers(spec.fanin[0], spec.fanin[1] + 1)
            flexible[j] = True
        elif op == ATLEAST:
            n = int(rng.integers(spec.atleast_n[0], spec.atleast_n[1] + 1))
            fanin[j] = n
            kvals[j] = int(rng.integers(2, max(2, n - spec.atleast_k_max_offset) + 1))
        elif op == XOR:
            fanin[j] = 2
        elif op == NOT:
            fanin[j] = 1
        else:
            raise ValueError(f"unsupported connective {op} in generator")

    # Which nodes get a second parent.
    share_be = np.zeros(B, dtype=bool)
    share_gate = np.zeros(G, dtype=bool)
    if spec.share_node_frac > 0:
        n_share = int(round(spec.share_node_frac * (B + G)))
        pick = rng.choice(B + G - 1, size=min(n_share, B + G - 1), replace=False)  # top excluded
        for x in pick:
            if x < B:
                share_be[x] = True
            else:
                share_gate[x - B] = True
    if spec.share_be_frac > 0:
        n_share = int(round(spec.share_be_frac * B))
        share_be[rng.choice(B, size=n_share, replace=False)] = True
    # gates sharing must have a possible second parent above them
    share_gate[depth >= L - 1] = False
    need_be = 1 + share_be.astype(np.int64)
    need_gate = np.where(np.arange(G) == top, 0, 1 + share_gate.astype(np.int64))
    demand = int(need_be.sum() + need_gate.sum())

    # Match supply (sum of fan-in) to demand within the AND/OR ranges.
    supply = int(fanin.sum())
    flex_idx = np.nonzero(flexible)[0]
    guard = 0
    while supply != demand:
        guard += 1
        if guard > 50 * (G + B) or flex_idx.size == 0:
            raise ValueError(f"cannot match fan-in supply {supply} to demand {demand} within ranges")
        j = int(flex_idx[rng.integers(flex_idx.size)])
        if supply < demand and fanin[j] < spec.fanin[1]:
            fanin[j] += 1
            supply += 1
        elif supply > demand and fanin[j] > spec.fanin[0]:
            fanin[j] -= 1
            supply -= 1

    children = [[] for _ in range(G)]
    parents_of = [set() for _ in range(G)]
    free = fanin.copy()
    rem_gate = need_gate.copy()
    by_depth = [np.nonzero(depth == d)[0] for d in range(L + 1)]

    # A: depth edges, distinct children from the layer below.
    for d in range(L, 1, -1):
        parents = by_depth[d]
        below = by_depth[d - 1].copy()
        rng.shuffle(below)
        for i, p in enumerate(parents):
            c = int(below[i % below.size])
            children[p].append(B + c)
            parents_of[c].add(int(p))
            free[p] -= 1
            rem_gate[c] -= 1

    # B: remaining gate requirements, the highest (most constrained) layers first.
    above_cache = {}
    widened = 0
    for d in range(L - 1, 0, -1):
        for c in by_depth[d]:
            while rem_gate[c] > 0:
                cand = above_cache.get(d)
                if cand is None:
                    cand = np.nonzero(depth > d)[0]
                    above_cache[d] = cand
                ok = cand[(free[cand] > 0)]
                if parents_of[c]:
                    ok = ok[~np.isin(ok, list(parents_of[c]))]
                if ok.size == 0:
                    # Widen an AND/OR gate above by one input and narrow another
                    # AND/OR gate with a free slot, so the totals still match.
                    grow = [p for p in cand if flexible[p] and p not in parents_of[c]]
                    shrink = [q for q in np.nonzero(flexible & (free > 0) & (fanin > spec.fanin[0]))[0]]
                    if not grow or not shrink:
                        raise ValueError("generator ran out of parent slots for gates; adjust layers/fan-in")
                    p = int(grow[rng.integers(len(grow))])
                    q = int(shrink[rng.integers(len(shrink))])
                    fanin[p] += 1
                    free[p] += 1
                    fanin[q] -= 1
                    free[q] -= 1
                    widened += 1
                    continue
                w = free[ok].astype(np.float64)
                p = int(rng.choice(ok, p=w / w.sum()))
                children[p].append(B + int(c))
                parents_of[c].add(p)
                free[p] -= 1
                rem_gate[c] -= 1

    # C: basic events into the remaining slots.
    be_req = np.repeat(np.arange(B), need_be)
    rng.shuffle(be_req)
    slots = np.repeat(np.arange(G), free)
    rng.shuffle(slots)
    if slots.size != be_req.size:
        raise ValueError(f"slot/requirement mismatch {slots.size} vs {be_req.size}")
    if spec.share_scope is not None and share_be.any():
        be_req, slots = _local_sharing(rng, children, be_req, slots, share_be, B, G, spec.share_scope)
    # assign avoiding duplicate children; repair collisions by swapping
    assign = slots.copy()
    child_sets = [set(ch) for ch in children]
    pending = []
    for i, e in enumerate(be_req):
        p = int(assign[i])
        if int(e) in child_sets[p]:
            pending.append(i)
        else:
            child_sets[p].add(int(e))
    for i in pending:
        e = int(be_req[i])
        placed = False
        for _ in range(200):
            k = int(rng.integers(be_req.size))
            if k == i:
                continue
            p, q = int(assign[i]), int(assign[k])
            ek = int(be_req[k])
            # swap parents of i and k if both stay duplicate-free
            if e not in child_sets[q] and (ek == e or ek not in child_sets[p]) and k not in pending:
                child_sets[q].discard(ek)
                child_sets[q].add(e)
                child_sets[p].add(ek)
                assign[i], assign[k] = q, p
                placed = True
                break
        if not placed:
            raise ValueError("could not place a basic event without duplicate inputs")
    for i, e in enumerate(be_req):
        children[int(assign[i])].append(int(e))

    # Flatten.
    inputs, in_begin, in_count = [], [], []
    for j in range(G):
        ch = sorted(children[j], key=lambda x: (x < B, x))  # gate inputs first, then events
        in_begin.append(len(inputs))
        in_count.append(len(ch))
        inputs.extend(ch)
    lo, hi = spec.p_range
    p = np.exp(rng.uniform(np.log(lo), np.log(hi), size=B))
    fg = FlatGraph(
        be_pdag_idx=np.arange(B, dtype=np.int32) + 2,
        be_event_idx=np.arange(B, dtype=np.uint32),
        be_threshold=probability_threshold(p),
        gate_op=kinds.astype(np.uint8),
        gate_k=kvals.astype(np.uint32),
        gate_in_begin=np.array(in_begin, dtype=np.uint32),
        gate_in_count=np.array(in_count, dtype=np.uint32),
        gate_neg_count=np.zeros(G, dtype=np.uint32),
        inputs=np.array(inputs, dtype=np.uint32),
        tally_nodes=np.arange(B, B + G, dtype=np.uint32),
        gate_pdag_idx=np.arange(G, dtype=np.int32) + 2 + B,
        be_prob=p,
        root=B + G - 1,
        name=spec.name,
        meta={"seed": spec.seed, "n_layers": L, "fanin_widened": widened},
    )
    fg.validate()
    return fg


# --- benchmark configurations ------------------------------------------------

def config1(seed: int = 372) -> FlatGraph:
    """200 basic events, 100 gates (50/50 AND/OR), fan-in 2-4, 20% of events
    shared by >= 2 gates, p log-uniform in [1e-3, 1e-1]."""
    return generate(TreeSpec(n_be=200, n_gates=100, mix={AND: 0.5, OR: 0.5}, p_range=(1e-3, 1e-1), seed=seed,
                             n_layers=7, share_be_frac=0.2, name="config1-200be-100g"))


def config2(seed: int = 11) -> FlatGraph:
    """5,000 basic events, 3,000 gates (45% AND, 40% OR, 10% ATLEAST k-of-n with
    n in 3-8, k in [2, n-1], 5% NOT/XOR), 20 layers, 30% of nodes with fan-out
    >= 2, p log-uniform in [1e-5, 1e-2]."""
    return generate(TreeSpec(n_be=5000, n_gates=3000, mix={AND: 0.45, OR: 0.40, ATLEAST: 0.10, NOT: 0.025, XOR: 0.025},
                             p_range=(1e-5, 1e-2), seed=seed, n_layers=20, share_node_frac=0.30,
                             name="config2-5000be-3000g"))


def config4(seed: int = 49) -> FlatGraph:
    """Rare-event tree: 2,000 basic events, 1,200 gates (60% AND, 30% OR, 10%
    ATLEAST 2-of-3 .. 3-of-5), p log-uniform in [1e-6, 1e-3], 12 layers, no
    shared events (a read-once tree, so the exact BDD stays small).  Seed 49
    was picked from a scan of seeds 0-149 x 12-16 layers as the one whose exact
    top-event probability (at the quantised thresholds) is closest to 1e-8:
    9.3787e-09."""
    return generate(TreeSpec(n_be=2000, n_gates=1200, mix={AND: 0.6, OR: 0.3, ATLEAST: 0.1}, p_range=(1e-6, 1e-3),
                             seed=seed, n_layers=12, atleast_n=(3, 5), share_be_frac=0.0,
                             name="config4-2000be-1200g"))


def small_tree(seed: int, n_be: int = 24, n_gates: int = 12, mix=None, p_range=(0.05, 0.5), n_layers=4,
               share_node_frac: float = 0.2, atleast_n=(3, 5)) -> FlatGraph:
    """A small random DAG with every connective the generator knows, for tests."""
    mix = mix or {AND: 0.3, OR: 0.3, ATLEAST: 0.2, XOR: 0.1, NOT: 0.1}
    return generate(TreeSpec(n_be=n_be, n_gates=n_gates, mix=mix, p_range=p_range, seed=seed, n_layers=n_layers,
                             share_node_frac=share_node_frac, atleast_n=atleast_n, name=f"small-{seed}"))


def config3(n_trees: int = 512, seed: int = 3) -> list:
    """Batched uncertainty-analysis trees: gate count log-uniform in [20, 5,000],
    basic events ~1.6x the gates, otherwise the config-1 generator (50/50
    AND/OR, fan-in 2-4, 20% of events shared, base probabilities log-uniform
    in [1e-3, 1e-1])."""
    rng = np.random.default_rng(seed)
    trees = []
    for t in range(n_trees):
        g = int(round(np.exp(rng.uniform(np.log(20), np.log(5000)))))
        b = int(round(1.6 * g))
        trees.append(generate(TreeSpec(n_be=b, n_gates=g, mix={AND: 0.5, OR: 0.5}, p_range=(1e-3, 1e-1),
                                       seed=int(rng.integers(1 << 31)), share_be_frac=0.2,
                                       name=f"config3-tree{t}-{b}be-{g}g")))
    return trees


def read_once_probability(g: FlatGraph, p: Optional[np.ndarray] = None) -> np.ndarray:
    """Exact probability of every node of a read-once tree (no node with more
    than one parent): AND = prod p, OR = 1 - prod (1 - p) (as -expm1(sum
    log1p(-p)), which keeps its relative precision for tiny p), XOR as a
    fold, NOT, ATLEAST k-of-n by the usual count recursion.  Gates of one
    depth are evaluated together.  Used to calibrate generated rare-event
    instances; raises for graphs with shared nodes."""
    from .graph import NAND, NOR, NULL
    fanout = np.bincount(g.inputs, minlength=g.n_nodes)
    if np.any(fanout > 1):
        raise ValueError("read_once_probability needs a tree (a node has several parents)")
    nb, ng = g.n_be, g.n_gates
    pr = np.zeros(g.n_nodes)
    pr[:nb] = g.quantised_probabilities() if p is None else p
    if ng == 0:
        return pr
    depth = g.layers()[nb:]
    cnt = g.gate_in_count.astype(np.int64)
    pos_neg = cnt - g.gate_neg_count.astype(np.int64)
    ops = g.gate_op.astype(np.int64)
    kk = (g.gate_k.astype(np.int64) & 0xFF)
    for d in range(1, int(depth.max()) + 1):
        gs = np.nonzero(depth == d)[0]
        c = cnt[gs]
        m = int(c.max()) if gs.size else 0
        col = np.arange(m)
        valid = col[None, :] < c[:, None]
        idx = np.where(valid, g.gate_in_begin.astype(np.int64)[gs][:, None] + col[None, :], 0)
        v = pr[g.inputs[idx].astype(np.int64)] if g.inputs.size else np.zeros((gs.size, m))
        v = np.where(col[None, :] >= pos_neg[gs][:, None], 1.0 - v, v)
        v = np.where(valid, v, 0.0)
        op = ops[gs]
        r = np.zeros(gs.size)
        s_and = (op == AND) | (op == NAND)
        r[s_and] = np.prod(np.where(valid[s_and], v[s_and], 1.0), axis=1)
        s_or = (op == OR) | (op == NOR)
        with np.errstate(divide="ignore"):
            r[s_or] = -np.expm1(np.sum(np.log1p(-v[s_or]), axis=1))
        s_x = op == XOR
        if np.any(s_x):
            acc = np.zeros(int(s_x.sum()))
            for j in range(m):
                x = v[s_x, j]
                acc = acc * (1 - x) + (1 - acc) * x
            r[s_x] = acc
        s_k = op == ATLEAST
        if np.any(s_k):
            dist = np.zeros((int(s_k.sum()), m + 1))
            dist[:, 0] = 1.0
            for j in range(m):
                x = v[s_k, j][:, None]
                dist[:, 1:] = dist[:, 1:] * (1 - x) + dist[:, :-1] * x
                dist[:, 0] *= 1 - x[:, 0]
            k = kk[gs][s_k]
            tail = np.cumsum(dist[:, ::-1], axis=1)[:, ::-1]  # tail[:, j] = P(count >= j)
            r[s_k] = np.where(k <= c[s_k], tail[np.arange(k.size), np.minimum(k, m)], 0.0)
        s_l = (op == NOT) | (op == NULL)
        if np.any(s_l):
            last = np.maximum(c[s_l] - 1, 0)
            r[s_l] = np.where(c[s_l] > 0, v[s_l][np.arange(last.size), last] if m else 0.0, 0.0)
        comp = (op == NAND) | (op == NOR) | (op == NOT)
        r[comp] = 1.0 - r[comp]
        pr[nb + gs] = r
    return pr


def calibrate_rare(g: FlatGraph, target: float, p_floor: float = 1e-9, p_cap: float = 0.5) -> FlatGraph:
    """Rescales the basic-event probabilities of a read-once tree as
    p -> clip(p^gamma, p_floor, p_cap), bisecting gamma until the exact top
    probability (at the quantised thresholds) is within 1 % of `target`."""
    base = np.clip(g.quantised_probabilities(), 1e-12, 1.0)

    def top(gamma):
        p = np.clip(base ** gamma, p_floor, p_cap)
        thr = probability_threshold(p)
        return read_once_probability(g, thr.astype(np.float64) / (1 << 32))[g.root], thr

    lo, hi = 0.05, 20.0  # top probability decreases with gamma
    t_lo, _ = top(lo)
    t_hi, _ = top(hi)
    if not (t_hi <= target <= t_lo):
        raise ValueError(f"target {target:g} outside the reachable range [{t_hi:g}, {t_lo:g}]")
    thr = None
    for _ in range(200):
        mid = np.sqrt(lo * hi)
        t, thr = top(mid)
        if t > 0 and abs(np.log(t / target)) < 0.01:
            break
        if t > target:
            lo = mid
        else:
            hi = mid
    out = g.with_thresholds(thr)
    out.be_prob = thr.astype(np.float64) / (1 << 32)
    out.meta = dict(g.meta, target_p_top=target, exact_p_top=float(t))
    return out


def config5_instance(i: int, seed: int = 5) -> FlatGraph:
    """Instance i of the batched rare-event set: basic events log-uniform in
    [50, 10,000] (gates = events / 1.6 for the AND-heavy 60/30/10
    AND/OR/ATLEAST mix of even i, events / 2 for the ATLEAST-heavy 30/30/40
    mix of odd i, whose ATLEAST gates take 3-5 inputs), a read-once tree
    whose base probabilities (log-uniform [1e-6, 1e-3]) are rescaled so that
    the exact top-event probability is a target drawn log-uniformly from
    [1e-10, 1e-5].  Draws come from a generator seeded by (seed, i), so
    every instance can be built on its own; an infeasible draw is redrawn."""
    rng = np.random.default_rng([seed, i])
    and_heavy = i % 2 == 0
    mix = {AND: 0.6, OR: 0.3, ATLEAST: 0.1} if and_heavy else {AND: 0.3, OR: 0.3, ATLEAST: 0.4}
    for _ in range(100):
        nb = int(round(np.exp(rng.uniform(np.log(50), np.log(10000)))))
        ng = max(4, int(round(nb / (1.6 if and_heavy else 2.0))))
        target = float(np.exp(rng.uniform(np.log(1e-10), np.log(1e-5))))
        try:
            g = generate(TreeSpec(n_be=nb, n_gates=ng, mix=mix, p_range=(1e-6, 1e-3),
                                  seed=int(rng.integers(1 << 31)), atleast_n=(3, 5), share_be_frac=0.0,
                                  name=f"config5-{i}-{nb}be"))
            return calibrate_rare(g, target)
        except ValueError:
            continue
    raise RuntimeError(f"no feasible draw for instance {i}")


def calibrate_rare_approx(g: FlatGraph, target: float, p_floor: float = 1e-9, p_cap: float = 0.5) -> FlatGraph:
    """calibrate_rare for graphs with shared events: the same rescaling
    p -> clip(p^gamma, p_floor, p_cap), bisected on the top probability of
    the independence approximation (importance.approximate_importance), which
    is not exact on a DAG; meta records the approximate value, the exact one
    comes from elsewhere (an exact BDD)."""
    from .importance import approximate_importance
    base = np.clip(g.quantised_probabilities(), 1e-12, 1.0)

    def top(gamma):
        p = np.clip(base ** gamma, p_floor, p_cap)
        thr = probability_threshold(p)
        h = g.with_thresholds(thr)
        return float(approximate_importance(h)[0][g.root]), thr

    lo, hi = 0.05, 20.0
    t_lo, _ = top(lo)
    t_hi, _ = top(hi)
    if not (t_hi <= target <= t_lo):
        raise ValueError(f"target {target:g} outside the reachable range [{t_hi:g}, {t_lo:g}]")
    thr, t = None, None
    for _ in range(200):
        mid = np.sqrt(lo * hi)
        t, thr = top(mid)
        if t > 0 and abs(np.log(t / target)) < 0.01:
            break
        if t > target:
            lo = mid
        else:
            hi = mid
    out = g.with_thresholds(thr)
    out.be_prob = thr.astype(np.float64) / (1 << 32)
    out.meta = dict(g.meta, target_p_top=target, approx_p_top=float(t))
    return out


def config4_dag(seed: int = 4) -> FlatGraph:
    """The rare-event tree of config 4 (2,000 basic events, 1,200 gates, 60% AND,
    30% OR, 10% ATLEAST 2-of-3 .. 3-of-5, 12 layers) with 20% of its basic
    events read by two gates, each second parent within the subtree of the
    first parent's parent (so that an exact BDD stays small); probabilities
    log-uniform in [1e-6, 1e-3] rescaled until the independence approximation
    gives P_top = 1e-8."""
    g = generate(TreeSpec(n_be=2000, n_gates=1200, mix={AND: 0.6, OR: 0.3, ATLEAST: 0.1}, p_range=(1e-6, 1e-3),
                          seed=seed, n_layers=12, atleast_n=(3, 5), share_be_frac=0.2, share_scope=1,
                          name="config4-dag-2000be-1200g"))
    return calibrate_rare_approx(g, 1e-8)


def config5_dag_instance(i: int, seed: int = 5) -> FlatGraph:
    """Instance i of the batched rare-event set with shared events: the
    config5_instance draws (events log-uniform in [50, 10,000], AND-heavy
    60/30/10 or ATLEAST-heavy 30/30/40 mix, target P_top log-uniform in
    [1e-10, 1e-5]) with 20% of the basic events read by two gates, the second
    parent within the subtree of the first parent's parent, calibrated with
    the independence approximation (calibrate_rare_approx)."""
    rng = np.random.default_rng([seed, i, 1])
    and_heavy = i % 2 == 0
    mix = {AND: 0.6, OR: 0.3, ATLEAST: 0.1} if and_heavy else {AND: 0.3, OR: 0.3, ATLEAST: 0.4}
    for _ in range(100):
        nb = int(round(np.exp(rng.uniform(np.log(50), np.log(10000)))))
        ng = max(4, int(round(nb / (1.6 if and_heavy else 2.0))))
        target = float(np.exp(rng.uniform(np.log(1e-10), np.log(1e-5))))
        try:
            g = generate(TreeSpec(n_be=nb, n_gates=ng, mix=mix, p_range=(1e-6, 1e-3),
                                  seed=int(rng.integers(1 << 31)), atleast_n=(3, 5), share_be_frac=0.2,
                                  share_scope=1, name=f"config5-dag-{i}-{nb}be"))
            return calibrate_rare_approx(g, target)
        except ValueError:
            continue
    raise RuntimeError(f"no feasible draw for instance {i}")


def config5(n_instances: int = 1024, seed: int = 5, workers: int = 0, first: int = 0) -> list:
    """Instances first .. first + n_instances - 1 of the batched rare-event set
    (config5_instance).  workers > 1 builds them in that many spawned
    processes."""
    return config5_instances(range(first, first + n_instances), seed, workers)


def config5_instances(ids, seed: int = 5, workers=0, shared: bool = False) -> list:
    """The batched rare-event instances with the given indices, in order
    (shared: the config5_dag_instance set); `workers` > 1 spawned processes,
    or an executor to run them on."""
    ids = list(ids)
    make = config5_dag_instance if shared else config5_instance
    if hasattr(workers, "map"):
        n = getattr(workers, "_max_workers", 1) or 1
        return list(workers.map(make, ids, [seed] * len(ids), chunksize=max(1, len(ids) // (4 * n))))
    if workers and workers > 1 and len(ids) > 1:
        import multiprocessing as mp
        from concurrent.futures import ProcessPoolExecutor
        with ProcessPoolExecutor(max_workers=workers, mp_context=mp.get_context("spawn")) as ex:
            return list(ex.map(make, ids, [seed] * len(ids), chunksize=max(1, len(ids) // (4 * workers))))
    return [make(i, seed) for i in ids]


_MEF_CONNECTIVE = {AND: "and", OR: "or", ATLEAST: "atleast", XOR: "xor", NOT: "not", 5: "nand", 6: "nor"}


def event_tree_xml(g: FlatGraph, n_functional: int = 8, initiating_event: str = "IE") -> str:
    """A MEF model of an event tree over a synthetic fault tree: the gates of
    `g` as the fault tree "Plant" (basic events e<i> at their quantised
    probabilities, so the thresholds are the graph's own), the last
    `n_functional` gates in topological order as the functional events' fault
    trees, and a complete binary event tree over them -- every path collects
    each functional event's top (failure) or its negation (success), so the
    2^n sequences partition the outcomes."""
    q = g.quantised_probabilities()
    n_be = g.n_be

    def ref(node: int, neg: bool = False) -> str:
        r = f'<basic-event name="e{node}"/>' if node < n_be else f'<gate name="g{node - n_be}"/>'
        return f"<not>{r}</not>" if neg else r

    out = ['<?xml version="1.0"?>', "<opsa-mef>",
           f'<define-initiating-event name="{initiating_event}" event-tree="Plant-ET"/>',
           '<define-event-tree name="Plant-ET">']
    tops = list(range(g.n_gates - n_functional, g.n_gates))
    out += [f'<define-functional-event name="F{k}"/>' for k in range(n_functional)]
    out += [f'<define-sequence name="S{s:0{n_functional}b}"/>' for s in range(1 << n_functional)]

    def fork(level: int, bits: int) -> str:
        if level == n_functional:
            return f'<sequence name="S{bits:0{n_functional}b}"/>'
        top = f'<gate name="g{tops[level]}"/>'
        return (f'<fork functional-event="F{level}">'
                f'<path state="success"><collect-formula><not>{top}</not></collect-formula>{fork(level + 1, bits << 1)}</path>'
                f'<path state="failure"><collect-formula>{top}</collect-formula>{fork(level + 1, (bits << 1) | 1)}</path>'
                "</fork>")

    out += ["<initial-state>", fork(0, 0), "</initial-state>", "</define-event-tree>",
            '<define-fault-tree name="Plant">']
    for j in range(g.n_gates):
        b, c, neg = int(g.gate_in_begin[j]), int(g.gate_in_count[j]), int(g.gate_neg_count[j])
        args = "".join(ref(int(x), i >= c - neg) for i, x in enumerate(g.inputs[b:b + c]))
        op = int(g.gate_op[j])
        if op == 7:  # NULL: a gate defined as its one argument
            body = args
        else:
            name = _MEF_CONNECTIVE[op]
            attr = f' min="{int(g.gate_k[j])}"' if op == ATLEAST else ""
            body = f"<{name}{attr}>{args}</{name}>"
        out.append(f'<define-gate name="g{j}">{body}</define-gate>')
    out += ["</define-fault-tree>", "<model-data>"]
    out += [f'<define-basic-event name="e{i}"><float value="{float(q[i])!r}"/></define-basic-event>'
            for i in range(n_be)]
    out += ["</model-data>", "</opsa-mef>"]
    return "\n".join(out)
