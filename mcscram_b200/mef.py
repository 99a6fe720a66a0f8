"""Open-PSA MEF fault trees -> the engine's PDAG.

Reads the subset of the Model Exchange Format that fault-tree models such as
the Aralia set use: ``define-fault-tree`` / ``model-data`` holding
``define-gate`` (formulas ``and``, ``or``, ``not``, ``xor``, ``nand``,
``nor``, ``atleast min=k``, or a single event reference, nested formulas
allowed), ``define-basic-event`` and ``define-parameter`` with an
expression, ``define-house-event`` (``constant value="true|false"``).
Expressions: ``float``, ``int``, ``parameter``, ``system-mission-time``,
``exponential`` (1 - exp(-lambda t)), ``GLM`` and ``Weibull`` (the
formulas of mcSCRAM src/expression/exponential.cc:37-38, 87-91, 108-111),
``add``, ``sub``, ``mul``, ``div``, ``neg``.  Event references are ``gate``,
``basic-event``, ``house-event`` or the untyped ``event``.  Other
expressions (random deviates, CCF groups, substitutions) are rejected with
an error naming the element.  Probabilities are taken at a mission time
(8760 hours unless given); ``probability_over_time`` evaluates the top
event on a grid of mission times in one batched GPU pass.

Node numbering follows the reference's PDAG construction from a MEF gate
(mcSCRAM src/pdag.cc:470-548): basic events get indices 2, 3, ... in the
order a depth-first walk of the top formula first meets them
(``GatherVariables``), then gates get the next indices in pre-order as they
are built (``ConstructGate``).  ``not`` of a single event inside a formula
becomes a complemented argument; other nested formulas become gates of their
own.  House events become variables with probability 0 or 1 (constant
words).  SCRAM's preprocessing passes are not applied, so event indices can
differ from the reference's for models the preprocessor rewrites.
"""
from __future__ import annotations

import math
import xml.etree.ElementTree as ET
from dataclasses import dataclass, field
from pathlib import Path
from typing import Dict, List, Optional, Tuple, Union

import numpy as np

from .graph import AND, ATLEAST, NAND, NOR, NOT, NULL, OR, XOR, FlatGraph

_CONNECTIVES = {"and": AND, "or": OR, "atleast": ATLEAST, "xor": XOR, "not": NOT, "nand": NAND, "nor": NOR}
_REFS = ("gate", "basic-event", "house-event", "event")
_SKIP = ("label", "attributes")


class MefError(ValueError):
    """A model the loader cannot read; the message names the element."""


DEFAULT_MISSION_TIME = 8760.0  # hours: SCRAM's default analysis setting


@dataclass
class Expr:
    """An expression tree: op "value" (args: [float]), "parameter" (args:
    [name]), "time", or a function of its argument expressions."""
    op: str
    args: list

    def value(self, t: float, params: Dict[str, "Expr"], _depth: int = 0) -> float:
        if _depth > 64:
            raise MefError("parameters refer to each other in a cycle")
        op, a = self.op, self.args
        if op == "value":
            return a[0]
        if op == "time":
            return t
        if op == "parameter":
            if a[0] not in params:
                raise MefError(f"unknown parameter {a[0]!r}")
            return params[a[0]].value(t, params, _depth + 1)
        v = [x.value(t, params, _depth + 1) for x in a]
        if op == "exponential":  # 1 - exp(-lambda t)
            return 1.0 - math.exp(-v[0] * v[1])
        if op == "GLM":  # gamma, lambda, mu, t
            g, lam, mu, tt = v
            r = lam + mu
            return (lam - (lam - g * r) * math.exp(-r * tt)) / r
        if op == "Weibull":  # alpha, beta, t0, t
            al, be, t0, tt = v
            return 0.0 if tt <= t0 else 1.0 - math.exp(-(((tt - t0) / al) ** be))
        if op == "add":
            return sum(v)
        if op == "mul":
            return math.prod(v)
        if op == "sub":
            return v[0] - sum(v[1:])
        if op == "div":
            out = v[0]
            for x in v[1:]:
                out /= x
            return out
        if op == "neg":
            return -v[0]
        raise MefError(f"unknown expression {op!r}")

    def depends_on_time(self, params: Dict[str, "Expr"], _depth: int = 0) -> bool:
        if _depth > 64:
            return False
        if self.op == "time":
            return True
        if self.op == "parameter":
            return self.args[0] in params and params[self.args[0]].depends_on_time(params, _depth + 1)
        return self.op not in ("value",) and any(x.depends_on_time(params, _depth + 1) for x in self.args)


@dataclass
class Formula:
    """A connective over arguments; an argument is (complement, kind, payload)
    with kind "gate" / "basic-event" / "house-event" (payload: name) or
    "formula" (payload: a nested Formula)."""
    connective: int
    args: List[Tuple[bool, str, object]]
    min_number: int = 0


@dataclass
class MefModel:
    gates: Dict[str, Formula] = field(default_factory=dict)
    basic_events: Dict[str, Expr] = field(default_factory=dict)
    house_events: Dict[str, bool] = field(default_factory=dict)
    parameters: Dict[str, Expr] = field(default_factory=dict)
    names: List[str] = field(default_factory=list)  # fault-tree names
    mission_time: float = DEFAULT_MISSION_TIME

    def probability(self, event: str, t: Optional[float] = None) -> float:
        """Probability of a basic event at mission time t (default: the model's)."""
        v = self.basic_events[event].value(self.mission_time if t is None else t, self.parameters)
        if not 0.0 <= v <= 1.0:
            raise MefError(f"basic event {event!r}: probability {v} outside [0, 1] at t = {t}")
        return v

    def top_gates(self) -> List[str]:
        """Gates that no other gate references, in definition order."""
        used = set()

        def walk(f: Formula):
            for _, kind, x in f.args:
                if kind == "gate":
                    used.add(x)
                elif kind == "formula":
                    walk(x)

        for f in self.gates.values():
            walk(f)
        return [g for g in self.gates if g not in used]

    def build(self, top: Optional[str] = None):
        """Host PDAG rooted at `top` (the only top gate when None).  Returns
        (host.Pdag, root index, {basic-event name: index}, {gate name: index})."""
        from .host import Pdag

        if top is None:
            tops = self.top_gates()
            if len(tops) != 1:
                raise MefError(f"model has {len(tops)} top gates {tops[:5]}; name one")
            top = tops[0]
        if top not in self.gates:
            raise MefError(f"unknown top gate {top!r}")
        # 1. variables in first-encounter order of a depth-first walk (GatherVariables)
        var_index: Dict[str, int] = {}
        house_index: Dict[str, int] = {}
        seen_gates = set()

        def gather(f: Formula):
            for _, kind, x in f.args:
                if kind == "basic-event":
                    if x not in var_index:
                        var_index[x] = 2 + len(var_index)
                elif kind == "gate":
                    if x not in seen_gates:
                        seen_gates.add(x)
                        gather(self.gates[x])
                elif kind == "formula":
                    gather(x)

        seen_gates.add(top)
        gather(self.gates[top])
        nxt = 2 + len(var_index)
        for f_name in self._house_events_in(top):
            house_index[f_name] = nxt
            nxt += 1
        # 2. gates in pre-order of construction (ConstructGate)
        pdag = Pdag()
        for name, idx in var_index.items():
            pdag.add_variable(idx, self.probability(name))
        for name, idx in house_index.items():
            pdag.add_variable(idx, 1.0 if self.house_events[name] else 0.0)
        gate_index: Dict[str, int] = {}
        pending: List[Tuple[int, Formula]] = []
        counter = [nxt]

        def construct(f: Formula) -> int:
            idx = counter[0]
            counter[0] += 1
            args = []
            for comp, kind, x in f.args:
                if kind == "basic-event":
                    a = var_index[x]
                elif kind == "house-event":
                    a = house_index[x]
                elif kind == "gate":
                    if x not in gate_index:
                        gate_index[x] = construct(self.gates[x])
                    a = gate_index[x]
                else:
                    a = construct(x)
                args.append(-a if comp else a)
            pending.append((idx, Formula(f.connective, args, f.min_number)))
            return idx

        root = construct(self.gates[top])
        gate_index[top] = root
        for idx, f in pending:
            pdag.add_gate(idx, f.connective, f.args, f.min_number)
        pdag.set_root(root)
        return pdag, root, var_index, gate_index

    def _house_events_in(self, top: str) -> List[str]:
        out, seen = [], set()

        def walk(f: Formula):
            for _, kind, x in f.args:
                if kind == "house-event" and x not in out:
                    out.append(x)
                elif kind == "gate" and x not in seen:
                    seen.add(x)
                    walk(self.gates[x])
                elif kind == "formula":
                    walk(x)

        seen.add(top)
        walk(self.gates[top])
        return out

    def flat(self, top: Optional[str] = None) -> FlatGraph:
        """The flattened graph of `top` with its root tallied (the engine's input)."""
        pdag, root, _, _ = self.build(top)
        g = pdag.flatten([root])
        g.root = int(g.tally_nodes[0])
        g.name = top or self.top_gates()[0]
        return g


def _local(tag: str) -> str:
    return tag.rsplit("}", 1)[-1]


_ARITY = {"exponential": 2, "GLM": 4, "Weibull": 4, "neg": 1}


def _parse_expr(e: ET.Element, what: str) -> Expr:
    tag = _local(e.tag)
    if tag in ("float", "int"):
        return Expr("value", [float(e.get("value"))])
    if tag == "parameter":
        return Expr("parameter", [e.get("name")])
    if tag == "system-mission-time":
        return Expr("time", [])
    if tag in ("exponential", "GLM", "Weibull", "add", "sub", "mul", "div", "neg"):
        args = [_parse_expr(c, what) for c in e if _local(c.tag) not in _SKIP]
        if tag in _ARITY and len(args) != _ARITY[tag]:
            raise MefError(f"{what}: <{tag}> takes {_ARITY[tag]} arguments, found {len(args)}")
        if not args:
            raise MefError(f"{what}: <{tag}> without arguments")
        return Expr(tag, args)
    raise MefError(f"{what}: unsupported expression <{tag}>")


def _parse_expression(el: ET.Element, what: str) -> Expr:
    kids = [c for c in el if _local(c.tag) not in _SKIP]
    if len(kids) != 1:
        raise MefError(f"{what}: expected one expression, found {len(kids)}")
    return _parse_expr(kids[0], what)


def _parse_formula(el: ET.Element, where: str) -> Formula:
    tag = _local(el.tag)
    if tag in _REFS or tag == "constant":
        # a gate defined as a single event: a pass-through (NULL) gate
        return Formula(NULL, [_parse_arg(el, where)])
    if tag not in _CONNECTIVES:
        raise MefError(f"{where}: unsupported formula <{tag}>")
    args = [_parse_arg(c, where) for c in el if _local(c.tag) not in _SKIP]
    f = Formula(_CONNECTIVES[tag], args)
    if tag == "atleast":
        if el.get("min") is None:
            raise MefError(f"{where}: <atleast> without min")
        f.min_number = int(el.get("min"))
    return f


def _parse_arg(el: ET.Element, where: str) -> Tuple[bool, str, object]:
    tag = _local(el.tag)
    if tag in _REFS:
        name = el.get("name")
        if not name:
            raise MefError(f"{where}: <{tag}> without a name")
        return False, tag, name
    if tag == "constant":
        return False, "constant", el.get("value", "").strip().lower() == "true"
    if tag == "not":
        kids = [c for c in el if _local(c.tag) not in _SKIP]
        if len(kids) == 1 and _local(kids[0].tag) in _REFS:
            comp, kind, x = _parse_arg(kids[0], where)
            return (not comp), kind, x
    return False, "formula", _parse_formula(el, where)


def parse(source: Union[str, Path], mission_time: float = DEFAULT_MISSION_TIME) -> MefModel:
    """Reads a MEF document (a path, or the XML text itself); probabilities are
    evaluated at `mission_time` unless asked for at another time."""
    text = Path(source).read_text() if isinstance(source, Path) or (
        isinstance(source, str) and not source.lstrip().startswith("<")) else source
    try:
        root = ET.fromstring(text.lstrip("﻿"))
    except ET.ParseError as e:
        raise MefError(f"not well-formed XML: {e}") from None
    if _local(root.tag) != "opsa-mef":
        raise MefError("root element is not <opsa-mef>")
    m = MefModel(mission_time=float(mission_time))

    def visit(container: ET.Element):
        for el in container:
            tag = _local(el.tag)
            name = el.get("name")
            if tag in ("define-fault-tree", "define-component"):
                if tag == "define-fault-tree":
                    m.names.append(name)
                visit(el)
            elif tag == "model-data":
                visit(el)
            elif tag == "define-gate":
                kids = [c for c in el if _local(c.tag) not in _SKIP]
                if len(kids) != 1:
                    raise MefError(f"gate {name!r}: expected one formula, found {len(kids)}")
                if name in m.gates:
                    raise MefError(f"gate {name!r} defined twice")
                m.gates[name] = _parse_formula(kids[0], f"gate {name!r}")
            elif tag == "define-basic-event":
                m.basic_events[name] = _parse_expression(el, f"basic event {name!r}")
            elif tag == "define-house-event":
                kids = [c for c in el if _local(c.tag) not in _SKIP]
                m.house_events[name] = bool(kids) and kids[0].get("value", "").strip().lower() == "true"
            elif tag == "define-parameter":
                m.parameters[name] = _parse_expression(el, f"parameter {name!r}")
            elif tag in _SKIP:
                continue
            else:
                raise MefError(f"unsupported element <{tag}>")

    visit(root)
    for name in m.basic_events:
        try:
            m.probability(name)
        except MefError as e:
            raise MefError(f"basic event {name!r}: {e}") from None
    # resolve untyped references and constants; check every reference
    consts = {}

    def resolve(f: Formula, where: str):
        out = []
        for comp, kind, x in f.args:
            if kind == "event":
                kind = ("gate" if x in m.gates else "basic-event" if x in m.basic_events
                        else "house-event" if x in m.house_events else None)
                if kind is None:
                    raise MefError(f"{where}: unknown event {x!r}")
            if kind == "constant":
                key = f"__constant_{'true' if x else 'false'}"
                m.house_events.setdefault(key, bool(x))
                kind, x = "house-event", key
                consts[key] = True
            table = {"gate": m.gates, "basic-event": m.basic_events, "house-event": m.house_events}.get(kind)
            if table is not None and x not in table:
                raise MefError(f"{where}: unknown {kind} {x!r}")
            if kind == "formula":
                resolve(x, where)
            out.append((comp, kind, x))
        f.args = out

    for name, f in m.gates.items():
        resolve(f, f"gate {name!r}")
    return m


def load(source: Union[str, Path], top: Optional[str] = None,
         mission_time: float = DEFAULT_MISSION_TIME) -> FlatGraph:
    """MEF document -> flattened graph of its top gate (probabilities at the
    mission time), root tallied."""
    return parse(source, mission_time).flat(top)


def probability_over_time(model: MefModel, time_step: float, top: Optional[str] = None,
                          mission_time: Optional[float] = None, words: int = 1 << 16, iteration: int = 1,
                          device: int = 0):
    """P(top) at t = 0, dt, 2 dt, ... and at the mission time (when it is not a
    multiple of dt), as (probability, time) pairs -- the pairs the reference's
    CalculateProbabilityOverTime returns (mcSCRAM src/mc/core/
    probability_analysis.cc:280-311, left unimplemented there).  Every time
    point is one instance of one batched launch over the same tree, with its
    own thresholds and the same random numbers (the same counters), so for a
    tree without negations the estimates never decrease in t."""
    from .graph import probability_threshold
    from .uncertainty import Batch

    T = model.mission_time if mission_time is None else float(mission_time)
    if time_step <= 0:
        return []
    times = []
    k = 0
    while k * time_step < T:
        times.append(k * time_step)
        k += 1
    times.append(T)
    pdag, root, var_index, _ = model.build(top)
    g = pdag.flatten([root])
    g.root = int(g.tally_nodes[0])
    name_of = {idx: name for name, idx in var_index.items()}
    thresholds = []
    for t in times:
        p = np.array([model.probability(name_of[int(x)], t) if int(x) in name_of else
                      g.quantised_probabilities()[i] for i, x in enumerate(g.be_pdag_idx)])
        thresholds.append(probability_threshold(p))
    with Batch([g], device=device) as b:
        ones = b.run([0] * len(times), thresholds, iteration=iteration, words_per_instance=words)
    n = float(words) * 64.0
    return [(float(o) / n, t) for o, t in zip(ones, times)]


def main(argv=None) -> int:
    """python -m mcscram_b200.mef MODEL.xml [--top GATE] [--samples N] [--mode strip|staged|fused]:
    estimates the top-event probability of a MEF model on the GPU and prints
    it with its 95 % interval as one JSON line."""
    import argparse
    import json
    import math

    from . import _capi

    ap = argparse.ArgumentParser(description=main.__doc__)
    ap.add_argument("model")
    ap.add_argument("--top", default=None)
    ap.add_argument("--samples", type=float, default=2 ** 30)
    ap.add_argument("--mode", default="strip", choices=list(_capi.MODES))
    ap.add_argument("--device", type=int, default=0)
    args = ap.parse_args(argv)
    g = load(args.model, args.top)
    words = max(1, int(math.ceil(args.samples / 64)))
    with _capi.Engine(g, mode=_capi.MODES[args.mode], device=args.device) as e:
        done, it = 0, 1
        while done < words:  # passes of at most 2^24 words (the 32-bit sample counter per pass)
            n = min(words - done, 1 << 24)
            e.run(it, 1, 0, n)
            done += n
            it += 1
        ones, total = e.tallies()
    p = int(ones[0]) / total
    half = 1.959963984540054 * math.sqrt(max(p * (1 - p), 0.0) / total)
    out = {"model": args.model, "top": g.name, "basic_events": g.n_be, "gates": g.n_gates, "samples": int(total),
           "p_top": p, "ci95": [max(p - half, 0.0), min(p + half, 1.0)]}
    print(json.dumps(out))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
