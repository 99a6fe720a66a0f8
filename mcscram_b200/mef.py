"""Open-PSA MEF fault trees -> the engine's PDAG.

Reads the subset of the Model Exchange Format that fault-tree models such as
the Aralia set use: ``define-fault-tree`` / ``model-data`` holding
``define-gate`` (formulas ``and``, ``or``, ``not``, ``xor``, ``nand``,
``nor``, ``atleast min=k``, or a single event reference, nested formulas
allowed), ``define-basic-event`` (a ``float`` value or a ``parameter``
reference), ``define-house-event`` (``constant value="true|false"``) and
``define-parameter`` (a ``float`` value).  Event references are ``gate``,
``basic-event``, ``house-event`` or the untyped ``event``.  Other
expressions (time-dependent distributions, CCF groups, substitutions) are
rejected with an error naming the element.

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

import xml.etree.ElementTree as ET
from dataclasses import dataclass, field
from pathlib import Path
from typing import Dict, List, Optional, Tuple, Union

from .graph import AND, ATLEAST, NAND, NOR, NOT, NULL, OR, XOR, FlatGraph

_CONNECTIVES = {"and": AND, "or": OR, "atleast": ATLEAST, "xor": XOR, "not": NOT, "nand": NAND, "nor": NOR}
_REFS = ("gate", "basic-event", "house-event", "event")
_SKIP = ("label", "attributes")


class MefError(ValueError):
    """A model the loader cannot read; the message names the element."""


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
    basic_events: Dict[str, float] = field(default_factory=dict)
    house_events: Dict[str, bool] = field(default_factory=dict)
    parameters: Dict[str, float] = field(default_factory=dict)
    names: List[str] = field(default_factory=list)  # fault-tree names

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
            pdag.add_variable(idx, self.basic_events[name])
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


def _parse_expression(el: ET.Element, what: str) -> Tuple[str, Union[float, str]]:
    kids = [c for c in el if _local(c.tag) not in _SKIP]
    if len(kids) != 1:
        raise MefError(f"{what}: expected one expression, found {len(kids)}")
    e = kids[0]
    tag = _local(e.tag)
    if tag == "float" or tag == "int":
        return "value", float(e.get("value"))
    if tag == "parameter":
        return "parameter", e.get("name")
    raise MefError(f"{what}: unsupported expression <{tag}>")


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


def parse(source: Union[str, Path]) -> MefModel:
    """Reads a MEF document (a path, or the XML text itself)."""
    text = Path(source).read_text() if isinstance(source, Path) or (
        isinstance(source, str) and not source.lstrip().startswith("<")) else source
    try:
        root = ET.fromstring(text.lstrip("﻿"))
    except ET.ParseError as e:
        raise MefError(f"not well-formed XML: {e}") from None
    if _local(root.tag) != "opsa-mef":
        raise MefError("root element is not <opsa-mef>")
    m = MefModel()
    basic_expr: Dict[str, Tuple[str, object]] = {}

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
                basic_expr[name] = _parse_expression(el, f"basic event {name!r}")
            elif tag == "define-house-event":
                kids = [c for c in el if _local(c.tag) not in _SKIP]
                m.house_events[name] = bool(kids) and kids[0].get("value", "").strip().lower() == "true"
            elif tag == "define-parameter":
                kind, v = _parse_expression(el, f"parameter {name!r}")
                if kind != "value":
                    raise MefError(f"parameter {name!r}: only float values are read")
                m.parameters[name] = float(v)
            elif tag in _SKIP:
                continue
            else:
                raise MefError(f"unsupported element <{tag}>")

    visit(root)
    for name, (kind, v) in basic_expr.items():
        if kind == "parameter":
            if v not in m.parameters:
                raise MefError(f"basic event {name!r}: unknown parameter {v!r}")
            v = m.parameters[v]
        if not 0.0 <= float(v) <= 1.0:
            raise MefError(f"basic event {name!r}: probability {v} outside [0, 1]")
        m.basic_events[name] = float(v)
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


def load(source: Union[str, Path], top: Optional[str] = None) -> FlatGraph:
    """MEF document -> flattened graph of its top gate, root tallied."""
    return parse(source).flat(top)


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
