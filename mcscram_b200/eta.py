"""Event-tree analysis on the combined Monte Carlo path.

Restates mcSCRAM's event-tree analysis (src/event_tree_analysis.cc:101-239)
and its combined Monte Carlo pass (src/risk_analysis.cc:273-437,
``RunCombinedEtaAnalysis``): the paths of an initiating event's event tree
are walked, every sequence becomes one gate (the OR over its paths of the AND
of the formulas collected on each path, or, for trees that collect
expressions, a basic event whose probability is the sum over paths of the
product of the collected expressions), one synthetic OR root joins the
sequence gates, and a single PDAG is sampled with every sequence gate tallied
-- one run to convergence yields every sequence's probability.  Fault-tree
top events that appear in that PDAG are tallied in the same run (the
reference's watched gates, src/risk_analysis.cc:377-420).

Deviations: sequences are kept in the order the walk first reaches them (the
reference keys them by pointer in an unordered map, src/event_tree_analysis.h:90-94,
so its order is not defined); a gate cloned under a set of house-event
states is built once per distinct set (the reference clones it at every
collection, src/event_tree_analysis.cc:39-81; the clones are identical); an
event tree with a single sequence gets a pass-through (NULL) root, where the
reference's one-argument OR formula would be rejected by its own formula
check (src/event.cc:178-184).
"""
from __future__ import annotations

import copy
import json
import math
from dataclasses import dataclass, field
from pathlib import Path
from typing import Dict, List, Optional, Tuple

from . import _capi
from .graph import AND, NULL, OR, FlatGraph
from .mef import Expr, Formula, MefError, MefModel, parse

TRUE_HOUSE = "__constant_true"


@dataclass
class _Path:
    """What one path collects (PathCollector, src/event_tree_analysis.h:65-73)."""
    expressions: list = field(default_factory=list)
    formulas: list = field(default_factory=list)
    set_house: Dict[str, bool] = field(default_factory=dict)

    def copy(self) -> "_Path":
        return _Path(list(self.expressions), list(self.formulas), dict(self.set_house))


@dataclass
class SequenceResult:
    """One sequence of the analysis (EventTreeAnalysis::Result,
    src/event_tree_analysis.h:38-44): its gate in the analysed model and, once
    sampled, its probability."""
    sequence: str
    gate: str
    is_expression_only: bool
    p_sequence: float = math.nan


class EventTreeAnalysis:
    """Collects the sequences of one initiating event's event tree and turns
    them into gates of a working copy of the model (``self.model``)."""

    def __init__(self, model: MefModel, initiating_event: str):
        if initiating_event not in model.initiating_events:
            raise MefError(f"unknown initiating event {initiating_event!r}")
        tree = model.initiating_events[initiating_event]
        if tree is None:
            raise MefError(f"initiating event {initiating_event!r} has no event tree")
        self.initiating_event = initiating_event
        self.event_tree = model.event_trees[tree]
        m = copy.copy(model)
        m.gates = dict(model.gates)
        m.basic_events = dict(model.basic_events)
        m.house_events = dict(model.house_events)
        self.model = m
        self.sequences: List[SequenceResult] = []
        self._clones: Dict[tuple, str] = {}

    # -- cloning under set-house-event (src/event_tree_analysis.cc:39-81) --
    def _clone(self, f: Formula, set_house: Dict[str, bool]) -> Formula:
        m = self.model
        args = []
        for comp, kind, x in f.args:
            if kind == "house-event" and x in set_house and set_house[x] != m.house_events[x]:
                key = f"__clone__.{x}={'true' if set_house[x] else 'false'}"
                m.house_events.setdefault(key, set_house[x])
                x = key
            elif kind == "gate" and set_house:
                key = (x, tuple(sorted(set_house.items())))
                if key not in self._clones:
                    name = f"__clone__{len(self._clones)}.{x}"
                    self._clones[key] = name
                    m.gates[name] = self._clone(m.gates[x], set_house)
                x = self._clones[key]
            elif kind == "formula":
                x = self._clone(x, set_house)
            args.append((comp, kind, x))
        return Formula(f.connective, args, f.min_number)

    # -- the walk (src/event_tree_analysis.cc:164-236) --
    def _collect(self) -> Dict[str, List[_Path]]:
        m = self.model
        out: Dict[str, List[_Path]] = {}
        ctx = {"initiating_event": self.initiating_event, "functional_events": {}}

        def instruction(ins, pc: _Path, state: dict, tree):
            kind = ins[0]
            if kind == "set-house-event":
                pc.set_house[ins[1]] = ins[2]
            elif kind == "collect-formula":
                pc.formulas.append(self._clone(ins[1], pc.set_house))
            elif kind == "collect-expression":
                pc.expressions.append(ins[1])
            elif kind == "if":
                if ins[1].value(m.mission_time, m.parameters, ctx):
                    instruction(ins[2], pc, state, tree)
                elif ins[3] is not None:
                    instruction(ins[3], pc, state, tree)
            elif kind == "block":
                for x in ins[1]:
                    instruction(x, pc, state, tree)
            elif kind == "rule":
                for x in m.rules[ins[1]]:
                    instruction(x, pc, state, tree)
            elif kind == "link":
                state["linked"] = True
                linked = m.event_trees[ins[1]]
                saved = ctx["functional_events"]
                ctx["functional_events"] = {}
                branch(linked.initial_state, pc.copy(), linked)
                ctx["functional_events"] = saved

        def branch(b, pc: _Path, tree):
            state = {"linked": False}
            for ins in b.instructions:
                instruction(ins, pc, state, tree)
            kind, x = b.target
            if kind == "sequence":
                seq_state = {"linked": False}
                for ins in m.sequences[x]:
                    instruction(ins, pc, seq_state, tree)
                if not seq_state["linked"]:
                    out.setdefault(x, []).append(pc)
            elif kind == "fork":
                fes = ctx["functional_events"]
                for st, path in x.paths:
                    fes[x.functional_event] = st
                    branch(path, pc.copy(), tree)
                fes.pop(x.functional_event, None)
            else:
                branch(tree.branches[x], pc, tree)

        branch(self.event_tree.initial_state, _Path(), self.event_tree)
        return out

    def analyze(self) -> List[SequenceResult]:
        """Sequence gates (src/event_tree_analysis.cc:101-162)."""
        m = self.model
        formula_id = [0]

        def make_gate(f: Formula) -> str:
            name = f"___{self.initiating_event}__formula_{formula_id[0]}__"
            formula_id[0] += 1
            m.gates[name] = f
            return name

        self.sequences = []
        for seq, paths in self._collect().items():
            gate_formulas, arg_exprs = [], []
            for pc in paths:
                if len(pc.formulas) == 1:
                    gate_formulas.append(pc.formulas[0])
                elif len(pc.formulas) > 1:
                    gate_formulas.append(Formula(AND, [(False, "gate", make_gate(f)) for f in pc.formulas]))
                if len(pc.expressions) == 1:
                    arg_exprs.append(pc.expressions[0])
                elif len(pc.expressions) > 1:
                    arg_exprs.append(Expr("mul", list(pc.expressions)))
            gate = f"__{seq}"
            if len(gate_formulas) == 1:
                f = gate_formulas[0]
            elif gate_formulas:
                f = Formula(OR, [(False, "gate", make_gate(x)) for x in gate_formulas])
            elif arg_exprs:
                m.basic_events[gate] = arg_exprs[0] if len(arg_exprs) == 1 else Expr("add", arg_exprs)
                m.probability(gate)  # a sum of path products outside [0, 1] is an error
                f = Formula(NULL, [(False, "basic-event", gate)])
            else:
                m.house_events.setdefault(TRUE_HOUSE, True)
                f = Formula(NULL, [(False, "house-event", TRUE_HOUSE)])
            m.gates[gate] = f
            self.sequences.append(SequenceResult(seq, gate, bool(arg_exprs) and not gate_formulas))
        return self.sequences


@dataclass
class CombinedPdag:
    """The PDAG of one initiating event: the synthetic OR root over its
    sequence gates; `sequences` pairs each result with its node index,
    `watched` the fault-tree tops found in the PDAG with theirs."""
    initiating_event: str
    pdag: object
    root: int
    sequences: List[Tuple[SequenceResult, int]]
    watched: List[Tuple[str, int]]
    model: MefModel

    def tally_indices(self) -> List[int]:
        """Node indices of the sequence gates, then of the watched gates."""
        return [i for _, i in self.sequences] + [i for _, i in self.watched]

    def flat(self) -> FlatGraph:
        """The flattened graph with the root, every sequence gate and every
        watched gate tallied, in that order."""
        g = self.pdag.flatten([self.root] + self.tally_indices())
        g.root = int(g.tally_nodes[0])
        g.name = f"{self.initiating_event} event tree"
        return g


def combined_pdag(model: MefModel, initiating_event: str) -> CombinedPdag:
    """Steps 1-2 of RunCombinedEtaAnalysis (src/risk_analysis.cc:280-306)."""
    eta = EventTreeAnalysis(model, initiating_event)
    seqs = eta.analyze()
    if not seqs:
        raise MefError(f"the event tree of {initiating_event!r} has no sequences")
    m = eta.model
    root_name = f"__ETA_OR_ROOT__{initiating_event}"
    args = [(False, "gate", s.gate) for s in seqs]
    m.gates[root_name] = Formula(OR if len(args) > 1 else NULL, args)
    pdag, root, _, gate_index = m.build(root_name)
    watched = []
    for tree in m.fault_trees:
        for top in m.fault_tree_tops(tree):
            if top in gate_index and all(top != w for w, _ in watched):
                watched.append((top, gate_index[top]))
    return CombinedPdag(initiating_event, pdag, root, [(s, gate_index[s.gate]) for s in seqs], watched, m)


@dataclass
class EventTreeResult:
    """One combined run: the root, every sequence and every watched gate with
    their tallies ({num_one_bits, total_bits, mean, std_err, ...}), and the
    convergence report."""
    initiating_event: str
    phase: Optional[Tuple[str, str]]
    root: dict
    sequences: List[dict]
    gates: List[dict]
    report: dict


def run_combined(model: MefModel, initiating_event: str, settings=None, mode: int = _capi.MODE_STRIP,
                 device: int = 0, phase: Optional[Tuple[str, str]] = None) -> EventTreeResult:
    """RunCombinedEtaAnalysis: one PDAG, every sequence gate observed with
    convergence tracking, one ComputeTallies run on the GPU."""
    from . import host

    c = combined_pdag(model, initiating_event)
    watch = c.tally_indices()
    tallies, rep = host.compute_tallies(c.pdag, settings, watch, device=device, mode=mode)
    by_index = {t["index"]: t for t in tallies}
    seqs = []
    for s, idx in c.sequences:
        t = dict(by_index[idx])
        s.p_sequence = t["mean"]
        seqs.append({"sequence": s.sequence, "gate": s.gate, "is_expression_only": s.is_expression_only, **t})
    gates = [{"gate": g, **by_index[idx]} for g, idx in c.watched]
    return EventTreeResult(initiating_event, phase, tallies[0], seqs, gates, rep)


def analyze(model: MefModel, settings=None, mode: int = _capi.MODE_STRIP, device: int = 0):
    """RiskAnalysis::RunAnalysis on the combined Monte Carlo path
    (src/risk_analysis.cc:51-166): for every alignment phase (or once without
    alignments) and every initiating event with an event tree, one combined
    run; then every fault-tree top event not already tallied in one of them
    gets its own run.  Returns (event-tree results, {gate: tally})."""
    from . import host

    phases: List[Tuple[Optional[Tuple[str, str]], MefModel]] = []
    if model.alignments:
        for name, ps in model.alignments.items():
            for ph in ps:
                phases.append(((name, ph.name), model.with_phase(ph)))
    else:
        phases.append((None, model))
    results, tops = [], {}
    for tag, m in phases:
        seen = set()
        for ie, tree in m.initiating_events.items():
            if tree is None:
                continue
            r = run_combined(m, ie, settings, mode, device, tag)
            results.append(r)
            seen.update(g["gate"] for g in r.gates)
        for tree in m.fault_trees:
            for top in m.fault_tree_tops(tree):
                if top in seen:
                    continue
                pdag, root, _, _ = m.build(top)
                t, rep = host.compute_tallies(pdag, settings, (), device=device, mode=mode)
                tops[(tag, top)] = {**t[0], "report": rep}
    return results, tops


def main(argv=None) -> int:
    """python -m mcscram_b200.eta MODEL.xml [MORE.xml ...] [--rel-err E] [--trials N]
    [--mode strip|staged|fused] [--ccf]: event-tree analysis of a MEF model on the GPU;
    prints one JSON line per sequence (probability and 95 % interval) and per
    fault-tree top event."""
    import argparse

    from . import host

    ap = argparse.ArgumentParser(description=main.__doc__)
    ap.add_argument("model", nargs="+")
    ap.add_argument("--rel-err", type=float, default=0.01)
    ap.add_argument("--trials", type=float, default=0, help="fixed trial budget (no early stop)")
    ap.add_argument("--mission-time", type=float, default=None)
    ap.add_argument("--mode", default="strip", choices=list(_capi.MODES))
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--ccf", action="store_true", help="expand common-cause groups (CCF analysis)")
    ap.add_argument("--allow-extern", action="store_true", help="load the model's extern libraries (runs their code)")
    args = ap.parse_args(argv)
    kw = {} if args.mission_time is None else {"mission_time": args.mission_time}
    m = parse([Path(x) for x in args.model], ccf_analysis=args.ccf, allow_extern=args.allow_extern, **kw)
    s = host.Settings.default(ci_rel_margin_error=args.rel_err)
    if args.trials:
        s = host.Settings.default(num_trials=int(args.trials), early_stop=0, ci_rel_margin_error=1e-9)
    results, tops = analyze(m, s, _capi.MODES[args.mode], args.device)
    z = 1.959963984540054
    for r in results:
        for q in r.sequences:
            half = z * q["std_err"]
            print(json.dumps({"initiating_event": r.initiating_event, "phase": r.phase, "sequence": q["sequence"],
                              "p": q["mean"], "ci95": [max(q["mean"] - half, 0.0), min(q["mean"] + half, 1.0)],
                              "samples": q["total_bits"]}))
    for (tag, top), t in tops.items():
        print(json.dumps({"phase": tag, "gate": top, "p": t["mean"], "samples": t["total_bits"]}))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
