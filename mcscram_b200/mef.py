"""Open-PSA MEF models -> the engine's PDAG.

Reads the subset of the Model Exchange Format that fault-tree models such as
the Aralia set and event-tree models use.

Fault trees: ``define-fault-tree`` / ``define-component`` / ``model-data``
holding ``define-gate`` (formulas ``and``, ``or``, ``not``, ``xor``,
``nand``, ``nor``, ``atleast min=k``, ``cardinality min max``, ``imply``,
``iff``, or a single event reference; the arguments are events, their
negations or constants, as the reference's schema has them),
``define-basic-event`` and ``define-parameter`` with an expression,
``define-house-event`` (``constant value="true|false"``).  Expressions:
``float``, ``int``, ``bool``, ``pi``, ``parameter``,
``system-mission-time``, ``exponential`` (1 - exp(-lambda t)), ``GLM`` and
``Weibull`` (the formulas of mcSCRAM src/expression/exponential.cc:37-38,
87-91, 108-111), ``periodic-test`` (4, 5 and 11 arguments), ``add``,
``sub``, ``mul``, ``div``, ``neg``, the numeric built-ins (``abs``, ``exp``,
``log``, ``log10``, ``sqrt``, ``pow``, ``mod``, ``min``, ``max``, ``mean``,
``ceil``, ``floor`` and the trigonometric and hyperbolic functions), the
boolean ``not``, ``and``, ``or``, ``eq``, ``df``, ``lt``, ``gt``, ``leq``,
``geq``, ``ite``, ``switch``, and the random deviates (``uniform-``,
``normal-``, ``lognormal-``, ``gamma-`` and ``beta-deviate``,
``histogram``), which stand for their means in point values and are drawn
once per trial by ``sample_expressions`` / ``uncertainty``.  Event references are ``gate``, ``basic-event``,
``house-event`` or the untyped ``event``.  ``define-CCF-group`` (beta
factor, MGL, alpha factor and phi factor models) defines its members; with
``ccf_analysis`` they are expanded into common-cause events
(``ccf_level_probabilities``).  ``define-substitution``: declarative
substitutions constrain the analysed top as the reference's PDAG does
(``MefModel.build``); non-declarative ones are checked and kept, and serve
no Monte Carlo graph.  ``define-extern-library`` / ``define-extern-function``
and the ``extern-function`` expression call into a shared library, loaded
only when ``allow_extern`` asks for it.  Other elements and expressions are
rejected with an error naming the element.  Probabilities are taken at a mission
time (8760 hours unless given); ``probability_over_time`` evaluates the top
event on a grid of mission times in one batched GPU pass.

Event trees (read here, analysed by ``mcscram_b200.eta``):
``define-initiating-event``, ``define-event-tree`` (functional events,
sequences, named branches, the initial state with ``fork`` / ``path``
targets), ``define-rule`` and ``define-alignment`` / ``define-phase``; the
instructions ``collect-formula``, ``collect-expression``,
``set-house-event``, ``if`` (with ``test-initiating-event`` and
``test-functional-event`` conditions), ``block``, ``rule`` and the
end-state link ``event-tree``.  The checks of the reference's initializer
are restated (src/initializer.cc:1628-1791): undefined and doubly defined
elements, cycles of gates, rules, branches and links, the order of
functional events along fork paths, links only in sequences, and no
collect-expression mixed with collect-formula on one tree.

Scoping follows the MEF rules of the reference's initializer
(src/initializer.cc:1400-1466, 736-775): an element defined inside a
``define-fault-tree`` / ``define-component`` has the container's path as its
base path and the container's role unless it names its own; a public element
is known by its name, a private one only by its full path
(``Tree.Component.name``); a reference is looked up in the referring
element's own scope first (base path + "." + reference), then among the
public names (a reference without a dot) or the full paths (with a dot).

Node numbering follows the reference's PDAG construction from a MEF gate
(mcSCRAM src/pdag.cc:470-548): basic events get indices 2, 3, ... in the
order a depth-first walk of the top formula first meets them
(``GatherVariables``), then gates get the next indices in pre-order as they
are built (``ConstructGate``).  ``not`` of a single event inside a formula
becomes a complemented argument.  ``imply``, ``iff`` and ``cardinality`` become the gates the
reference's ``ConstructComplexGate`` builds (src/pdag.cc:660-716).  House
events become variables with probability 0 or 1 (constant words).  SCRAM's
preprocessing passes are not applied, so event indices can differ from the
reference's for models the preprocessor rewrites.
"""
from __future__ import annotations

import copy
import math
import xml.etree.ElementTree as ET
from dataclasses import dataclass, field
from pathlib import Path
from typing import Dict, List, Optional, Tuple, Union

import numpy as np

from .graph import AND, ATLEAST, NAND, NOR, NOT, NULL, OR, XOR, FlatGraph

_CONNECTIVES = {"and": AND, "or": OR, "atleast": ATLEAST, "xor": XOR, "not": NOT, "nand": NAND, "nor": NOR}
_COMPLEX = ("imply", "iff", "cardinality")
_REFS = ("gate", "basic-event", "house-event", "event")
_SKIP = ("label", "attributes")
_TABLES = ("gate", "basic-event", "house-event", "parameter")
_EVENTS = ("gate", "basic-event", "house-event")


class MefError(ValueError):
    """A model the loader cannot read; the message names the element."""


DEFAULT_MISSION_TIME = 8760.0  # hours: SCRAM's default analysis setting


@dataclass
class Expr:
    """An expression tree: op "value" (args: [float]), "parameter" (args:
    [id]), "time", "test-initiating-event" (args: [name]),
    "test-functional-event" (args: [name, state]), or a function of its
    argument expressions."""
    op: str
    args: list

    def value(self, t: float, params: Dict[str, "Expr"], context: Optional[dict] = None,
              _depth: int = 0) -> float:
        """Value at mission time t.  `context` ({"initiating_event": name,
        "functional_events": {name: state}}) answers the test events, as the
        reference's mef::Context does during an event-tree walk; without one
        they are false."""
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
            return params[a[0]].value(t, params, context, _depth + 1)
        if op == "test-initiating-event":
            return float(bool(context) and context.get("initiating_event") == a[0])
        if op == "test-functional-event":
            return float(bool(context) and context.get("functional_events", {}).get(a[0]) == a[1])
        if op == "ite":
            branch = a[1] if a[0].value(t, params, context, _depth + 1) else a[2]
            return branch.value(t, params, context, _depth + 1)
        if op == "switch":
            for i in range(0, len(a) - 1, 2):
                if a[i].value(t, params, context, _depth + 1):
                    return a[i + 1].value(t, params, context, _depth + 1)
            return a[-1].value(t, params, context, _depth + 1)
        if op == "extern-function":  # args: the function, then its argument expressions
            if not isinstance(a[0], ExternFunction):
                raise MefError(f"extern function {a[0]!r} is not resolved")
            return a[0](*(x.value(t, params, context, _depth + 1) for x in a[1:]))
        v = [x.value(t, params, context, _depth + 1) for x in a]
        if op in _DEVIATES:  # a random deviate stands for its mean (mcSCRAM src/expression/random_deviate.h)
            return _deviate_mean(op, v)
        if op == "periodic-test":
            return periodic_test(*v)
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
        if op in _UNARY:
            return float(_UNARY[op](v[0]))
        if op == "pow":
            return v[0] ** v[1]
        if op == "mod":  # integer remainder, truncated like C++'s % on ints
            return float(int(math.fmod(int(v[0]), int(v[1]))))
        if op == "min":
            return min(v)
        if op == "max":
            return max(v)
        if op == "mean":
            return sum(v) / len(v)
        if op == "not":
            return float(not v[0])
        if op == "and":
            return float(all(v))
        if op == "or":
            return float(any(v))
        if op in _COMPARE:
            return float(_COMPARE[op](v[0], v[1]))
        raise MefError(f"unknown expression {op!r}")

    def depends_on_time(self, params: Dict[str, "Expr"], _depth: int = 0) -> bool:
        if _depth > 64:
            return False
        if self.op == "time":
            return True
        if self.op == "parameter":
            return self.args[0] in params and params[self.args[0]].depends_on_time(params, _depth + 1)
        if self.op in ("value", "test-initiating-event", "test-functional-event"):
            return False
        return any(x.depends_on_time(params, _depth + 1) for x in _expr_args(self))


def _expr_args(e: Expr) -> list:
    """The argument expressions (an extern function's first arg is the function)."""
    return e.args[1:] if e.op == "extern-function" else e.args


class ExternFunction:
    """A function of an extern library (mcSCRAM src/expression/extern.h:84-198):
    `int` or `double` return and up to 5 `int`/`double` parameters; arguments
    are evaluated as doubles and converted to the parameter types as C++
    converts them (toward zero for int), the result returned as a double."""
    MAX_PARAMS = 5

    def __init__(self, name: str, symbol: str, library, types: List[str]):
        import ctypes
        self.name, self.types = name, types
        try:
            fn = getattr(library, symbol)
        except AttributeError:
            raise MefError(f"extern function {name!r}: symbol {symbol!r} is not in the library") from None
        ct = {"int": ctypes.c_int, "double": ctypes.c_double}
        fn.restype = ct[types[0]]
        fn.argtypes = [ct[x] for x in types[1:]]
        self._fn = fn

    @property
    def arity(self) -> int:
        return len(self.types) - 1

    def __call__(self, *args) -> float:
        conv = [int(x) if ty == "int" else float(x) for x, ty in zip(args, self.types[1:])]
        return float(self._fn(*conv))

    def __repr__(self):
        return f"ExternFunction({self.name!r})"


_DEVIATES = ("uniform-deviate", "normal-deviate", "lognormal-deviate", "gamma-deviate", "beta-deviate", "histogram")


def _deviate_mean(op: str, v: list) -> float:
    if op == "uniform-deviate":
        return (v[0] + v[1]) / 2
    if op == "normal-deviate":
        return v[0]
    if op == "lognormal-deviate":  # (mean, error factor, level) or (mu, sigma) of the logarithm
        return v[0] if len(v) == 3 else math.exp(v[0] + v[1] ** 2 / 2)
    if op == "gamma-deviate":  # shape k, scale theta
        return v[0] * v[1]
    if op == "beta-deviate":
        return v[0] / (v[0] + v[1])
    bounds, weights = [v[0]] + v[1::2], v[2::2]  # histogram: lower bound, then (upper, weight) per bin
    return sum((bounds[i] + bounds[i + 1]) * w for i, w in enumerate(weights)) / (2 * sum(weights))


def _p_fail(rate: float, t: float) -> float:
    return 1.0 - math.exp(-rate * t)


def _p_second(p_first: float, p_second: float, first: float, second: float, t: float) -> float:
    """Probability that the second of two Poisson processes, started when the
    first (rate `first`) occurs, has occurred by t (rate `second`)."""
    if first == second:
        return p_second - (1.0 - p_second) * second * t
    return (second * p_first - first * p_second) / (second - first)


def periodic_test(*v) -> float:
    """Unavailability of a periodically tested component at time t, the MEF
    periodic-test (mcSCRAM src/expression/exponential.cc:113-330):
    (lambda, tau, theta, t) with instant test and repair;
    (lambda, mu, tau, theta, t) with instant test and repair at rate mu;
    (lambda, lambda_test, mu, tau, theta, gamma, test_duration,
    available_at_test, sigma, omega, t) with a test phase of its own.  The
    first test is at theta, then every tau."""
    if len(v) == 4:
        lam, tau, theta, t = v
        if t <= theta:
            return _p_fail(lam, t)
        delta = t - theta
        after = delta - int(delta / tau) * tau
        return _p_fail(lam, after if after else tau)
    if len(v) == 5:
        lam, mu, tau, theta, t = v
        if t <= theta:
            return _p_fail(lam, t)

        def keep(pl, pm, dt):  # state carried through dt: still failed, or failed and not yet repaired
            return 1.0 - pm + _p_second(pl, pm, lam, mu, dt) - pl

        delta = t - theta
        n = int(delta / tau)
        frac = keep(_p_fail(lam, tau), _p_fail(mu, tau), tau)
        geo = frac ** n
        prob = _p_fail(lam, theta) * geo + _p_fail(lam, tau) * (geo - 1.0) / (frac - 1.0)
        after = delta - n * tau
        pl, pm = _p_fail(lam, after), _p_fail(mu, after)
        return prob * keep(pl, pm, after) + pl
    lam, lam_test, mu, tau, theta, gamma, dur, avail_at_test, sigma, omega, t = v
    if t <= theta:
        return _p_fail(lam, t)
    state = {"fail": _p_fail(lam, theta), "repair": 0.0}
    state["avail"] = 1.0 - state["fail"]

    def repaired_then_failed(pm, pl, dt):
        return pm * omega + (1.0 - omega) * _p_second(pm, pl, mu, lam, dt)

    def test_phase(pl_test, pm, pl, dt, available=True):
        transient = state["fail"] + state["avail"] * (gamma + (1.0 - gamma) * pl_test)
        fail = state["repair"] * repaired_then_failed(pm, pl, dt) + (1.0 - sigma) * transient
        repair = (1.0 - pm) * state["repair"] + sigma * transient
        off = 0.0 if available else state["avail"] * (1.0 - gamma) * (1.0 - pl_test)
        state.update(fail=fail, repair=repair, avail=1.0 - fail - repair - off)

    def run_phase(pl, pm, dt):
        fail = state["avail"] * pl + state["fail"] + state["repair"] * repaired_then_failed(pm, pl, dt)
        repair = state["repair"] * (1.0 - pm)
        state.update(fail=fail, repair=repair, avail=1.0 - fail - repair)

    delta = t - theta
    n = int(delta / tau)
    run = tau - dur
    at_test = (_p_fail(lam_test, dur), _p_fail(mu, dur), _p_fail(lam, dur), dur)
    between = (_p_fail(lam, run), _p_fail(mu, run), run)
    for _ in range(n):
        test_phase(*at_test)
        run_phase(*between)
    after = delta - n * tau
    if after <= dur:
        test_phase(_p_fail(lam_test, after), _p_fail(mu, after), _p_fail(lam, after), after, bool(avail_at_test))
    else:
        test_phase(*at_test)
        rest = after - dur
        run_phase(_p_fail(lam, rest), _p_fail(mu, rest), rest)
    return 1.0 - state["avail"]


def _lognormal_scale(ef, level):
    """sigma of the logarithm from an error factor at a one-sided confidence
    level: ln(ef) / z(level) (mcSCRAM src/expression/random_deviate.cc:94-101)."""
    from statistics import NormalDist
    z = np.vectorize(NormalDist().inv_cdf)(np.asarray(level, dtype=np.float64))
    return np.log(ef) / z


_COMPARE = {"eq": lambda x, y: x == y, "df": lambda x, y: x != y, "lt": lambda x, y: x < y,
            "gt": lambda x, y: x > y, "leq": lambda x, y: x <= y, "geq": lambda x, y: x >= y}


@dataclass
class Formula:
    """A connective over arguments; an argument is (complement, kind, payload)
    with kind "gate" / "basic-event" / "house-event" (payload: the element's
    id) or "formula" (payload: a nested Formula)."""
    connective: int
    args: List[Tuple[bool, str, object]]
    min_number: int = 0


# --- event trees (mcSCRAM src/event_tree.h, src/instruction.h) -------------
#
# An instruction is a tuple: ("collect-formula", Formula),
# ("collect-expression", Expr), ("set-house-event", house id, state),
# ("if", Expr, then, else or None), ("block", [instructions]),
# ("rule", name), ("link", event-tree name).


@dataclass
class Branch:
    """Instructions followed by one target: ("fork", Fork), ("sequence",
    name) or ("branch", name of a branch of the same event tree)."""
    instructions: list
    target: Tuple[str, object]


@dataclass
class Fork:
    functional_event: str
    paths: List[Tuple[str, Branch]]  # (state, branch)


@dataclass
class EventTree:
    name: str
    functional_events: List[str] = field(default_factory=list)  # definition order = fork order
    sequences: List[str] = field(default_factory=list)
    branches: Dict[str, Branch] = field(default_factory=dict)
    initial_state: Optional[Branch] = None


@dataclass
class Phase:
    name: str
    time_fraction: float
    house_events: List[Tuple[str, bool]]  # set-house-event instructions


@dataclass
class CcfGroup:
    """A common-cause failure group (mcSCRAM src/ccf_group.h): its members
    (basic-event ids, defined by the group), their distribution Q and the
    model's factors by level."""
    name: str
    model: str                      # beta-factor, MGL, alpha-factor, phi-factor
    members: List[str]
    member_names: List[str]
    distribution: Expr
    factors: List[Tuple[int, Expr]]  # (level, factor), levels ascending without gaps
    base: str = ""
    role: str = "public"


_CCF_MIN_LEVEL = {"beta-factor": None, "MGL": 2, "alpha-factor": 1, "phi-factor": 1}  # beta: the member count


@dataclass
class Substitution:
    """A substitution (mcSCRAM src/substitution.h): a hypothesis over basic
    events, the source events it replaces (none: declarative) and a target,
    either an argument (False, "basic-event" or -- members under CCF analysis
    -- "gate", id) or a constant."""
    name: str
    hypothesis: Formula
    source: List[str]
    target: Union[Tuple[bool, str, str], bool]
    type: Optional[str] = None

    @property
    def declarative(self) -> bool:
        return not self.source


_SUBSTITUTION_TYPES = ("delete-terms", "recovery-rule", "exchange-event")


@dataclass
class MefModel:
    gates: Dict[str, Formula] = field(default_factory=dict)
    basic_events: Dict[str, Expr] = field(default_factory=dict)
    house_events: Dict[str, bool] = field(default_factory=dict)
    parameters: Dict[str, Expr] = field(default_factory=dict)
    names: List[str] = field(default_factory=list)  # fault-tree names
    mission_time: float = DEFAULT_MISSION_TIME
    fault_trees: Dict[str, List[str]] = field(default_factory=dict)  # fault tree -> its gate ids
    initiating_events: Dict[str, Optional[str]] = field(default_factory=dict)  # -> event tree
    event_trees: Dict[str, EventTree] = field(default_factory=dict)
    sequences: Dict[str, list] = field(default_factory=dict)  # sequence -> instructions
    rules: Dict[str, list] = field(default_factory=dict)
    alignments: Dict[str, List[Phase]] = field(default_factory=dict)
    ccf_groups: Dict[str, CcfGroup] = field(default_factory=dict)
    substitutions: Dict[str, Substitution] = field(default_factory=dict)
    extern_libraries: Dict[str, object] = field(default_factory=dict)  # name -> loaded ctypes library
    extern_functions: Dict[str, "ExternFunction"] = field(default_factory=dict)

    def probability(self, event: str, t: Optional[float] = None) -> float:
        """Probability of a basic event at mission time t (default: the model's)."""
        e = self.basic_events[event]
        if e is None:
            raise MefError(f"basic event {event!r} has no probability expression")
        v = e.value(self.mission_time if t is None else t, self.parameters)
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

    def fault_tree_tops(self, tree: str) -> List[str]:
        """Top events of one fault tree: its gates (components included) that
        no other gate of the same tree references (mcSCRAM
        src/fault_tree.cc:63-92), in definition order."""
        own = self.fault_trees[tree]
        members = set(own)
        used = set()

        def walk(f: Formula):
            for _, kind, x in f.args:
                if kind == "gate" and x in members:
                    used.add(x)
                elif kind == "formula":
                    walk(x)

        for gid in own:
            walk(self.gates[gid])
        return [g for g in own if g not in used]

    def with_phase(self, phase: Phase) -> "MefModel":
        """A copy at the phase's share of the mission time with its house-event
        states (mcSCRAM src/risk_analysis.cc:68-96)."""
        m = copy.copy(self)
        m.mission_time = self.mission_time * phase.time_fraction
        m.house_events = dict(self.house_events)
        for name, state in phase.house_events:
            m.house_events[name] = state
        return m

    def build(self, top: Optional[str] = None):
        """Host PDAG rooted at `top` (the only top gate when None).  Returns
        (host.Pdag, root index, {basic-event name: index}, {gate name: index}).

        Declarative substitutions constrain the analysed root as the
        reference's Pdag(mef::Gate, ccf, model) does (src/pdag.cc:470-494,
        721-734): the root becomes AND(S1, ..., Sn, top) with Si = OR(NOT
        hypothesis, target), or NULL(NOT hypothesis) for a false target; the
        returned root is then that AND and gate_index[top] the top's own gate.
        Non-declarative substitutions serve cut-set approximations only: their
        events are gathered, as the reference gathers them, but the graph
        does not change."""
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

        def gather_arg(kind: str, x: str):
            gather(Formula(NULL, [(False, kind, x)]))

        seen_gates.add(top)
        gather(self.gates[top])
        outside = set()  # events only non-declarative substitutions name: never in the graph
        for s in self.substitutions.values():  # GatherVariables(mef::Substitution)
            before = set(var_index)
            gather(s.hypothesis)
            for x in s.source:
                gather_arg("basic-event", x)
            if not isinstance(s.target, bool):
                gather_arg(s.target[1], s.target[2])
            if not s.declarative:
                outside.update(set(var_index) - before)
        for s in self.substitutions.values():
            if s.declarative:
                outside.difference_update(x for _, _, x in s.hypothesis.args)
                if not isinstance(s.target, bool):
                    outside.discard(s.target[2])
        nxt = 2 + len(var_index)
        for f_name in self._house_events_in(top):
            house_index[f_name] = nxt
            nxt += 1
        # 2. gates in pre-order of construction (ConstructGate)
        pdag = Pdag()
        for name, idx in var_index.items():
            unused = name in outside and self.basic_events[name] is None
            pdag.add_variable(idx, 0.0 if unused else self.probability(name))
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
        application = counter[0]  # made whether or not a substitution applies
        counter[0] += 1
        applied = []
        for s in self.substitutions.values():
            if not s.declarative:
                continue
            idx = counter[0]
            counter[0] += 1
            hyp = construct(s.hypothesis)
            if isinstance(s.target, bool):  # a delete term
                pending.append((idx, Formula(NULL, [-hyp])))
            else:
                _, kind, x = s.target
                if kind == "gate" and x not in gate_index:
                    gate_index[x] = construct(self.gates[x])
                pending.append((idx, Formula(OR, [-hyp, var_index[x] if kind == "basic-event" else gate_index[x]])))
            applied.append(idx)
        if applied:
            pending.append((application, Formula(AND, applied + [root])))
            root = application
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


def _kids(el: ET.Element) -> List[ET.Element]:
    return [c for c in el if _local(c.tag) not in _SKIP]


_UNARY = {"abs": abs, "acos": math.acos, "asin": math.asin, "atan": math.atan, "cos": math.cos, "sin": math.sin,
          "tan": math.tan, "cosh": math.cosh, "sinh": math.sinh, "tanh": math.tanh, "exp": math.exp,
          "log": math.log, "log10": math.log10, "sqrt": math.sqrt, "ceil": math.ceil, "floor": math.floor}
_UNARY_NP = {"abs": np.abs, "acos": np.arccos, "asin": np.arcsin, "atan": np.arctan, "cos": np.cos, "sin": np.sin,
             "tan": np.tan, "cosh": np.cosh, "sinh": np.sinh, "tanh": np.tanh, "exp": np.exp, "log": np.log,
             "log10": np.log10, "sqrt": np.sqrt, "ceil": np.ceil, "floor": np.floor}
_ARITY = {"exponential": 2, "GLM": 4, "Weibull": 4, "neg": 1, "not": 1, "ite": 3,
          "eq": 2, "df": 2, "lt": 2, "gt": 2, "leq": 2, "geq": 2, "pow": 2, "mod": 2, **{k: 1 for k in _UNARY}}
_NARY = ("exponential", "GLM", "Weibull", "add", "sub", "mul", "div", "neg", "not", "and", "or", "ite", "pow", "mod",
         "min", "max", "mean") + tuple(_COMPARE) + tuple(_UNARY)


def _parse_expr(e: ET.Element, what: str) -> Expr:
    tag = _local(e.tag)
    if tag in ("float", "int"):
        return Expr("value", [float(e.get("value"))])
    if tag == "bool":
        return Expr("value", [1.0 if e.get("value", "").strip().lower() == "true" else 0.0])
    if tag == "pi":
        return Expr("value", [math.pi])
    if tag == "parameter":
        return Expr("parameter", [e.get("name")])
    if tag == "system-mission-time":
        return Expr("time", [])
    if tag == "test-initiating-event":
        return Expr(tag, [e.get("name")])
    if tag == "test-functional-event":
        return Expr(tag, [e.get("name"), e.get("state")])
    if tag == "switch":  # cases (condition, value) in order, then the default value
        kids = _kids(e)
        if not kids:
            raise MefError(f"{what}: <switch> needs a default value")
        args = []
        for c in kids[:-1]:
            if _local(c.tag) != "case" or len(_kids(c)) != 2:
                raise MefError(f"{what}: a <case> holds a condition and a value")
            args += [_parse_expr(x, what) for x in _kids(c)]
        return Expr(tag, args + [_parse_expr(kids[-1], what)])
    if tag == "periodic-test":
        args = [_parse_expr(c, what) for c in _kids(e)]
        if len(args) not in (4, 5, 11):
            raise MefError(f"{what}: <periodic-test> takes 4, 5 or 11 arguments, found {len(args)}")
        return Expr(tag, args)
    if tag in _DEVIATES:
        kids = _kids(e)
        if tag == "histogram":
            if len(kids) < 2:
                raise MefError(f"{what}: <histogram> needs a lower boundary and at least one bin")
            args = [_parse_expr(kids[0], what)]
            for b in kids[1:]:
                if _local(b.tag) != "bin" or len(_kids(b)) != 2:
                    raise MefError(f"{what}: a histogram <bin> holds an upper boundary and a weight")
                args += [_parse_expr(x, what) for x in _kids(b)]
            return Expr(tag, args)
        need = (3, 2) if tag == "lognormal-deviate" else (2,)
        if len(kids) not in need:
            raise MefError(f"{what}: <{tag}> takes {' or '.join(map(str, need))} arguments, found {len(kids)}")
        return Expr(tag, [_parse_expr(c, what) for c in kids])
    if tag == "extern-function":  # the function is resolved by name once the model is read
        return Expr(tag, [e.get("name")] + [_parse_expr(c, what) for c in _kids(e)])
    if tag in _NARY:
        args = [_parse_expr(c, what) for c in _kids(e)]
        if tag in _ARITY and len(args) != _ARITY[tag]:
            raise MefError(f"{what}: <{tag}> takes {_ARITY[tag]} arguments, found {len(args)}")
        if tag in ("add", "sub", "mul", "div", "and", "or", "min", "max", "mean") and len(args) < 2:
            raise MefError(f"{what}: <{tag}> takes 2 or more arguments, found {len(args)}")
        if not args:
            raise MefError(f"{what}: <{tag}> without arguments")
        return Expr(tag, args)
    raise MefError(f"{what}: unsupported expression <{tag}>")


def _parse_expression(el: ET.Element, what: str) -> Expr:
    kids = _kids(el)
    if len(kids) != 1:
        raise MefError(f"{what}: expected one expression, found {len(kids)}")
    return _parse_expr(kids[0], what)


def _check_arity(tag: str, n: int, where: str, k: Optional[int] = None, kmax: Optional[int] = None):
    """Argument counts the reference's mef::Formula accepts (src/event.cc:174-225)."""
    if tag in ("and", "or", "nand", "nor") and n < 2:
        raise MefError(f"{where}: <{tag}> must have 2 or more arguments")
    if tag in ("not",) and n != 1:
        raise MefError(f"{where}: <not> must have exactly one argument")
    if tag in ("xor", "imply", "iff") and n != 2:
        raise MefError(f"{where}: <{tag}> must have exactly 2 arguments")
    if tag == "atleast":
        if k is None:
            raise MefError(f"{where}: <atleast> without min")
        if k < 2:
            raise MefError(f"{where}: <atleast> min cannot be less than 2")
        if n <= k:
            raise MefError(f"{where}: <atleast> must have more arguments than its min number")
    if tag == "cardinality":
        if k is None or kmax is None:
            raise MefError(f"{where}: <cardinality> requires min and max")
        if k < 0 or k > kmax:
            raise MefError(f"{where}: <cardinality> min {k} > max {kmax}")
        if n < 1 or n < kmax:
            raise MefError(f"{where}: <cardinality> max {kmax} exceeds its {n} arguments")


def _threshold_formula(k: int, args: list) -> Tuple[bool, str, object]:
    """At least k of args, well formed as the reference shapes its two
    cardinality halves (src/pdag.cc:699-709): true for k = 0, OR for k = 1,
    AND for k = n, ATLEAST otherwise; a single argument passes through."""
    if k <= 0:
        return False, "constant", True
    if len(args) == 1:
        return args[0]
    if k == 1:
        return False, "formula", Formula(OR, list(args))
    if k == len(args):
        return False, "formula", Formula(AND, list(args))
    return False, "formula", Formula(ATLEAST, list(args), k)


def _parse_formula(el: ET.Element, where: str) -> Formula:
    tag = _local(el.tag)
    if tag in _REFS or tag == "constant":
        # a formula of a single event: a pass-through (NULL) gate
        return Formula(NULL, [_parse_arg(el, where)])
    if tag not in _CONNECTIVES and tag not in _COMPLEX:
        raise MefError(f"{where}: unsupported formula <{tag}>")
    if tag == "not" and not (len(_kids(el)) == 1 and _local(_kids(el)[0].tag) in _REFS):
        raise MefError(f"{where}: <not> takes one event")
    args = [_parse_arg(c, where) for c in _kids(el)]
    k = int(el.get("min")) if el.get("min") is not None else None
    kmax = int(el.get("max")) if el.get("max") is not None else None
    _check_arity(tag, len(args), where, k, kmax)
    if tag == "imply":  # x -> y  ==  not x or y
        (c0, k0, x0), second = args
        return Formula(OR, [(not c0, k0, x0), second])
    if tag == "iff":  # a NULL gate over the complemented XOR
        return Formula(NULL, [(True, "formula", Formula(XOR, args))])
    if tag == "cardinality":  # at least min of args and at least n - max of their complements
        negated = [(not c, kind, x) for c, kind, x in args]
        return Formula(AND, [_threshold_formula(k, args), _threshold_formula(len(args) - kmax, negated)])
    f = Formula(_CONNECTIVES[tag], args)
    if tag == "atleast":
        f.min_number = k
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
        kids = _kids(el)
        if len(kids) == 1 and _local(kids[0].tag) in _REFS:
            comp, kind, x = _parse_arg(kids[0], where)
            return (not comp), kind, x
    # share/input.rng:664-672: an argument is an event, the negation of one or a constant
    raise MefError(f"{where}: nested formula <{tag}>: an argument is an event, its negation or a constant")


class _Scope:
    """Element ids and full paths per element type, and the MEF lookup rule
    (mcSCRAM src/initializer.cc:1400-1466)."""

    def __init__(self):
        self.paths: Dict[str, Dict[str, str]] = {k: {} for k in _TABLES}  # full path -> id
        self.public: Dict[str, set] = {k: set() for k in _TABLES}
        self.ids: Dict[str, set] = {k: set() for k in _TABLES}

    def register(self, kind: str, name: str, base: str, role: str) -> str:
        if not name:
            raise MefError(f"<define-{kind}> without a name")
        full = f"{base}.{name}" if base else name
        ident = name if role == "public" else full
        if full in self.paths[kind] or ident in self.ids[kind]:
            raise MefError(f"{kind} {ident!r} defined twice")
        if kind in _EVENTS:  # gates, basic and house events share one namespace
            for other in _EVENTS:
                if other != kind and (full in self.paths[other] or ident in self.ids[other]):
                    raise MefError(f"{kind} {ident!r} clashes with the {other} of that name")
        self.paths[kind][full] = ident
        self.ids[kind].add(ident)
        if role == "public":
            self.public[kind].add(ident)
        return ident

    def lookup(self, kinds, ref: str, base: str) -> Optional[Tuple[str, str]]:
        if base:
            full = f"{base}.{ref}"
            for k in kinds:
                if full in self.paths[k]:
                    return k, self.paths[k][full]
        for k in kinds:
            if "." not in ref:
                if ref in self.public[k]:
                    return k, ref
            elif ref in self.paths[k]:
                return k, self.paths[k][ref]
        return None


def _role(el: ET.Element, parent: str) -> str:
    r = (el.get("role") or "").strip()
    return parent if not r else ("public" if r == "public" else "private")


def _parse_instruction(el: ET.Element, where: str):
    tag = _local(el.tag)
    kids = _kids(el)
    if tag == "collect-formula":
        if len(kids) != 1:
            raise MefError(f"{where}: <collect-formula> takes one formula")
        return "collect-formula", _parse_formula(kids[0], where)
    if tag == "collect-expression":
        return "collect-expression", _parse_expression(el, where)
    if tag == "set-house-event":
        if len(kids) != 1 or _local(kids[0].tag) != "constant":
            raise MefError(f"{where}: <set-house-event> takes one <constant>")
        return "set-house-event", el.get("name"), kids[0].get("value", "").strip().lower() == "true"
    if tag == "if":
        if len(kids) not in (2, 3):
            raise MefError(f"{where}: <if> takes a condition, an instruction and an optional else")
        return ("if", _parse_expr(kids[0], where), _parse_instruction(kids[1], where),
                _parse_instruction(kids[2], where) if len(kids) == 3 else None)
    if tag == "block":
        return "block", [_parse_instruction(c, where) for c in kids]
    if tag == "rule":
        return "rule", el.get("name")
    if tag == "event-tree":
        return "link", el.get("name")
    raise MefError(f"{where}: unsupported instruction <{tag}>")


def _parse_branch(kids: List[ET.Element], where: str) -> Branch:
    """Instructions, then the target as the last element (mcSCRAM
    src/initializer.cc:911-926)."""
    if not kids:
        raise MefError(f"{where}: a branch needs a target")
    *ins, last = kids
    tag = _local(last.tag)
    if tag == "fork":
        paths, states = [], set()
        for p in last:
            if _local(p.tag) != "path":
                continue
            state = p.get("state")
            if state in states:
                raise MefError(f"{where}: path state {state!r} defined twice in a fork")
            states.add(state)
            paths.append((state, _parse_branch(_kids(p), where)))
        if not paths:
            raise MefError(f"{where}: a fork without paths")
        target = ("fork", Fork(last.get("functional-event"), paths))
    elif tag in ("sequence", "branch"):
        target = (tag, last.get("name"))
    else:
        raise MefError(f"{where}: <{tag}> is not a branch target")
    return Branch([_parse_instruction(c, where) for c in ins], target)


def _walk_instructions(ins, fn, rules, seen_rules=None):
    """Calls fn on every instruction reachable from `ins` (blocks, both arms
    of an if, rules followed once)."""
    seen_rules = set() if seen_rules is None else seen_rules
    for x in ins:
        fn(x)
        kind = x[0]
        if kind == "block":
            _walk_instructions(x[1], fn, rules, seen_rules)
        elif kind == "if":
            arms = [x[2]] + ([x[3]] if x[3] is not None else [])
            _walk_instructions(arms, fn, rules, seen_rules)
        elif kind == "rule" and x[1] in rules and x[1] not in seen_rules:
            seen_rules.add(x[1])
            _walk_instructions(rules[x[1]], fn, rules, seen_rules)


def _find_cycle(edges: Dict[str, List[str]]) -> Optional[str]:
    state: Dict[str, int] = {}
    for start in edges:
        if state.get(start):
            continue
        stack = [(start, iter(edges.get(start, ())))]
        state[start] = 1
        while stack:
            node, it = stack[-1]
            nxt = next(it, None)
            if nxt is None:
                state[node] = 2
                stack.pop()
                continue
            s = state.get(nxt, 0)
            if s == 1:
                return nxt
            if s == 0:
                state[nxt] = 1
                stack.append((nxt, iter(edges.get(nxt, ()))))
    return None


_XINCLUDE = "{http://www.w3.org/2001/XInclude}include"
_INT_MAX = (1 << 31) - 1


def _document(source: Union[str, Path], _including: Tuple[Path, ...] = ()) -> ET.Element:
    """One MEF document, its XIncludes resolved, with the checks the
    reference's RELAX NG schema makes on what this reader keeps
    (share/input.rng): no element or attribute of a foreign namespace, no
    blank label or attribute value, ints within 32 bits."""
    is_file = isinstance(source, Path) or not source.lstrip().startswith("<")
    if is_file and Path(source).resolve() in _including:
        raise MefError(f"XInclude cycle through {str(source)!r}")
    text = Path(source).read_text() if is_file else source
    try:
        root = ET.fromstring(text.lstrip("\ufeff"))
    except ET.ParseError as e:
        raise MefError(f"not well-formed XML: {e}") from None
    if _local(root.tag) != "opsa-mef":
        raise MefError("root element is not <opsa-mef>")
    chain = _including + ((Path(source).resolve(),) if is_file else ())
    for parent in list(root.iter()):  # XInclude of another document's top-level elements
        for i, child in reversed(list(enumerate(parent))):
            if child.tag != _XINCLUDE:
                continue
            href, xp = child.get("href"), (child.get("xpointer") or "").replace(" ", "")
            if not href or xp != "xpointer(/opsa-mef/*)":
                raise MefError(f"XInclude of {href!r}: only xpointer(/opsa-mef/*) of a file is read")
            target = _directory(source) / href
            if not target.is_file():
                raise MefError(f"XInclude of {href!r}: no such file")
            parent[i:i + 1] = list(_document(target, chain))
    for el in root.iter():
        if "}" in el.tag or any("}" in a for a in el.keys()):
            raise MefError(f"<{el.tag}>: elements and attributes of other namespaces are not MEF")
        for a in ("name", "event-tree", "functional-event", "state"):  # names without surrounding blanks
            if el.get(a) is not None:
                el.set(a, el.get(a).strip())
        tag = el.tag
        if tag == "label" and not (el.text or "").strip():
            raise MefError("a <label> without text")
        if tag == "attribute" and not (el.get("value") or "").strip():
            raise MefError(f"attribute {el.get('name')!r} without a value")
        if tag == "int" and el.get("value") is not None:  # a valueless <int/> is an extern parameter type
            try:
                v = int((el.get("value") or "").strip())
            except ValueError:
                raise MefError(f"<int value={el.get('value')!r}> is not an integer") from None
            if abs(v) > _INT_MAX:
                raise MefError(f"<int value={el.get('value')!r}> overflows a 32-bit int")
        if tag == "attributes":
            names = [a.get("name") for a in el]
            if len(names) != len(set(names)):
                raise MefError(f"an element repeats one of its attributes {sorted(names)}")
    return root


def _directory(source: Union[str, Path]) -> Path:
    """The directory relative library paths of a document start from."""
    if isinstance(source, Path) or not source.lstrip().startswith("<"):
        return Path(source).resolve().parent
    return Path.cwd()


def _load_library(el: ET.Element, directory: Path):
    """An extern library (mcSCRAM src/expression/extern.cc:29-65): the path
    is relative to the defining document unless `system` asks for the
    loader's own search (a bare name); `decorate` adds the platform's lib
    prefix and .so suffix."""
    import ctypes
    name, path = el.get("name"), el.get("path") or ""
    fname = Path(path).name
    if not path or fname in (".", "..") or path[-1] in ":/\\":
        raise MefError(f"extern library {name!r}: invalid library path format {path!r}")
    system = (el.get("system") or "false").strip().lower() == "true"
    if (el.get("decorate") or "false").strip().lower() == "true":
        path = str(Path(path).with_name(f"lib{fname}.so"))
    if not system or "/" in path:
        path = str(directory / path)
    try:
        return ctypes.CDLL(path)
    except OSError as e:
        raise MefError(f"extern library {name!r}: {e}") from None


def parse(source: Union[str, Path, List[Union[str, Path]]],
          mission_time: float = DEFAULT_MISSION_TIME, ccf_analysis: bool = False,
          allow_extern: bool = False) -> MefModel:
    """Reads a MEF document (a path, or the XML text itself) or several
    documents forming one model (a list; references may cross them);
    probabilities are evaluated at `mission_time` unless asked for at another
    time.  With `ccf_analysis` the members of common-cause groups become OR
    gates over their CCF events (SCRAM's --ccf); without it they are basic
    events with the group's distribution, as in SCRAM.  Extern libraries
    are loaded only with `allow_extern` (SCRAM's --allow-extern): loading one
    runs its code."""
    sources = source if isinstance(source, (list, tuple)) else [source]
    files = [Path(x).resolve() for x in sources if isinstance(x, Path) or not x.lstrip().startswith("<")]
    if len(files) != len(set(files)):
        raise MefError("the same file is given twice")
    roots = [_document(x) for x in sources]
    dirs = [_directory(x) for x in sources]
    m = MefModel(mission_time=float(mission_time))
    scope = _Scope()
    gate_base: Dict[str, str] = {}
    expr_base: List[Tuple[Expr, str]] = []
    collected: List[Formula] = []  # collect-formula formulas (global scope)

    components = set()

    def visit_data(container: ET.Element, base: str, role: str, tree: Optional[str]):
        for el in container:
            tag = _local(el.tag)
            name = el.get("name")
            if not base and _role(el, role) != "public":
                raise MefError(f"{name!r}: private elements need a fault tree or component")
            if tag == "define-gate":
                kids = _kids(el)
                ident = scope.register("gate", name, base, _role(el, role))
                if len(kids) != 1:
                    raise MefError(f"gate {ident!r}: expected one formula, found {len(kids)}")
                m.gates[ident] = _parse_formula(kids[0], f"gate {ident!r}")
                gate_base[ident] = base
                if tree is not None:
                    m.fault_trees[tree].append(ident)
            elif tag == "define-basic-event":
                ident = scope.register("basic-event", name, base, _role(el, role))
                if _kids(el):  # an event without an expression serves qualitative analyses only
                    m.basic_events[ident] = _parse_expression(el, f"basic event {ident!r}")
                    expr_base.append((m.basic_events[ident], base))
                else:
                    m.basic_events[ident] = None
            elif tag == "define-house-event":
                ident = scope.register("house-event", name, base, _role(el, role))
                kids = _kids(el)
                m.house_events[ident] = bool(kids) and kids[0].get("value", "").strip().lower() == "true"
            elif tag == "define-parameter":
                ident = scope.register("parameter", name, base, _role(el, role))
                m.parameters[ident] = _parse_expression(el, f"parameter {ident!r}")
                expr_base.append((m.parameters[ident], base))
            elif tag == "define-CCF-group":
                define_ccf(el, base, _role(el, role))
            elif tag == "define-component":
                if tree is None:
                    raise MefError("<define-component> outside a fault tree")
                if f"{base}.{name}" in components:
                    raise MefError(f"component {base + '.' + name!r} defined twice")
                components.add(f"{base}.{name}")
                visit_data(el, f"{base}.{name}", _role(el, role), tree)
            elif tag in _SKIP:
                continue
            else:
                raise MefError(f"unsupported element <{tag}>")

    def define_ccf(el: ET.Element, base: str, role: str):
        """A CCF group with the checks of mcSCRAM src/ccf_group.cc:51-139."""
        name, model = el.get("name"), el.get("model")
        where = f"CCF group {name!r}"
        if name in m.ccf_groups:
            raise MefError(f"{where} defined twice")
        if model not in _CCF_MIN_LEVEL:
            raise MefError(f"{where}: unknown model {model!r}")
        members, names, dist, factors = [], [], None, {}
        prev = 0
        for c in _kids(el):
            tag = _local(c.tag)
            if tag == "members":
                for b in _kids(c):
                    nm = b.get("name")
                    if nm in names:
                        raise MefError(f"{where}: member {nm!r} listed twice")
                    names.append(nm)
                    members.append(scope.register("basic-event", nm, base, role))
            elif tag == "distribution":
                dist = _parse_expression(c, where)
            elif tag in ("factor", "factors"):
                for f in ([c] if tag == "factor" else _kids(c)):
                    n = len(members)
                    min_level = n if model == "beta-factor" else _CCF_MIN_LEVEL[model]
                    level = int(f.get("level")) if f.get("level") else (prev + 1 if prev else min_level)
                    if level < min_level:
                        raise MefError(f"{where}: factor level {level} below the minimum {min_level}")
                    if level > n:
                        raise MefError(f"{where}: factor level {level} above the {n} members")
                    if level in factors:
                        raise MefError(f"{where}: factor for level {level} defined twice")
                    factors[level] = _parse_expression(f, where)
                    prev = level
            else:
                raise MefError(f"{where}: unsupported element <{tag}>")
        if len(members) < 2:
            raise MefError(f"{where}: a CCF group needs at least 2 members")
        if dist is None or not factors:
            raise MefError(f"{where}: distribution and factors are required")
        min_level = len(members) if model == "beta-factor" else _CCF_MIN_LEVEL[model]
        if sorted(factors) != list(range(min_level, max(factors) + 1)):
            raise MefError(f"{where}: missing CCF factors")
        for mid in members:
            m.basic_events[mid] = dist
        expr_base.append((dist, base))
        for f in factors.values():
            expr_base.append((f, base))
        m.ccf_groups[name] = CcfGroup(name, model, members, names, dist, sorted(factors.items()), base, role)

    def define_event_tree(el: ET.Element):
        name = el.get("name")
        if name in m.event_trees:
            raise MefError(f"event tree {name!r} defined twice")
        et = EventTree(name)
        where = f"event tree {name!r}"
        for c in el:
            tag = _local(c.tag)
            cname = c.get("name")
            if tag == "define-functional-event":
                if cname in et.functional_events:
                    raise MefError(f"{where}: functional event {cname!r} defined twice")
                et.functional_events.append(cname)
            elif tag == "define-sequence":
                if cname in m.sequences:
                    raise MefError(f"sequence {cname!r} defined twice")
                m.sequences[cname] = [_parse_instruction(i, f"sequence {cname!r}") for i in _kids(c)]
                et.sequences.append(cname)
            elif tag == "define-branch":
                if cname in et.branches:
                    raise MefError(f"{where}: branch {cname!r} defined twice")
                et.branches[cname] = _parse_branch(_kids(c), f"{where}, branch {cname!r}")
            elif tag == "initial-state":
                et.initial_state = _parse_branch(_kids(c), f"{where}, initial state")
            elif tag in _SKIP:
                continue
            else:
                raise MefError(f"{where}: unsupported element <{tag}>")
        if et.initial_state is None:
            raise MefError(f"{where}: no initial state")
        m.event_trees[name] = et

    def define_substitution(el: ET.Element):
        """<define-substitution> as read by mcSCRAM src/initializer.cc:619-669;
        references are resolved, and the checks made, once every file is read."""
        name = el.get("name")
        if not name:
            raise MefError("<define-substitution> without a name")
        where = f"substitution {name!r}"
        if name in m.substitutions:
            raise MefError(f"{where} defined twice")
        parts = {_local(c.tag): c for c in _kids(el)}
        hyp, tgt = parts.get("hypothesis"), parts.get("target")
        if hyp is None or len(_kids(hyp)) != 1 or tgt is None or len(_kids(tgt)) != 1:
            raise MefError(f"{where}: needs one hypothesis formula and one target")
        source = []
        for b in _kids(parts["source"]) if "source" in parts else []:
            if _local(b.tag) != "basic-event":
                raise MefError(f"{where}: the source holds basic events only")
            source.append(b.get("name"))
        t = _kids(tgt)[0]
        if _local(t.tag) == "basic-event":
            target = (False, "basic-event", t.get("name"))
        elif _local(t.tag) == "constant":
            target = t.get("value", "").strip().lower() == "true"
        else:
            raise MefError(f"{where}: the target is a basic event or a constant")
        stype = el.get("type")
        if stype is not None and stype not in _SUBSTITUTION_TYPES:
            raise MefError(f"{where}: unknown type {stype!r}")
        m.substitutions[name] = Substitution(name, _parse_formula(_kids(hyp)[0], where), source, target, stype)

    for el, doc_dir in ((x, d) for r, d in zip(roots, dirs) for x in r):
        tag = _local(el.tag)
        name = el.get("name")
        if tag == "define-fault-tree":
            if name in m.fault_trees:
                raise MefError(f"fault tree {name!r} defined twice")
            m.names.append(name)
            m.fault_trees[name] = []
            visit_data(el, name, "public", name)  # fault trees are public (src/fault_tree.h:128-130)
        elif tag == "model-data":
            visit_data(el, "", "public", None)
        elif tag in ("define-gate", "define-basic-event", "define-house-event", "define-parameter",
                     "define-CCF-group"):
            visit_data([el], "", "public", None)
        elif tag == "define-event-tree":
            define_event_tree(el)
        elif tag == "define-substitution":
            define_substitution(el)
        elif tag == "define-extern-library":  # initializer.cc:481-488
            if not allow_extern:
                raise MefError(f"extern library {name!r}: loading external libraries is disallowed")
            if name in m.extern_libraries:
                raise MefError(f"extern library {name!r} defined twice")
            m.extern_libraries[name] = _load_library(el, doc_dir)
        elif tag == "define-extern-function":
            continue  # once every library is loaded
        elif tag == "define-initiating-event":
            if name in m.initiating_events:
                raise MefError(f"initiating event {name!r} defined twice")
            m.initiating_events[name] = el.get("event-tree") or None
        elif tag == "define-rule":
            if name in m.rules:
                raise MefError(f"rule {name!r} defined twice")
            m.rules[name] = [_parse_instruction(c, f"rule {name!r}") for c in _kids(el)]
        elif tag == "define-alignment":
            if name in m.alignments:
                raise MefError(f"alignment {name!r} defined twice")
            phases, total = [], 0.0
            for ph in el:
                if _local(ph.tag) != "define-phase":
                    continue
                frac = float(ph.get("time-fraction"))
                if not 0.0 < frac <= 1.0:
                    raise MefError(f"alignment {name!r}: phase time fraction {frac} outside (0, 1]")
                if any(p.name == ph.get("name") for p in phases):
                    raise MefError(f"alignment {name!r}: phase {ph.get('name')!r} defined twice")
                sets = [_parse_instruction(c, f"phase {ph.get('name')!r}") for c in _kids(ph)]
                if any(s[0] != "set-house-event" for s in sets):
                    raise MefError(f"alignment {name!r}: phases hold only set-house-event instructions")
                phases.append(Phase(ph.get("name"), frac, [(s[1], s[2]) for s in sets]))
                total += frac
            if not phases or abs(total - 1.0) > 1e-9:
                raise MefError(f"alignment {name!r}: phase time fractions sum to {total}, not 1")
            m.alignments[name] = phases
        elif tag in _SKIP:
            continue
        else:
            raise MefError(f"unsupported element <{tag}>")

    # extern functions, from every document (initializer.cc:1578-1626)
    for el in (x for r in roots for x in r if _local(x.tag) == "define-extern-function"):
        name = el.get("name")
        where = f"extern function {name!r}"
        if name in m.extern_functions:
            raise MefError(f"{where} defined twice")
        if el.get("library") not in m.extern_libraries:
            raise MefError(f"{where}: undefined extern library {el.get('library')!r}")
        types = [_local(c.tag) for c in _kids(el)]
        if not types or any(t not in ("int", "double") for t in types):
            raise MefError(f"{where}: needs a return type and parameter types, each <int/> or <double/>")
        if len(types) - 1 > ExternFunction.MAX_PARAMS:
            raise MefError(f"{where}: the number of function parameters {len(types) - 1} exceeds the "
                           f"{ExternFunction.MAX_PARAMS} allowed")
        m.extern_functions[name] = ExternFunction(name, el.get("symbol") or "", m.extern_libraries[el.get("library")],
                                                  types)

    # resolve parameter references and extern functions in expressions
    def resolve_expr(e: Expr, base: str, where: str):
        if e.op == "parameter":
            hit = scope.lookup(("parameter",), e.args[0], base)
            if hit is None:
                raise MefError(f"{where}: unknown parameter {e.args[0]!r}")
            e.args = [hit[1]]
        elif e.op == "extern-function":
            if not isinstance(e.args[0], ExternFunction):
                fn = m.extern_functions.get(e.args[0])
                if fn is None:
                    raise MefError(f"{where}: undefined extern function {e.args[0]!r}")
                if len(e.args) - 1 != fn.arity:
                    raise MefError(f"{where}: extern function {fn.name!r} takes {fn.arity} arguments, "
                                   f"found {len(e.args) - 1}")
                e.args[0] = fn
            for x in e.args[1:]:
                resolve_expr(x, base, where)
        elif e.op not in ("value", "time", "test-initiating-event", "test-functional-event"):
            for x in e.args:
                resolve_expr(x, base, where)

    for e, base in expr_base:
        resolve_expr(e, base, "expression")
    for e, _ in expr_base:
        _check_deviates(e, m)
    for name, e in m.basic_events.items():
        if e is not None:
            v = e.value(m.mission_time, m.parameters)
            if not 0.0 <= v <= 1.0:
                raise MefError(f"basic event {name!r}: probability {v} outside [0, 1]")

    # resolve event references, untyped references and constants
    def resolve(f: Formula, base: str, where: str):
        out = []
        for comp, kind, x in f.args:
            if kind == "constant":
                key = f"__constant_{'true' if x else 'false'}"
                m.house_events.setdefault(key, bool(x))
                scope.public["house-event"].add(key)
                kind, x = "house-event", key
            elif kind == "formula":
                resolve(x, base, where)
            else:
                kinds = ("gate", "basic-event", "house-event") if kind == "event" else (kind,)
                hit = scope.lookup(kinds, x, base)
                if hit is None:
                    raise MefError(f"{where}: unknown {kind} {x!r}")
                kind, x = hit
            if kind != "formula" and any(k == kind and y == x for _, k, y in out):
                raise MefError(f"{where}: {kind} {x!r} is an argument twice")
            out.append((comp, kind, x))
        f.args = out

    for gid, f in m.gates.items():
        resolve(f, gate_base[gid], f"gate {gid!r}")
    for grp in m.ccf_groups.values():
        _check_ccf(m, grp)
    for s in m.substitutions.values():
        where = f"substitution {s.name!r}"
        resolve(s.hypothesis, "", where)
        seen = set()
        for i, x in enumerate(s.source):
            hit = scope.lookup(("basic-event",), x, "")
            if hit is None:
                raise MefError(f"{where}: unknown basic event {x!r}")
            if hit[1] in seen:
                raise MefError(f"{where}: source event {hit[1]!r} listed twice")
            seen.add(hit[1])
            s.source[i] = hit[1]
        if not isinstance(s.target, bool):
            hit = scope.lookup(("basic-event",), s.target[2], "")
            if hit is None:
                raise MefError(f"{where}: unknown basic event {s.target[2]!r}")
            s.target = (False, "basic-event", hit[1])
        _check_substitution(s)
    _check_substitution_conflicts(m)

    def resolve_instructions(ins, where: str):
        def fn(x):
            if x[0] == "collect-formula":
                resolve(x[1], "", where)
            elif x[0] == "collect-expression":
                resolve_expr(x[1], "", where)
            elif x[0] == "if":
                resolve_expr(x[1], "", where)
            elif x[0] == "set-house-event":
                if scope.lookup(("house-event",), x[1], "") is None:
                    raise MefError(f"{where}: set-house-event of undefined house event {x[1]!r}")
            elif x[0] == "rule" and x[1] not in m.rules:
                raise MefError(f"{where}: undefined rule {x[1]!r}")
            elif x[0] == "link" and x[1] not in m.event_trees:
                raise MefError(f"{where}: link to undefined event tree {x[1]!r}")
        _walk_instructions(ins, fn, {})

    for rname, ins in m.rules.items():
        resolve_instructions(ins, f"rule {rname!r}")
    for sname, ins in m.sequences.items():
        resolve_instructions(ins, f"sequence {sname!r}")
    for aname, phases in m.alignments.items():
        for ph in phases:
            for h, _ in ph.house_events:
                if scope.lookup(("house-event",), h, "") is None:
                    raise MefError(f"alignment {aname!r}: undefined house event {h!r}")
    for et in m.event_trees.values():
        where = f"event tree {et.name!r}"
        for b in _branches_of(et):
            resolve_instructions(b.instructions, where)
            if b.target[0] == "fork" and b.target[1].functional_event not in et.functional_events:
                raise MefError(f"{where}: undefined functional event {b.target[1].functional_event!r}")
            if b.target[0] == "sequence" and b.target[1] not in m.sequences:
                raise MefError(f"{where}: undefined sequence {b.target[1]!r}")
            if b.target[0] == "branch" and b.target[1] not in et.branches:
                raise MefError(f"{where}: undefined branch {b.target[1]!r}")
    for ie, tree in m.initiating_events.items():
        if tree is not None and tree not in m.event_trees:
            raise MefError(f"initiating event {ie!r}: undefined event tree {tree!r}")

    _validate(m)
    if ccf_analysis:
        _expand_ccf(m)
    return m


def _check_deviates(e: Expr, m: MefModel, _depth: int = 0):
    """Parameter domains of the random deviates (mcSCRAM
    src/expression/random_deviate.cc), at the arguments' point values."""
    if _depth > 64 or e.op in ("value", "time", "parameter", "test-initiating-event", "test-functional-event"):
        return
    for x in _expr_args(e):
        _check_deviates(x, m, _depth + 1)
    if e.op in ("log", "log10", "sqrt", "acos", "asin", "div", "mod"):
        v = [x.value(m.mission_time, m.parameters) for x in e.args]
        if (e.op in ("log", "log10") and v[0] <= 0) or (e.op == "sqrt" and v[0] < 0) or \
                (e.op in ("acos", "asin") and not -1 <= v[0] <= 1) or \
                (e.op == "div" and any(x == 0 for x in v[1:])) or (e.op == "mod" and int(v[1]) == 0):
            raise MefError(f"<{e.op}>: argument {v} outside its domain")
        return
    if e.op == "periodic-test":
        v = [x.value(m.mission_time, m.parameters) for x in e.args]
        lam, tau, theta, t = (v[0], v[1], v[2], v[3]) if len(v) == 4 else (v[0], v[2], v[3], v[4]) if len(v) == 5 \
            else (v[0], v[3], v[4], v[10])
        bad = lam <= 0 or tau <= 0 or theta < 0 or t < 0
        if len(v) == 5:
            bad |= v[1] < 0
        if len(v) == 11:
            bad |= v[1] < 0 or v[2] < 0 or v[6] <= 0 or v[6] > tau or not all(0 <= v[i] <= 1 for i in (5, 8, 9))
        if bad:
            raise MefError("<periodic-test>: a rate, period, time or probability is out of its domain "
                           "(or the test lasts longer than the period)")
        return
    if e.op not in _DEVIATES:
        return
    v = [x.value(m.mission_time, m.parameters) for x in e.args]
    op = e.op
    bad = None
    if op == "uniform-deviate" and v[0] >= v[1]:
        bad = "min is not below max"
    elif op == "normal-deviate" and v[1] <= 0:
        bad = "standard deviation is not positive"
    elif op == "lognormal-deviate" and len(v) == 3 and not (0 < v[2] < 1 and v[1] > 1 and v[0] > 0):
        bad = "needs a positive mean, an error factor above 1 and a level in (0, 1)"
    elif op == "lognormal-deviate" and len(v) == 2 and v[1] <= 0:
        bad = "standard deviation is not positive"
    elif op in ("gamma-deviate", "beta-deviate") and (v[0] <= 0 or v[1] <= 0):
        bad = "shape and scale parameters must be positive"
    elif op == "histogram":
        bounds, weights = [v[0]] + v[1::2], v[2::2]
        if any(w < 0 for w in weights) or any(b1 <= b0 for b0, b1 in zip(bounds, bounds[1:])):
            bad = "weights must not be negative and boundaries must increase"
    if bad:
        raise MefError(f"<{op}>: {bad}")


def sample_expressions(model: MefModel, exprs: Dict[str, Expr], n: int, rng: np.random.Generator,
                       t: Optional[float] = None) -> Dict[str, np.ndarray]:
    """n joint samples of several expressions, as one uncertainty trial each
    (UncertaintyAnalyzer::SampleExpressions, mcSCRAM
    src/uncertainty_analysis.cc:108-120): every random deviate is drawn once
    per trial however many expressions reach it (through parameters or
    otherwise) and the rest is evaluated on those draws.  Draws come from
    numpy's generator, not the reference's mt19937, so the numbers differ and
    the distributions agree."""
    t = model.mission_time if t is None else float(t)
    cache: Dict[int, np.ndarray] = {}

    def s(e: Expr, depth: int = 0) -> np.ndarray:
        if depth > 64:
            raise MefError("parameters refer to each other in a cycle")
        key = id(e)
        if key in cache:
            return cache[key]
        op, a = e.op, e.args
        if op == "value":
            r = np.full(n, float(a[0]))
        elif op == "time":
            r = np.full(n, t)
        elif op == "parameter":
            r = s(model.parameters[a[0]], depth + 1)
        elif op in ("test-initiating-event", "test-functional-event"):
            r = np.zeros(n)
        elif op == "ite":
            r = np.where(s(a[0], depth + 1) != 0, s(a[1], depth + 1), s(a[2], depth + 1))
        elif op == "switch":
            r = s(a[-1], depth + 1)
            for i in range(len(a) - 3, -1, -2):  # the first true case wins
                r = np.where(s(a[i], depth + 1) != 0, s(a[i + 1], depth + 1), r)
        elif op == "extern-function":  # one call per trial
            v = [np.broadcast_to(s(x, depth + 1), (n,)) for x in a[1:]]
            r = np.array([a[0](*(x[i] for x in v)) for i in range(n)], dtype=np.float64)
        else:
            v = [s(x, depth + 1) for x in a]
            if op == "uniform-deviate":
                r = rng.uniform(v[0], v[1])
            elif op == "normal-deviate":
                r = rng.normal(v[0], v[1])
            elif op == "lognormal-deviate":
                if len(v) == 3:
                    sigma = _lognormal_scale(v[1], v[2])
                    r = np.exp(rng.normal(np.log(v[0]) - sigma ** 2 / 2, sigma))
                else:
                    r = np.exp(rng.normal(v[0], v[1]))
            elif op == "gamma-deviate":
                r = rng.gamma(v[0], v[1])
            elif op == "beta-deviate":
                r = rng.beta(v[0], v[1])
            elif op == "histogram":  # piecewise constant: a bin by weight, then uniform within it
                bounds = np.stack([v[0]] + v[1::2], axis=1)
                weights = np.stack(v[2::2], axis=1)
                cum = np.cumsum(weights, axis=1)
                k = np.minimum((cum < rng.random(n)[:, None] * cum[:, -1:]).sum(axis=1), weights.shape[1] - 1)
                lo = np.take_along_axis(bounds, k[:, None], axis=1)[:, 0]
                hi = np.take_along_axis(bounds, k[:, None] + 1, axis=1)[:, 0]
                r = rng.uniform(lo, hi)
            elif op == "periodic-test":
                r = np.array([periodic_test(*(float(x[i]) for x in v)) for i in range(n)])
            elif op == "exponential":
                r = -np.expm1(-v[0] * v[1])
            elif op == "GLM":
                g, lam, mu, tt = v
                rr = lam + mu
                r = (lam - (lam - g * rr) * np.exp(-rr * tt)) / rr
            elif op == "Weibull":
                al, be, t0, tt = v
                r = np.where(tt <= t0, 0.0, -np.expm1(-(np.maximum(tt - t0, 0.0) / al) ** be))
            elif op == "add":
                r = np.sum(v, axis=0)
            elif op == "mul":
                r = np.prod(v, axis=0)
            elif op == "sub":
                r = v[0] - np.sum(v[1:], axis=0)
            elif op == "div":
                r = v[0]
                for x in v[1:]:
                    r = r / x
            elif op == "neg":
                r = -v[0]
            elif op in _UNARY_NP:
                r = _UNARY_NP[op](v[0]).astype(np.float64)
            elif op == "pow":
                r = np.power(v[0], v[1])
            elif op == "mod":
                r = np.fmod(np.trunc(v[0]), np.trunc(v[1]))
            elif op == "min":
                r = np.min(v, axis=0)
            elif op == "max":
                r = np.max(v, axis=0)
            elif op == "mean":
                r = np.mean(v, axis=0)
            elif op == "not":
                r = (v[0] == 0).astype(np.float64)
            elif op == "and":
                r = np.all(np.stack(v) != 0, axis=0).astype(np.float64)
            elif op == "or":
                r = np.any(np.stack(v) != 0, axis=0).astype(np.float64)
            elif op in _COMPARE:
                r = _COMPARE[op](v[0], v[1]).astype(np.float64)
            else:
                raise MefError(f"unknown expression {op!r}")
        cache[key] = r
        return r

    return {name: s(e) for name, e in exprs.items()}


def uncertainty(model: MefModel, trials: int = 1000, words: int = 1 << 14, seed: int = 0,
                top: Optional[str] = None, device: int = 0, iteration: int = 1):
    """Uncertainty analysis of a MEF model on the GPU (UncertaintyAnalyzer,
    mcSCRAM src/uncertainty_analysis.h:154-168, .cc:122-158): each trial draws
    the model's random deviates once, evaluates the basic-event probabilities
    and estimates P(top) from `words` * 64 samples; all trials are instances
    of one tree in one batched launch (they share their counters, so four at a
    time share their Philox calls).  Returns the per-trial estimates, the
    point estimate's inputs and the reference's statistics (mean, sigma,
    error factor exp(1.96 sigma), 95 % interval of the mean, quantiles)."""
    from .graph import probability_threshold
    from .uncertainty import Batch

    pdag, root, var_index, _ = model.build(top)
    g = pdag.flatten([root])
    g.root = int(g.tally_nodes[0])
    name_of = {idx: name for name, idx in var_index.items()}
    in_graph = set(map(int, g.be_pdag_idx))
    rng = np.random.default_rng(seed)
    draws = sample_expressions(model, {n: model.basic_events[n] for n, i in var_index.items() if i in in_graph},
                               trials, rng)
    qp = g.quantised_probabilities()
    p = np.empty((trials, g.n_be))
    for i, x in enumerate(g.be_pdag_idx):
        name = name_of.get(int(x))
        p[:, i] = qp[i] if name is None else draws[name]  # house events keep their constant word
    p = np.clip(p, 0.0, 1.0)
    thr = [probability_threshold(row) for row in p]
    with Batch([g], device=device) as b:
        ones = b.run([0] * trials, thr, iteration=iteration, words_per_instance=words)
        ms = b.info()["last_kernel_ms"]
    v = np.asarray(ones, dtype=np.float64) / (words * 64.0)
    mean = float(v.mean())
    sd = float(v.std(ddof=1)) if trials > 1 else 0.0
    half = 1.96 * sd / math.sqrt(trials)
    stats = {"mean": mean, "sigma": sd, "error_factor": math.exp(1.96 * sd), "ci95": [mean - half, mean + half],
             "p05": float(np.quantile(v, 0.05)), "p50": float(np.quantile(v, 0.50)),
             "p95": float(np.quantile(v, 0.95)), "min": float(v.min()), "max": float(v.max())}
    return {"p_top": v, "stats": stats, "thresholds": thr, "graph": g, "kernel_ms": ms}


def _check_ccf(m: MefModel, grp: CcfGroup):
    where = f"CCF group {grp.name!r}"
    q = grp.distribution.value(m.mission_time, m.parameters)
    if not 0.0 <= q <= 1.0:
        raise MefError(f"{where}: distribution {q} is not a probability")
    vals = [f.value(m.mission_time, m.parameters) for _, f in grp.factors]
    if any(not 0.0 <= v <= 1.0 for v in vals):
        raise MefError(f"{where}: factors {vals} are not all probabilities")
    if grp.model == "phi-factor" and abs(sum(vals) - 1.0) > 1e-4:
        raise MefError(f"{where}: phi factors sum to {sum(vals)}, not 1")


def substitution_type(s: Substitution) -> Optional[str]:
    """The type a substitution's form implies (mcSCRAM
    src/substitution.cc:92-133): delete-terms for a false target over two
    mutually exclusive events (AND of two, or at least 2 of n), recovery-rule
    for a declarative AND or a source equal to the hypothesis' events,
    exchange-event for one source event of an AND/NULL hypothesis."""
    hyp = s.hypothesis
    events = [x for _, _, x in hyp.args]
    if not s.source:
        if isinstance(s.target, bool):
            exclusive = (hyp.connective == ATLEAST and hyp.min_number == 2) or (
                hyp.connective == AND and len(hyp.args) == 2)
            return "delete-terms" if exclusive else None
        return "recovery-rule" if hyp.connective == AND else None
    if isinstance(s.target, bool) or hyp.connective not in (AND, NULL):
        return None
    if len(s.source) == len(events):
        return "recovery-rule" if all(x in events for x in s.source) else None
    if len(s.source) == 1 and s.source[0] in events:
        return "exchange-event"
    return None


def _check_substitution(s: Substitution):
    """Substitution::Validate and the declared-type check (mcSCRAM
    src/substitution.cc:38-90, src/initializer.cc:655-668)."""
    where = f"substitution {s.name!r}"
    hyp = s.hypothesis
    if any(kind != "basic-event" for _, kind, _ in hyp.args):
        raise MefError(f"{where}: the hypothesis must be built over basic events only")
    if any(comp for comp, _, _ in hyp.args):
        raise MefError(f"{where}: the hypothesis must be coherent")
    if s.declarative:
        if hyp.connective not in (NULL, AND, ATLEAST, OR):
            raise MefError(f"{where}: the hypothesis must be coherent")
        if s.target is True:
            raise MefError(f"{where}: the substitution has no effect")
    else:
        if hyp.connective not in (NULL, AND, OR):
            raise MefError(f"{where}: a non-declarative hypothesis allows AND/OR/NULL connectives only")
        if s.target is False:
            raise MefError(f"{where}: the source set is irrelevant")
    if s.type is not None and substitution_type(s) != s.type:
        raise MefError(f"{where}: the declared type {s.type!r} does not match the deduced one")


def _check_substitution_conflicts(m: MefModel):
    """EnsureNoSubstitutionConflicts and EnsureNoCcfSubstitutions (mcSCRAM
    src/initializer.cc:1805-1866) over the non-declarative substitutions.
    Non-declarative substitutions are kept for a Monte Carlo analysis, whose
    approximation is not `none` (src/settings.cc:30-45), as the reference
    keeps them; they do not change its graph."""
    subs = [s for s in m.substitutions.values() if not s.declarative]
    ccf_members = {x for grp in m.ccf_groups.values() for x in grp.members}
    for origin in subs:
        where = f"substitution {origin.name!r}"
        target = None if isinstance(origin.target, bool) else origin.target[2]
        for other in subs:
            if target is not None and target in other.source:
                raise MefError(f"{where}: the target event should not appear in any substitution source")
            if other is origin:
                continue
            events = {x for _, _, x in other.hypothesis.args}
            if target is not None and target in events:
                raise MefError(f"{where}: the target event should not appear in another substitution hypothesis")
            if any(x in events for x in origin.source):
                raise MefError(f"{where}: a source event should not appear in another substitution hypothesis")
    for s in subs:
        events = [x for _, _, x in s.hypothesis.args] + list(s.source)
        if not isinstance(s.target, bool):
            events.append(s.target[2])
        if any(x in ccf_members for x in events):
            raise MefError(f"substitution {s.name!r}: non-declarative substitution events cannot be in a CCF group")


def ccf_level_probabilities(grp: CcfGroup) -> List[Tuple[int, Expr]]:
    """Probability expression of one CCF event of each level, by model
    (mcSCRAM src/ccf_group.cc:178-297): beta factor (1 - b) Q and b Q; MGL
    Q / C(n-1, i) times the factors of levels 2 .. i+1 and (1 - factor of
    level i+2) below the top level; alpha factor (i+1) / C(n-1, i) * a_(i+1)
    / sum_l l a_l * Q; phi factor f_l Q."""
    n = len(grp.members)
    q = grp.distribution
    one = Expr("value", [1.0])
    fs = [f for _, f in grp.factors]
    levels = [lv for lv, _ in grp.factors]
    if grp.model == "beta-factor":
        return [(1, Expr("mul", [Expr("sub", [one, fs[0]]), q])), (levels[0], Expr("mul", [fs[0], q]))]
    if grp.model == "phi-factor":
        return [(lv, Expr("mul", [f, q])) for lv, f in grp.factors]
    top = levels[-1]
    out = []
    if grp.model == "MGL":
        for i in range(top):
            args = [Expr("value", [1.0 / math.comb(n - 1, i)])] + fs[:i]
            if i < top - 1:
                args.append(Expr("sub", [one, fs[i]]))
            out.append((i + 1, Expr("mul", args + [q])))
        return out
    total = Expr("add", [Expr("mul", [Expr("value", [float(lv)]), f]) for lv, f in grp.factors])
    for i in range(top):
        out.append((i + 1, Expr("mul", [Expr("value", [float(i + 1)]), Expr("value", [1.0 / math.comb(n - 1, i)]),
                                        Expr("div", [fs[i], total]), q])))
    return out


def _expand_ccf(m: MefModel):
    """CCF analysis (mcSCRAM src/ccf_group.cc:141-175): each member becomes
    an OR gate, under the member's id, over the CCF events of every member
    combination of every level that contains it; a CCF event \"[a b ...]\"
    has the probability of its level."""
    import itertools

    as_gate = set()
    for grp in m.ccf_groups.values():
        args = {mid: [] for mid in grp.members}
        for level, prob in ccf_level_probabilities(grp):
            for combo in itertools.combinations(range(len(grp.members)), level):
                nm = "[" + " ".join(grp.member_names[j] for j in combo) + "]"
                ev = nm if grp.role == "public" or not grp.base else f"{grp.base}.{nm}"
                if ev in m.basic_events or ev in m.gates:
                    raise MefError(f"CCF event {ev!r} clashes with an element of that name")
                m.basic_events[ev] = prob
                for j in combo:
                    args[grp.members[j]].append((False, "basic-event", ev))
        for mid in grp.members:
            del m.basic_events[mid]
            m.gates[mid] = Formula(OR, args[mid])
            as_gate.add(mid)

    def retarget(f: Formula):
        f.args = [(c, "gate" if k == "basic-event" and x in as_gate else k, x) if k != "formula" else (c, k, x)
                  for c, k, x in f.args]
        for _, k, x in f.args:
            if k == "formula":
                retarget(x)

    for gid, f in m.gates.items():
        if gid not in as_gate:
            retarget(f)
    for ins in list(m.sequences.values()) + list(m.rules.values()):
        _walk_instructions(ins, lambda x: retarget(x[1]) if x[0] == "collect-formula" else None, {})
    for et in m.event_trees.values():
        for b in _branches_of(et):
            _walk_instructions(b.instructions, lambda x: retarget(x[1]) if x[0] == "collect-formula" else None, {})
    for s in m.substitutions.values():  # declarative ones: non-declarative events are never CCF members
        retarget(s.hypothesis)
        if not isinstance(s.target, bool) and s.target[2] in as_gate:
            s.target = (False, "gate", s.target[2])


def _branches_of(et: EventTree) -> List[Branch]:
    """Every branch of an event tree: named branches, the initial state and
    the paths of their forks."""
    out, todo = [], list(et.branches.values()) + [et.initial_state]
    while todo:
        b = todo.pop()
        out.append(b)
        if b.target[0] == "fork":
            todo.extend(p for _, p in b.target[1].paths)
    return out


def _validate(m: MefModel):
    """Cycles and the event-tree checks of mcSCRAM src/initializer.cc:1628-1791."""
    # gates
    edges: Dict[str, List[str]] = {}
    for gid, f in m.gates.items():
        refs: List[str] = []

        def walk(fm: Formula):
            for _, kind, x in fm.args:
                if kind == "gate":
                    refs.append(x)
                elif kind == "formula":
                    walk(x)

        walk(f)
        edges[gid] = refs
    c = _find_cycle(edges)
    if c is not None:
        raise MefError(f"gate {c!r} is part of a cycle")
    # rules
    redges = {}
    for rname, ins in m.rules.items():
        refs = []
        _walk_instructions(ins, lambda x: refs.append(x[1]) if x[0] == "rule" else None, {})
        redges[rname] = refs
    c = _find_cycle(redges)
    if c is not None:
        raise MefError(f"rule {c!r} is part of a cycle")
    for et in m.event_trees.values():
        where = f"event tree {et.name!r}"
        # named branches
        bedges = {}
        for bname, b in et.branches.items():
            refs = []
            todo = [b]
            while todo:
                x = todo.pop()
                if x.target[0] == "branch":
                    refs.append(x.target[1])
                elif x.target[0] == "fork":
                    todo.extend(p for _, p in x.target[1].paths)
            bedges[bname] = refs
        c = _find_cycle(bedges)
        if c is not None:
            raise MefError(f"{where}: branch {c!r} is part of a cycle")
    for et in m.event_trees.values():
        where = f"event tree {et.name!r}"
        order = {fe: i for i, fe in enumerate(et.functional_events)}
        for b in list(et.branches.values()) + [et.initial_state]:
            _check_fork_order(et, b, order, where)
            _links_only_in_sequences(m, b, where)
    # links: event tree -> event trees its sequences link to
    ledges = {name: sorted(_links_from(m, et)) for name, et in m.event_trees.items()}
    c = _find_cycle(ledges)
    if c is not None:
        raise MefError(f"event-tree link to {c!r} is part of a cycle")
    for et in m.event_trees.values():
        for b in list(et.branches.values()) + [et.initial_state]:
            _check_homogeneous(m, et, b, f"event tree {et.name!r}")


def _next_fork(et: EventTree, target) -> Optional[Fork]:
    seen = set()
    while target[0] == "branch" and target[1] not in seen:
        seen.add(target[1])
        target = et.branches[target[1]].target
    return target[1] if target[0] == "fork" else None


def _check_fork_order(et: EventTree, b: Branch, order: Dict[str, int], where: str):
    if b.target[0] != "fork":
        return
    fork = b.target[1]
    for _, path in fork.paths:
        _check_fork_order(et, path, order, where)
        nxt = _next_fork(et, path.target)
        if nxt is None:
            continue
        a, z = order[fork.functional_event], order[nxt.functional_event]
        if a == z:
            raise MefError(f"{where}: functional event {fork.functional_event!r} is duplicated in fork paths")
        if a > z:
            raise MefError(f"{where}: functional event {fork.functional_event!r} must appear after "
                           f"{nxt.functional_event!r} in fork paths")


def _links_only_in_sequences(m: MefModel, b: Branch, where: str):
    todo = [b]
    while todo:
        x = todo.pop()

        def fn(ins):
            if ins[0] == "link":
                raise MefError(f"{where}: link to {ins[1]!r} can only be used in end-state sequences")

        _walk_instructions(x.instructions, fn, m.rules)
        if x.target[0] == "fork":
            todo.extend(p for _, p in x.target[1].paths)


def _sequences_reached(et: EventTree) -> List[str]:
    out = []
    for b in _branches_of(et):
        if b.target[0] == "sequence" and b.target[1] not in out:
            out.append(b.target[1])
    return out


def _links_from(m: MefModel, et: EventTree) -> set:
    out = set()
    for s in _sequences_reached(et):
        _walk_instructions(m.sequences[s], lambda x: out.add(x[1]) if x[0] == "link" else None, m.rules)
    return out


def _check_homogeneous(m: MefModel, et: EventTree, b: Branch, where: str):
    kind = [None]
    visited_trees = set()

    def fn(ins):
        if ins[0] in ("collect-formula", "collect-expression"):
            if kind[0] is None:
                kind[0] = ins[0]
            elif kind[0] != ins[0]:
                raise MefError(f"{where}: mixed collect-expression and collect-formula")
        elif ins[0] == "link" and ins[1] not in visited_trees:
            visited_trees.add(ins[1])
            walk_branch(m.event_trees[ins[1]], m.event_trees[ins[1]].initial_state, set())

    def walk_branch(tree: EventTree, x: Branch, seen_branches: set):
        _walk_instructions(x.instructions, fn, m.rules)
        kind_, tgt = x.target
        if kind_ == "sequence":
            _walk_instructions(m.sequences[tgt], fn, m.rules)
        elif kind_ == "fork":
            for _, p in tgt.paths:
                walk_branch(tree, p, seen_branches)
        elif tgt not in seen_branches:
            seen_branches.add(tgt)
            walk_branch(tree, tree.branches[tgt], seen_branches)

    walk_branch(et, b, set())


def load(source: Union[str, Path], top: Optional[str] = None,
         mission_time: float = DEFAULT_MISSION_TIME, ccf_analysis: bool = False,
         allow_extern: bool = False) -> FlatGraph:
    """MEF document -> flattened graph of its top gate (probabilities at the
    mission time), root tallied."""
    return parse(source, mission_time, ccf_analysis, allow_extern).flat(top)


# Most time points of one probability curve: each point is one instance of a
# batched launch with its own threshold table held on the host and the device.
MAX_TIME_POINTS = 1 << 16


def time_points(mission_time: float, time_step: float) -> int:
    """Points t = 0, dt, 2 dt, ... below the mission time, plus the mission time."""
    return int(math.ceil(mission_time / time_step)) + 1 if time_step > 0 else 0


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
    if time_points(T, time_step) > MAX_TIME_POINTS:
        raise ValueError(f"time step {time_step} gives more than {MAX_TIME_POINTS} points up to {T}")
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


_SIL_PFD_BOUNDS = (1e-5, 1e-4, 1e-3, 1e-2, 1e-1, 1.0)  # SIL 4 .. 1, then beyond; lower bound 0
_SIL_PFH_BOUNDS = (1e-9, 1e-8, 1e-7, 1e-6, 1e-5, 1.0)


def _average_y(points) -> float:
    """Trapezoid integral of y over x divided by the x range (points are
    (y, x) in ascending x)."""
    area = sum((y1 + y0) * (x1 - x0) for (y0, x0), (y1, x1) in zip(points, points[1:])) / 2
    return area / (points[-1][1] - points[0][1])


def _partition_y(points, bounds) -> List[Tuple[float, float]]:
    """Share of the x range over which the piecewise-linear y lies in each
    bucket (lower, upper], the first bucket's lower bound being 0."""
    share = [0.0] * len(bounds)
    for (p0, t0), (p1, t1) in zip(points, points[1:]):
        k = (p1 - p0) / (t1 - t0)
        if k < 0:
            k, p0, p1 = -k, p1, p0
        b0 = 0.0
        for i, b1 in enumerate(bounds):
            if p0 <= b0 and b1 <= p1:  # the bucket lies inside the segment's y range
                share[i] += (b1 - b0) / k
            elif b0 <= p0 and p1 <= b1:  # the segment lies inside the bucket (k = 0 included)
                share[i] += t1 - t0
            elif p0 <= b0 <= p1:
                share[i] += (p1 - b0) / k
            elif p0 <= b1 <= p1:
                share[i] += (b1 - p0) / k
            b0 = b1
    span = points[-1][1] - points[0][1]
    return [(b, s / span) for b, s in zip(bounds, share)]


def safety_integrity_levels(curve) -> dict:
    """SIL metrics of a probability-over-time curve of (P(top), t) pairs, as
    the reference's ComputeSil makes them (mcSCRAM
    src/probability_analysis.cc:58-155): the average probability of failure
    on demand (PFD, the curve's time average), the average failure frequency
    per hour (PFH, the time average of P(t) / t, 0 at t = 0), and the share
    of the mission time spent in each SIL band, as (upper bound, fraction)
    pairs for the PFD bands 1e-5 .. 1 and the PFH bands 1e-9 .. 1.  A curve of
    one point puts its whole weight in the PFD band holding it."""
    curve = [(float(p), float(t)) for p, t in curve]
    if not curve:
        raise MefError("an empty probability curve")
    if len(curve) == 1:
        pfd = curve[0][0]
        band = next(i for i, b in enumerate(_SIL_PFD_BOUNDS) if pfd <= b)
        return {"pfd_avg": pfd, "pfh_avg": 0.0,
                "pfd_fractions": [(b, 1.0 if i == band else 0.0) for i, b in enumerate(_SIL_PFD_BOUNDS)],
                "pfh_fractions": [(b, 0.0) for b in _SIL_PFH_BOUNDS]}
    pfh = [(p / t if t else 0.0, t) for p, t in curve]
    return {"pfd_avg": _average_y(curve), "pfh_avg": _average_y(pfh),
            "pfd_fractions": _partition_y(curve, _SIL_PFD_BOUNDS),
            "pfh_fractions": _partition_y(pfh, _SIL_PFH_BOUNDS)}


def main(argv=None) -> int:
    """python -m mcscram_b200.mef MODEL.xml [--top GATE] [--samples N] [--mode strip|staged|fused] [--ccf]
    [--allow-extern] [--time-step DT [--sil]]: estimates the top-event probability of a MEF model on the GPU
    and prints it with its 95 % interval as one JSON line; with --time-step also the probability at t = 0,
    DT, ... and the mission time (one batched launch, --samples per time point up to 2^30), and with --sil
    the SIL metrics of that curve."""
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
    ap.add_argument("--ccf", action="store_true", help="expand common-cause groups (CCF analysis)")
    ap.add_argument("--allow-extern", action="store_true", help="load the model's extern libraries (runs their code)")
    ap.add_argument("--time-step", type=float, default=0.0, help="hours between points of the probability curve")
    ap.add_argument("--sil", action="store_true", help="SIL metrics of the probability curve (needs --time-step)")
    args = ap.parse_args(argv)
    if args.sil and args.time_step <= 0:
        ap.error("--sil needs --time-step")
    m = parse(args.model, ccf_analysis=args.ccf, allow_extern=args.allow_extern)
    if time_points(m.mission_time, args.time_step) > MAX_TIME_POINTS:
        ap.error(f"--time-step {args.time_step} gives more than {MAX_TIME_POINTS} points up to the mission time "
                 f"{m.mission_time}")
    g = m.flat(args.top)
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
    if args.time_step > 0:
        curve = probability_over_time(m, args.time_step, args.top, words=min(words, 1 << 24), device=args.device)
        out["p_time"] = [[pt, t] for pt, t in curve]
        if args.sil:
            out["sil"] = safety_integrity_levels(curve)
    print(json.dumps(out))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
