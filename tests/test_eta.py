"""Event-tree path: sequence collection and the combined PDAG checked against
an independent evaluation of the hand-written fixture (every construct of the
walk, by brute force over its basic events), the loader's checks against the
reference's lists of correct and incorrect event-tree inputs and its known
sequence probabilities (where the reference project is on disk), and on the
GPU the combined run: every tallied node bit-exact against the oracle, the
sequences of a complete tree partitioning the samples exactly, and the
convergence run within its error bars of the exact values."""
import itertools
import json
import math
from pathlib import Path

import pytest

from mcscram_b200 import eta, mef
from tests.conftest import reference_path

PLANT = Path(__file__).parent / "golden" / "eta" / "plant.xml"
REF = reference_path()
ETA_IN = REF / "tests" / "input" / "eta"
EVENT_TREES = REF / "input" / "EventTrees"
TWO32 = float(1 << 32)
SEQUENCES = ["OK", "CoreDamage", "SmallRelease", "LargeRelease"]

_PROB = {"tank": 0.01, "accumulator": 0.2, "pump-a": 0.1, "pump-b": 0.1, "pump-c": 0.1, "liner": 0.005,
         "iso-1": 0.02, "iso-2": 0.03, "spray-pump": 0.3, "spray-valve": 0.2, "spray-power": 0.1}


def _plant_exact(ie: str, large_break: bool, mission_time: float):
    """Sequence probabilities of the fixture, written out by hand from its
    XML: paths, house-event settings and links resolved on paper, each
    sequence the OR of its paths, evaluated over all 2^12 event states with
    the sampler's quantised probabilities."""
    prob = dict(_PROB, sump=1.0 - math.exp(-2e-5 * mission_time))
    names = sorted(prob)
    q = {n: math.floor(prob[n] * TWO32) / TWO32 for n in names}
    out = dict.fromkeys(SEQUENCES, 0.0)
    for bits in itertools.product([False, True], repeat=len(names)):
        x = dict(zip(names, bits))
        w = math.prod(q[n] if b else 1 - q[n] for n, b in zip(names, bits))
        pumps = x["pump-a"] + x["pump-b"] + x["pump-c"] >= 2
        inj = pumps or x["tank"] or (large_break and x["accumulator"])
        inj_broken = pumps or x["tank"] or x["accumulator"]  # set-house-event large-break = true
        inj_fail = inj_broken if ie == "LOCA" else inj
        rec = pumps or x["sump"]
        cont = (x["iso-1"] and x["iso-2"]) or x["liner"]
        n = x["spray-pump"] + x["spray-valve"] + x["spray-power"]
        spray = n >= 2 or (x["spray-valve"] and not x["spray-pump"])
        seq = {
            "OK": not inj and not rec,
            "CoreDamage": (not inj and rec and not cont) or (inj_fail and not cont),
            "SmallRelease": (not inj and rec and cont and not spray) or (inj_fail and cont and not spray),
            "LargeRelease": (not inj and rec and cont and spray) or (inj_fail and cont and spray),
        }
        for k, v in seq.items():
            if v:
                out[k] += w
    return out


def _phase(m, name):
    return m.with_phase(next(p for p in m.alignments["Mission"] if p.name == name))


@pytest.mark.parametrize("ie", ["LOCA", "Transient"])
@pytest.mark.parametrize("phase", [None, "Startup", "Power"])
def test_plant_sequences_exact(oracle_mod, ie, phase):
    m = mef.parse(PLANT)
    if phase is not None:
        m = _phase(m, phase)
    c = eta.combined_pdag(m, ie)
    assert [s.sequence for s, _ in c.sequences] == SEQUENCES
    g = c.flat()
    exact = _plant_exact(ie, phase == "Startup", m.mission_time)
    for k, (s, _) in enumerate(c.sequences):
        assert not s.is_expression_only
        got = oracle_mod.bdd_probability(g, root=int(g.tally_nodes[1 + k]))
        assert got == pytest.approx(exact[s.sequence], rel=1e-12, abs=1e-15), s.sequence
    if ie == "Transient" and phase != "Startup":  # the four sequences partition the outcomes
        assert sum(exact.values()) == pytest.approx(1.0, rel=1e-12)


def test_plant_scoping_and_watched_tops():
    m = mef.parse(PLANT)
    assert {"Injection.top", "Injection.pumps", "valves", "Containment.top", "Spray.top"} <= set(m.gates)
    assert "Containment.Isolation.iso-1" in m.basic_events and "Containment.Isolation.iso-p" in m.parameters
    assert m.fault_tree_tops("Containment") == ["Containment.top"]
    assert m.alignments["Mission"][0].time_fraction == 0.25
    c = eta.combined_pdag(m, "Transient")
    assert [w for w, _ in c.watched] == ["Spray.top", "Injection.top", "Recirculation.top", "Containment.top"]
    # the LOCA path collects Injection.top under large-break = true: a clone next to the original
    lo = eta.combined_pdag(m, "LOCA")
    assert any(k.startswith("__clone__") and k.endswith(".Injection.top") for k in lo.model.gates)
    assert not any(k.startswith("__clone__") for k in m.gates)  # the parsed model is left as it was


@pytest.mark.parametrize("xml,msg", [
    # a private gate is not known by its bare name outside its fault tree
    ("<opsa-mef><define-fault-tree name='F'><define-gate name='g' role='private'><or><house-event name='h'/>"
     "<house-event name='i'/></or></define-gate></define-fault-tree><define-fault-tree name='T'>"
     "<define-gate name='t'><and><gate name='g'/><house-event name='h'/></and></define-gate></define-fault-tree>"
     "<model-data><define-house-event name='h'/><define-house-event name='i'/></model-data></opsa-mef>",
     "unknown gate"),
    ("<opsa-mef><define-initiating-event name='I' event-tree='E'/><define-event-tree name='E'>"
     "<define-sequence name='S'/><initial-state><collect-expression><float value='0.7'/></collect-expression>"
     "<collect-expression><float value='0.9'/></collect-expression><fork functional-event='F'><path state='a'>"
     "<sequence name='S'/></path></fork></initial-state></define-event-tree></opsa-mef>",
     "undefined functional event"),
    ("<opsa-mef><define-alignment name='A'><define-phase name='p' time-fraction='0.5'/></define-alignment></opsa-mef>",
     "sum to"),
])
def test_event_tree_errors(xml, msg):
    with pytest.raises(mef.MefError, match=msg):
        mef.parse(xml)


def test_expression_sequences_and_phases():
    """Expression-only trees: a sequence's probability is the sum over its
    paths of the product of the collected expressions, evaluated at the
    phase's share of the mission time."""
    xml = """<opsa-mef>
      <define-initiating-event name="I" event-tree="E"/>
      <define-event-tree name="E">
        <define-functional-event name="F"/>
        <define-sequence name="A"/><define-sequence name="B"/>
        <initial-state><fork functional-event="F">
          <path state="up"><collect-expression><parameter name="q"/></collect-expression>
            <collect-expression><float value="0.5"/></collect-expression><sequence name="A"/></path>
          <path state="down"><collect-expression><sub><float value="1"/><parameter name="q"/></sub>
            </collect-expression><sequence name="B"/></path>
        </fork></initial-state>
      </define-event-tree>
      <model-data><define-parameter name="q"><exponential><float value="1e-4"/><system-mission-time/>
        </exponential></define-parameter></model-data>
      <define-alignment name="M"><define-phase name="one" time-fraction="0.4"/>
        <define-phase name="two" time-fraction="0.6"/></define-alignment>
    </opsa-mef>"""
    m = mef.parse(xml, mission_time=1000.0)
    for ph in m.alignments["M"]:
        mp = m.with_phase(ph)
        e = eta.EventTreeAnalysis(mp, "I")
        seqs = e.analyze()
        assert [s.sequence for s in seqs] == ["A", "B"] and all(s.is_expression_only for s in seqs)
        q = 1 - math.exp(-1e-4 * 1000.0 * ph.time_fraction)
        assert e.model.probability("__A") == pytest.approx(0.5 * q, rel=1e-14)
        assert e.model.probability("__B") == pytest.approx(1 - q, rel=1e-14)


# --- the reference's event-tree inputs (read only where the reference is on disk) ---

CORRECT = ["simplest_correct.xml", "public_sequence.xml", "initiating_event.xml", "set_house_event.xml",
           "collect_formula.xml", "single_expression.xml", "if_then_else_instruction.xml", "block_instruction.xml",
           "rule_instruction.xml", "link_instruction.xml", "link_in_rule.xml", "test_initiating_event.xml",
           "test_functional_event.xml"]
INCORRECT = ["doubly_defined_initiating_event.xml", "doubly_defined_event_tree.xml", "doubly_defined_sequence.xml",
             "doubly_defined_functional_event.xml", "doubly_defined_branch.xml", "doubly_defined_path_state.xml",
             "doubly_defined_rule.xml", "undefined_event_tree.xml", "undefined_sequence.xml",
             "undefined_branch.xml", "undefined_functional_event.xml", "undefined_rule.xml",
             "undefined_house_in_set_house.xml", "private_branch.xml", "private_functional_event.xml",
             "cyclic_branches_fork.xml", "cyclic_branches_self.xml", "cyclic_branches_transitive.xml",
             "cyclic_rule_block.xml", "cyclic_rule_self.xml", "cyclic_rule_transitive.xml", "cyclic_link_self.xml",
             "cyclic_link_transitive.xml", "invalid_duplicate_event_in_forks.xml",
             "invalid_event_order_in_branch.xml", "invalid_event_order_in_link.xml",
             "invalid_event_order_in_initial_state.xml", "invalid_event_order_in_ref_branch.xml",
             "invalid_collect_formula.xml", "invalid_link_undefined_event_tree.xml", "invalid_link_instruction.xml",
             "invalid_link_in_branch.xml", "invalid_link_in_rule.xml", "undefined_arg_collect_formula.xml",
             "mixing_collect_instructions.xml", "mixing_collect_instructions_link.xml",
             "mixing_collect_instructions_fork.xml"]
needs_ref = pytest.mark.skipif(not ETA_IN.exists(), reason="the reference's event-tree inputs are not on this machine")


@needs_ref
def test_reference_inputs_accepted_and_rejected():
    for name in CORRECT:
        mef.parse(ETA_IN / name)
    for name in INCORRECT:
        with pytest.raises(mef.MefError):
            mef.parse(ETA_IN / name)


# sequence probabilities the reference's own tests expect (tests/risk_analysis_tests.cc:428-482,
# tests/bench_core_tests.cc:546-555), and attack.xml worked out by hand from its parameters
KNOWN = [
    (["input/EventTrees/bcd.xml"], {"Success": 0.594, "Failure": 0.406}),
    (["input/EventTrees/attack.xml"], {"AttackSucceeds": 0.8 * (0.7 * 0.95 + 0.3), "AttackFails": 0.2 + 0.8 * 0.7 * 0.05}),
    (["tests/input/eta/single_expression.xml"], {"S": 0.5}),
    (["tests/input/eta/test_event_default.xml"], {"S": 0.5}),
    (["tests/input/eta/test_initiating_event.xml"], {"S": 0.5}),
    (["tests/input/eta/test_functional_event.xml"], {"S": 0.5}),
    (["tests/input/eta/test_functional_event_link.xml"], {"S": 0.5}),
]


@needs_ref
@pytest.mark.parametrize("files,expect", KNOWN, ids=[k[0][0].split("/")[-1] for k in KNOWN])
def test_reference_known_sequence_probabilities(oracle_mod, files, expect):
    m = mef.parse([REF / f for f in files])
    (ie,) = [i for i, t in m.initiating_events.items() if t]
    c = eta.combined_pdag(m, ie)
    assert {s.sequence for s, _ in c.sequences} == set(expect)
    g = c.flat()
    for k, (s, _) in enumerate(c.sequences):
        if s.is_expression_only:  # before quantisation: the collected expressions themselves
            assert c.model.probability(s.gate) == pytest.approx(expect[s.sequence], rel=1e-12)
        exact = oracle_mod.bdd_probability(g, root=int(g.tally_nodes[1 + k]))
        assert exact == pytest.approx(expect[s.sequence], abs=2.0 / TWO32)


@needs_ref
def test_reference_gas_leak_partition(oracle_mod):
    """The gas-leak tree (two files, linked) collects complementary formulas
    on every fork, so its sequences partition the outcomes."""
    m = mef.parse([EVENT_TREES / "gas_leak" / "gas_leak.xml", EVENT_TREES / "gas_leak" / "gas_leak_reactive.xml"])
    c = eta.combined_pdag(m, "Gas-Leak")
    g = c.flat()
    p = [oracle_mod.bdd_probability(g, root=int(g.tally_nodes[1 + k])) for k in range(len(c.sequences))]
    assert len(p) == 9 and sum(p) == pytest.approx(1.0, rel=1e-12)


# --- GPU -------------------------------------------------------------------

def _plant_graph(ie="Transient", phase="Power"):
    m = mef.parse(PLANT)
    if phase is not None:
        m = _phase(m, phase)
    return eta.combined_pdag(m, ie)


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["strip", "staged", "fused", "layered"])
@pytest.mark.parametrize("ie,phase", [("Transient", "Power"), ("LOCA", "Startup")])
def test_combined_tallies_match_oracle(oracle_mod, gpu, mode, ie, phase):
    from mcscram_b200 import _capi

    g = _plant_graph(ie, phase).flat()
    words = 1 << 14
    with _capi.Engine(g, mode=_capi.MODES[mode]) as e:
        e.run(3, 1, 0, words)
        ones, total = e.tallies()
    expect = oracle_mod.tallies(g, 3, 1, 0, words)
    assert total == words * 64
    assert [int(x) for x in ones] == [int(x) for x in expect]


@pytest.mark.gpu
def test_partition_counts_every_sample_once(gpu):
    """Transient in the Power phase: the four sequences partition the
    outcomes, so their tallies add up to the samples exactly and the OR root
    fires on every sample, at any size."""
    from mcscram_b200 import _capi

    c = _plant_graph("Transient", "Power")
    g = c.flat()
    words = 1 << 22
    with _capi.Engine(g, mode=_capi.MODE_STRIP) as e:
        e.run(1, 1, 0, words)
        ones, total = e.tallies()
    n_seq = len(c.sequences)
    assert int(ones[0]) == total == words * 64
    assert sum(int(x) for x in ones[1:1 + n_seq]) == total


@pytest.mark.gpu
@pytest.mark.parametrize("ie", ["LOCA", "Transient"])
def test_run_combined_converges_to_exact(oracle_mod, gpu, ie):
    from mcscram_b200 import host

    m = mef.parse(PLANT)
    s = host.Settings.default(num_trials=1 << 26, early_stop=0, ci_rel_margin_error=1e-9)
    r = eta.run_combined(m, ie, s)
    exact = _plant_exact(ie, False, m.mission_time)
    assert [q["sequence"] for q in r.sequences] == SEQUENCES
    for q in r.sequences:
        assert q["total_bits"] == 1 << 26
        sd = math.sqrt(exact[q["sequence"]] * (1 - exact[q["sequence"]]) / q["total_bits"])
        assert abs(q["mean"] - exact[q["sequence"]]) <= 5 * sd + 1e-12, q["sequence"]
    assert [gt["gate"] for gt in r.gates] == ["Spray.top", "Injection.top", "Recirculation.top", "Containment.top"]


@pytest.mark.gpu
def test_analyze_phases_and_cli(gpu, capsys):
    from mcscram_b200 import host

    m = mef.parse(PLANT)
    s = host.Settings.default(num_trials=1 << 22, early_stop=0, ci_rel_margin_error=1e-9)
    results, tops = eta.analyze(m, s)
    assert [(r.phase, r.initiating_event) for r in results] == [
        (("Mission", "Startup"), "LOCA"), (("Mission", "Startup"), "Transient"),
        (("Mission", "Power"), "LOCA"), (("Mission", "Power"), "Transient")]
    assert tops == {}  # every fault-tree top is tallied inside the combined runs
    for r in results:
        exact = _plant_exact(r.initiating_event, r.phase[1] == "Startup",
                             m.mission_time * (0.25 if r.phase[1] == "Startup" else 0.75))
        for q in r.sequences:
            sd = math.sqrt(exact[q["sequence"]] * (1 - exact[q["sequence"]]) / q["total_bits"])
            assert abs(q["mean"] - exact[q["sequence"]]) <= 5 * sd + 1e-12
    assert eta.main([str(PLANT), "--trials", str(1 << 20)]) == 0
    lines = [json.loads(x) for x in capsys.readouterr().out.splitlines()]
    assert len(lines) == 16 and {x["sequence"] for x in lines} == set(SEQUENCES)
