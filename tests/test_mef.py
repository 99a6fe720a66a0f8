"""MEF loader: a hand-written model with every construct the loader reads is
checked against a brute-force evaluation of the XML written here (not via
the loader), node numbering against the reference's first-encounter rule,
errors for what it does not read, and -- where the reference project is on
disk -- its Aralia models against the exact values listed in its benchmark
table, and its own test expectations: initializer input lists, core and
benchmark models, substitutions, extern functions, expressions, the
probability curve and SIL metrics.  The GPU tests run loaded models through
the engine."""
import csv
import itertools
import math
import xml.etree.ElementTree as ET
from pathlib import Path

import numpy as np
import pytest

from mcscram_b200 import mef
from tests.conftest import reference_path

FIX = Path(__file__).parent / "golden" / "mef" / "features.xml"
TWO32 = float(1 << 32)
ARALIA = reference_path("input", "Aralia")
TABLE = reference_path("benchmarks", "input.csv")


def _brute_force(path, top):
    """P(top) by enumerating the basic events, evaluating the XML directly."""
    root = ET.parse(path).getroot()
    gates = {g.get("name"): g[-1] for g in root.iter("define-gate")}
    params = {p.get("name"): float(p.find("float").get("value")) for p in root.iter("define-parameter")}
    house = {h.get("name"): h.find("constant").get("value") == "true" for h in root.iter("define-house-event")}
    prob = {}
    for b in root.iter("define-basic-event"):
        e = b[0]
        v = float(e.get("value")) if e.tag == "float" else params[e.get("name")]
        prob[b.get("name")] = np.floor(v * TWO32) / TWO32  # the sampler's quantised probability

    def ev(el, x):
        t = el.tag
        if t in ("gate", "event") and el.get("name") in gates:
            return ev(gates[el.get("name")], x)
        if t in ("basic-event", "event"):
            return x[el.get("name")]
        if t == "house-event":
            return house[el.get("name")]
        if t == "constant":
            return el.get("value") == "true"
        vals = [ev(c, x) for c in el]
        if t == "and":
            return all(vals)
        if t == "or":
            return any(vals)
        if t == "not":
            return not vals[0]
        if t == "xor":
            return sum(vals) % 2 == 1
        if t == "nand":
            return not all(vals)
        if t == "nor":
            return not any(vals)
        if t == "atleast":
            return sum(vals) >= int(el.get("min"))
        raise AssertionError(t)

    names = sorted(prob)
    total = 0.0
    for bits in itertools.product([False, True], repeat=len(names)):
        x = dict(zip(names, bits))
        w = np.prod([prob[n] if b else 1 - prob[n] for n, b in zip(names, bits)])
        total += w * ev(gates[top], x)
    return total


def test_features_model_exact(oracle_mod):
    g = mef.load(FIX, top="top")
    exact = _brute_force(FIX, "top")
    assert oracle_mod.bdd_probability(g) == pytest.approx(exact, rel=1e-12)


def test_numbering_follows_first_encounter():
    m = mef.parse(FIX)
    assert set(m.top_gates()) == {"top", "g_pass"}
    with pytest.raises(mef.MefError, match="top gates"):
        m.build()
    pdag, root, var_index, gate_index = m.build("top")
    # depth-first over top's arguments: g_and (a, b, g_nor (c)), g_atleast (b, c, e, (f)), g_xor (e, g_nand (a, f)), (d, a)
    assert var_index == {"a": 2, "b": 3, "c": 4, "e": 5, "f": 6, "d": 7}
    # then the house events, then the gates in pre-order (top first)
    assert root == 2 + len(var_index) + 3
    assert gate_index["g_and"] == root + 1 and gate_index["g_nor"] == root + 2
    assert pdag.event_order()  # the host layering accepts the PDAG


@pytest.mark.parametrize("xml,msg", [
    ("<opsa-mef><define-gate name='t'><and><basic-event name='x'/><basic-event name='y'/></and></define-gate>"
     "<define-basic-event name='y'><float value='0.1'/></define-basic-event></opsa-mef>", "unknown basic-event"),
    ("<opsa-mef><define-gate name='t'><or><event name='x'/><event name='y'/></or></define-gate>"
     "<define-basic-event name='y'><float value='0.1'/></define-basic-event></opsa-mef>", "unknown event"),
    ("<opsa-mef><define-basic-event name='x'><extern-function name='f'/></define-basic-event></opsa-mef>",
     "undefined extern function"),
    ("<opsa-mef><define-basic-event name='x'><exponential><float value='1'/></exponential>"
     "</define-basic-event></opsa-mef>", "takes 2 arguments"),
    ("<opsa-mef><define-gate name='t'><house-event name='h'/></define-gate>"
     "<define-gate name='t'><house-event name='h'/></define-gate></opsa-mef>", "defined twice"),
    ("<opsa-mef><define-gate name='t'><majority/></define-gate></opsa-mef>", "unsupported formula"),
    ("<opsa-mef><define-gate name='t'><and><basic-event name='x'/></and></define-gate></opsa-mef>",
     "2 or more arguments"),
    ("<opsa-mef><define-gate name='t'><atleast min='2'><house-event name='h'/><house-event name='i'/></atleast>"
     "</define-gate></opsa-mef>", "more arguments than its min"),
    ("<opsa-mef><define-gate name='t'><or><gate name='u'/><house-event name='h'/></or></define-gate>"
     "<define-gate name='u'><or><gate name='t'/><house-event name='h'/></or></define-gate>"
     "<define-house-event name='h'/></opsa-mef>", "cycle"),
    ("<opsa-mef><define-basic-event name='x'><float value='1.5'/></define-basic-event></opsa-mef>",
     "outside"),
    ("<model/>", "opsa-mef"),
])
def test_errors_name_the_problem(xml, msg):
    with pytest.raises(mef.MefError, match=msg):
        mef.parse(xml)


def _table():
    rows = list(csv.reader(TABLE.open(encoding="utf-8-sig")))[1:]
    return [(r[1], float(r[2])) for r in rows if float(r[2]) > 0]


# The listed value of das9204 does not belong to the model file: the file's
# exact probability is 2.1694e-11, and plain sampling of 2^30 of its samples
# finds no failure where the listed 6.08e-8 would give about 65.
_LISTED_INCONSISTENT = {"das9204.xml"}


@pytest.mark.skipif(not TABLE.exists(), reason="the reference's Aralia models are not on this machine")
def test_aralia_models_match_reference_values(oracle_mod):
    checked = 0
    sampled = []
    for name, listed in _table():
        g = mef.load(ARALIA / name)
        try:
            exact = oracle_mod.bdd_probability(g, max_nodes=1_000_000)
        except Exception:
            sampled.append((name, g, listed))  # BDD too large: checked by sampling below
            continue
        if name in _LISTED_INCONSISTENT:
            assert exact == pytest.approx(2.1694e-11, rel=1e-3)
            continue
        assert exact == pytest.approx(listed, rel=5e-5), name  # the table has six significant digits
        checked += 1
    assert checked >= 30
    for name, g, listed in sampled:
        W = 1 << 15
        hits = int(oracle_mod.tallies(g, 1, 1, 0, W)[0])
        n = W * 64
        sd = np.sqrt(listed * (1 - listed) / n)
        assert abs(hits / n - listed) <= 4 * sd + 1e-12, (name, hits / n, listed)


@pytest.mark.skipif(not TABLE.exists(), reason="the reference's Aralia models are not on this machine")
def test_das9204_listed_value_is_not_the_files(oracle_mod):
    g = mef.load(ARALIA / "das9204.xml")
    hits = int(oracle_mod.tallies(g, 1, 1, 0, 1 << 20)[0])
    assert hits <= 1  # 6.7e7 samples: ~4 expected at the listed 6.08e-8, ~0.001 at the file's value


@pytest.mark.gpu
def test_loaded_model_runs_bit_exact_on_gpu(capi, oracle_mod, gpu):
    g = mef.load(FIX, top="top")
    for mode in (capi.MODE_STRIP, capi.MODE_FUSED):
        with capi.Engine(g, mode=mode) as e:
            e.run(2, 1, 5, 20000)
            ones, total = e.tallies()
        assert np.array_equal(ones, oracle_mod.tallies(g, 2, 1, 5, 20000))
        assert total == 20000 * 64


@pytest.mark.gpu
def test_command_line_estimate_within_its_interval(gpu, capsys):
    import json
    assert mef.main([str(FIX), "--top", "top", "--samples", str(2 ** 26)]) == 0
    out = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    exact = _brute_force(FIX, "top")
    assert out["samples"] == 2 ** 26
    half = (out["ci95"][1] - out["ci95"][0]) / 2
    assert abs(out["p_top"] - exact) <= 2.1 * half  # a 4-sigma band around the 95 % half-width


TIMED = Path(__file__).parent / "golden" / "mef" / "timed.xml"


def test_time_dependent_expressions():
    import math
    m = mef.parse(TIMED)
    t = 1000.0
    assert m.probability("pump", t) == pytest.approx(1 - math.exp(-1e-4 * t), rel=1e-15)
    r = 3e-4 + 1e-2
    assert m.probability("valve", t) == pytest.approx((3e-4 - (3e-4 - 0.01 * r) * math.exp(-r * t)) / r, rel=1e-15)
    assert m.probability("sensor2", t) == pytest.approx(1 - math.exp(-4e-4 * t), rel=1e-15)
    assert m.probability("sensor3", 50.0) == 0.0
    assert m.probability("sensor3", t) == pytest.approx(1 - math.exp(-((t - 100) / 5000) ** 1.5), rel=1e-15)
    assert m.probability("demand", t) == 1e-3
    assert m.probability("pump") == pytest.approx(1 - math.exp(-1e-4 * 8760), rel=1e-15)  # default mission time
    g = mef.load(TIMED, mission_time=t)
    assert g.n_be == 6 and g.n_gates == 3


@pytest.mark.gpu
def test_probability_over_time_matches_oracle_per_time_point(oracle_mod, gpu):
    from mcscram_b200.graph import probability_threshold
    m = mef.parse(TIMED, mission_time=2000.0)
    W = 4096
    out = mef.probability_over_time(m, time_step=450.0, words=W, iteration=3)
    assert [t for _, t in out] == [0.0, 450.0, 900.0, 1350.0, 1800.0, 2000.0]
    pdag, root, var_index, _ = m.build()
    g = pdag.flatten([root])
    name_of = {idx: name for name, idx in var_index.items()}
    for p_hat, t in out:
        thr = probability_threshold(np.array([m.probability(name_of[int(x)], t) for x in g.be_pdag_idx]))
        ones = oracle_mod.tallies(g.with_thresholds(thr), 3, 1, 0, W)[0]
        assert p_hat == ones / (W * 64.0), t  # the same counters as a plain pass at that time's thresholds
    ps = [p for p, _ in out]
    assert all(b >= a for a, b in zip(ps, ps[1:]))  # same random numbers, rising probabilities: never decreasing


# The reference's initializer test lists for fault-tree inputs
# (tests/initializer_tests.cc:181-296).
FTA_IN = reference_path("tests", "input", "fta")
FTA_CORRECT = ["correct_tree_input.xml", "correct_formulas.xml", "constant_in_formulas.xml",
               "component_definition.xml", "mixed_definitions.xml", "mixed_roles.xml",
               "model_data_mixed_definitions.xml", "two_trees.xml", "two_top_events.xml",
               "two_top_through_formula.xml", "orphan_primary_event.xml", "very_long_mcs.xml",
               "unordered_structure.xml", "non_top_gate.xml", "unused_parameter.xml", "null_gate_with_label.xml",
               "case_sensitivity.xml", "missing_bool_constant.xml", "correct_tree_input_with_probs.xml",
               "trailing_spaces.xml", "flavored_types.xml", "mixed_references.xml", "ccf_unordered_factors.xml",
               "missing_ccf_level_number.xml", "weibull_lnorm_deviate_2p.xml", "weibull_lnorm_deviate_3p.xml",
               "correct_expressions.xml"]
FTA_UNSUPPORTED = {}
FTA_INCORRECT = ["invalid_probability.xml", "private_at_model_scope.xml", "doubly_defined_gate.xml",
                 "doubly_defined_house.xml", "doubly_defined_basic.xml", "doubly_defined_parameter.xml",
                 "doubly_defined_ccf_group.xml", "doubly_defined_component.xml", "extra_ccf_level_beta_factor.xml",
                 "missing_gate_definition.xml", "missing_ccf_factor.xml", "missing_ccf_members.xml",
                 "missing_arg_expression.xml", "undefined_event.xml", "undefined_basic_event.xml",
                 "undefined_house_event.xml", "undefined_gate.xml", "undefined_parameter.xml",
                 "reference_missing_fault_tree.xml", "reference_missing_component.xml", "wrong_parameter_unit.xml",
                 "name_clash_two_trees.xml", "def_clash_basic_gate.xml", "def_clash_house_gate.xml",
                 "def_clash_gate_primary.xml", "def_clash_basic_house.xml", "def_clash_house_basic.xml",
                 "atleast_gate.xml", "invalid_min_max_cardinality.xml", "cyclic_tree.xml", "cyclic_formula.xml",
                 "cyclic_parameter.xml", "cyclic_expression.xml", "invalid_expression.xml",
                 "invalid_periodic_test_num_args.xml", "repeated_child.xml", "repeated_attribute.xml",
                 "alpha_ccf_level_error.xml", "beta_ccf_level_error.xml", "mgl_ccf_level_error.xml",
                 "phi_ccf_wrong_sum.xml", "ccf_negative_factor.xml", "ccf_more_factors_than_needed.xml",
                 "ccf_wrong_distribution.xml", "repeated_ccf_members.xml", "duplicate_via_not.xml"]


@pytest.mark.skipif(not FTA_IN.exists(), reason="the reference's fault-tree inputs are not on this machine")
def test_reference_fault_tree_inputs_accepted_and_rejected():
    for name in FTA_CORRECT:
        mef.parse(FTA_IN / name)
        mef.parse(FTA_IN / name, ccf_analysis=True)
    for name, what in FTA_UNSUPPORTED.items():
        with pytest.raises(mef.MefError, match=what):
            mef.parse(FTA_IN / name)
    for name in FTA_INCORRECT:
        with pytest.raises(mef.MefError):
            mef.parse(FTA_IN / name)


CCF_FIX = Path(__file__).parent / "golden" / "mef" / "ccf.xml"


def _ccf_fixture_exact(ccf: bool) -> float:
    """P(top) of the CCF fixture by enumeration.  With CCF analysis the
    independent events are the common-cause events of the published models,
    written out here: alpha factor (non-staggered testing) Q_k = k /
    C(n-1, k-1) * a_k / sum_l l a_l * Q, beta factor (1 - b) Q for one valve
    and b Q for both; a member fails when any event that contains it does."""
    q = lambda p: math.floor(p * TWO32) / TWO32  # the sampler's quantised probability
    Qp, a = 0.05, {1: 0.8, 2: 0.15, 3: 0.05}
    at = sum(k * v for k, v in a.items())
    Qv, beta = 0.02, 0.1
    if ccf:
        events = {}
        for k in (1, 2, 3):
            for combo in itertools.combinations((1, 2, 3), k):
                events[("p",) + combo] = k / math.comb(2, k - 1) * a[k] / at * Qp
        events[("v", 1)] = events[("v", 2)] = (1 - beta) * Qv
        events[("v", 1, 2)] = beta * Qv
    else:
        events = {("p", 1): Qp, ("p", 2): Qp, ("p", 3): Qp, ("v", 1): Qv, ("v", 2): Qv}
    events[("power",)] = 0.01
    names = list(events)
    total = 0.0
    for bits in itertools.product([False, True], repeat=len(names)):
        x = dict(zip(names, bits))
        w = math.prod(q(events[n]) if b else 1 - q(events[n]) for n, b in zip(names, bits))
        pump = {i: any(v for n, v in x.items() if n[0] == "p" and i in n[1:]) for i in (1, 2, 3)}
        valve = {i: any(v for n, v in x.items() if n[0] == "v" and i in n[1:]) for i in (1, 2)}
        top = ((pump[1] or valve[1]) and (pump[2] or valve[2])) or (pump[3] and x[("power",)])
        total += w * top
    return total


@pytest.mark.parametrize("ccf", [False, True])
def test_ccf_fixture_exact(oracle_mod, ccf):
    g = mef.load(CCF_FIX, ccf_analysis=ccf)
    assert oracle_mod.bdd_probability(g) == pytest.approx(_ccf_fixture_exact(ccf), rel=1e-9)
    m = mef.parse(CCF_FIX, ccf_analysis=ccf)
    assert ("[pump1 pump2 pump3]" in m.basic_events) == ccf and ("pump1" in m.gates) == ccf


def test_ccf_errors():
    grp = ("<opsa-mef><define-fault-tree name='f'><define-gate name='t'><and><basic-event name='a'/>"
           "<basic-event name='b'/></and></define-gate><define-CCF-group name='g' model='{model}'><members>"
           "<basic-event name='a'/><basic-event name='b'/></members><distribution><float value='0.1'/>"
           "</distribution>{factors}</define-CCF-group></define-fault-tree></opsa-mef>")
    cases = [("MGL", "<factor level='1'><float value='0.1'/></factor>", "below the minimum"),
             ("alpha-factor", "<factor level='3'><float value='0.1'/></factor>", "above the 2 members"),
             ("phi-factor", "<factors><factor><float value='0.5'/></factor><factor><float value='0.4'/></factor>"
                            "</factors>", "sum to"),
             ("alpha-factor", "<factor level='2'><float value='0.1'/></factor>", "missing CCF factors"),
             ("gamma", "<factor level='2'><float value='0.1'/></factor>", "unknown model")]
    for model, factors, msg in cases:
        with pytest.raises(mef.MefError, match=msg):
            mef.parse(grp.format(model=model, factors=factors))


CORE_IN = reference_path("tests", "input", "core")


@pytest.mark.skipif(not CORE_IN.exists(), reason="the reference's core inputs are not on this machine")
@pytest.mark.parametrize("name,expect", [("beta_factor_ccf.xml", 0.04308), ("phi_factor_ccf.xml", 0.04104),
                                         ("mgl_ccf.xml", 0.01630), ("alpha_factor_ccf.xml", 0.05298)])
def test_reference_ccf_models(oracle_mod, name, expect):
    """The exact top-event probabilities the reference's tests expect with CCF
    analysis on (tests/bench_core_tests.cc:452-527, to their 1e-5)."""
    g = mef.load(CORE_IN / name, ccf_analysis=True)
    assert oracle_mod.bdd_probability(g) == pytest.approx(expect, abs=1e-5)


@pytest.mark.gpu
def test_ccf_model_through_the_engine(oracle_mod, gpu):
    from mcscram_b200 import _capi
    g = mef.load(CCF_FIX, ccf_analysis=True)
    with _capi.Engine(g, mode=_capi.MODE_STRIP) as e:
        e.run(2, 1, 0, 1 << 14)
        ones, total = e.tallies()
    assert int(ones[0]) == int(oracle_mod.tallies(g, 2, 1, 0, 1 << 14)[0])


DEV_FIX = Path(__file__).parent / "golden" / "mef" / "deviates.xml"


def test_deviate_point_values_and_moments():
    """Point values are the distributions' means (as the reference's value()),
    and 200,000 draws have the distributions' means and variances; a deviate
    reached through two parameters is drawn once per trial."""
    m = mef.parse(DEV_FIX, mission_time=1000.0)
    z95 = 1.6448536269514722
    s_log = math.log(3) / z95
    theory = {  # (mean, variance) of each parameter's distribution
        "lambda": (2e-4, (2e-4) ** 2 * (math.exp(s_log ** 2) - 1)),
        "log2": (math.exp(-2.5 + 0.08), (math.exp(0.16) - 1) * math.exp(-5 + 0.16)),
        "gamma": (0.1, 2 * 0.05 ** 2),
        "beta": (0.1, 2 * 18 / (20 ** 2 * 21)),
        "normal": (0.1, 0.01 ** 2),
        "uniform": (0.002, 0.002 ** 2 / 12),
        "histogram": ((0.0005 * 3 + 0.0025 * 1) / 4, None),
    }
    for name, (mu, _) in theory.items():
        assert m.parameters[name].value(1000.0, m.parameters) == pytest.approx(mu, rel=1e-12), name
    n = 200_000
    d = mef.sample_expressions(m, {k: m.parameters[k] for k in list(theory) + ["lambda-alias"]}, n,
                               np.random.default_rng(3))
    for name, (mu, var) in theory.items():
        x = d[name]
        sd = math.sqrt(var) if var is not None else x.std()
        assert abs(x.mean() - mu) <= 5 * sd / math.sqrt(n), name
        if var is not None:
            assert x.var() == pytest.approx(var, rel=0.05), name
    assert np.array_equal(d["lambda"], d["lambda-alias"])
    h = d["histogram"]
    assert np.all((h >= 0) & (h <= 0.004)) and abs(np.mean(h < 0.001) - 0.75) < 0.01
    b = mef.sample_expressions(m, {"a": m.basic_events["e-log3"], "b": m.basic_events["e-log3-again"]}, 10,
                               np.random.default_rng(1))
    np.testing.assert_allclose(-np.log1p(-b["a"]) / 1000.0, -np.log1p(-b["b"]) / 2000.0, rtol=1e-9)


@pytest.mark.parametrize("body,msg", [
    ("<uniform-deviate><float value='2'/><float value='1'/></uniform-deviate>", "min is not below max"),
    ("<normal-deviate><float value='0.1'/><float value='0'/></normal-deviate>", "not positive"),
    ("<lognormal-deviate><float value='0.1'/><float value='0.5'/><float value='0.95'/></lognormal-deviate>",
     "error factor"),
    ("<gamma-deviate><float value='0'/><float value='1'/></gamma-deviate>", "must be positive"),
    ("<histogram><float value='0'/><bin><float value='0'/><float value='1'/></bin></histogram>", "increase"),
    ("<beta-deviate><float value='1'/></beta-deviate>", "takes 2 arguments"),
])
def test_deviate_domain_errors(body, msg):
    with pytest.raises(mef.MefError, match=msg):
        mef.parse(f"<opsa-mef><define-parameter name='p'>{body}</define-parameter></opsa-mef>")


SMALL_TREE = reference_path("input", "SmallTree", "SmallTree.xml")


@pytest.mark.skipif(not SMALL_TREE.exists(), reason="the reference's SmallTree model is not on this machine")
def test_reference_small_tree_uncertainty(oracle_mod):
    """The reference's uncertainty test on its SmallTree model
    (tests/bench_small_tree_tests.cc:22-40): point value 0.02678 (1e-5), and
    over 10,000 trials of its lognormal deviates a mean of 0.0253 (1e-3) and a
    sigma of 0.022 (2e-3), here from exact per-trial probabilities."""
    m = mef.parse(SMALL_TREE)
    g = m.flat()
    assert oracle_mod.bdd_probability(g) == pytest.approx(0.02678, abs=1e-5)
    _, _, var_index, _ = m.build()
    d = mef.sample_expressions(m, {n: m.basic_events[n] for n in var_index}, 10_000, np.random.default_rng(11))
    p = {n: d[n] for n in var_index}
    top = 1 - (1 - p["e1"] * p["e2"]) * (1 - p["e3"] * p["e4"])  # the model's two cut sets, exactly
    assert top.mean() == pytest.approx(0.0253, abs=1e-3)
    assert top.std(ddof=1) == pytest.approx(0.022, abs=2e-3)


@pytest.mark.gpu
def test_mef_uncertainty_on_the_gpu(oracle_mod, gpu):
    """Trials of the deviate fixture run as one batch: every trial's count
    bit-exact against the oracle at its sampled thresholds, and the mean of
    the estimates within 5 sigma (of one trial, the errors being correlated)
    of the mean of the exact trial values."""
    m = mef.parse(DEV_FIX, mission_time=1000.0)
    trials, words = 400, 1 << 12
    r = mef.uncertainty(m, trials=trials, words=words, seed=7, iteration=2)
    g = r["graph"]
    exact = np.array([oracle_mod.bdd_probability(g.with_thresholds(t)) for t in r["thresholds"]])
    for k in (0, 1, 2, 3, 4, 199, 399):
        want = int(oracle_mod.tallies(g.with_thresholds(r["thresholds"][k]), 2, 1, 0, words)[0])
        assert int(round(r["p_top"][k] * words * 64)) == want, k
    # the trials share their counters (as a fresh manager per trial would), so
    # their sampling errors are correlated: bound the mean by one trial's error
    se = float(np.mean(np.sqrt(exact * (1 - exact) / (words * 64))))
    assert abs(r["stats"]["mean"] - exact.mean()) <= 5 * se + 1e-12
    assert r["stats"]["sigma"] == pytest.approx(exact.std(ddof=1), rel=0.1)


# (arguments, value) of the reference's periodic-test cases
# (tests/expression_tests.cc:216-324), to their 1e-5
_PERIODIC = [
    ((0.1, 1, 2, 5), 1 - math.exp(-0.1)),
    ((7e-4, 4e-4, 4020, 4740, 8760), 0.817508),
    ((7e-4, 4e-4, 2010, 4740, 8760), 0.736611),
    ((7e-4, 4e-4, 120, 4740, 8760), 0.645377),
    ((7e-4, 7e-4, 120, 4740, 8760), 0.511579),   # mu == lambda
    ((7e-4, 0.0, 120, 4740, 8760), 0.997828),    # no repair
    ((7e-4, 6e-4, 4e-4, 120, 4740, 0.01, 20, 1, 0.9, 0.01, 8760), 0.668316),
    ((7e-4, 6e-4, 4e-4, 120, 4740, 0.01, 20, 0, 0.9, 0.01, 8760), 0.668316),
    ((7e-4, 6e-4, 4e-4, 120, 4740, 0.01, 20, 0, 0.9, 0.01, 4750), 1.0),
    ((7e-4, 6e-4, 4e-4, 120, 4740, 0.01, 20, 0, 0.9, 0.01, 4870), 0.996715),
    ((7e-4, 6e-4, 4e-4, 120, 4740, 0.01, 20, 0, 0.9, 0.01, 8710), 0.997478),
    ((7e-4, 7e-4, 7e-4, 120, 4740, 0.01, 20, 1, 0.9, 0.01, 8760), 0.543401),
    ((7e-4, 6e-4, 4e-4, 120, 4740, 0.01, 120, 1, 0.9, 0.01, 8760), 0.6469),
    ((7e-4, 6e-4, 4e-4, 4020, 4740, 0.0, 0, 1, 1.0, 0.0, 8760), 0.817508),
    ((7e-4, 6e-4, 4e-4, 120, 4740, 0.0, 0, 1, 1.0, 0.0, 8760), 0.645377),
]


@pytest.mark.parametrize("args,want", _PERIODIC)
def test_periodic_test_values(args, want):
    assert mef.periodic_test(*args) == pytest.approx(want, abs=1e-5)


def test_periodic_test_in_a_model():
    """The 5-argument form read from MEF, its point value and its draws when
    its failure rate is a deviate; a huge repair rate gives the 4-argument
    form."""
    xml = ("<opsa-mef><define-basic-event name='pump'><periodic-test><parameter name='lam'/>"
           "<float value='4e-4'/><float value='4020'/><float value='4740'/><system-mission-time/></periodic-test>"
           "</define-basic-event><define-parameter name='lam'>{}</define-parameter></opsa-mef>")
    m = mef.parse(xml.format("<float value='7e-4'/>"), mission_time=8760.0)
    assert m.probability("pump") == pytest.approx(0.817508, abs=1e-5)
    m = mef.parse(xml.format("<uniform-deviate><float value='6e-4'/><float value='8e-4'/></uniform-deviate>"),
                  mission_time=8760.0)
    d = mef.sample_expressions(m, {"pump": m.basic_events["pump"], "lam": m.parameters["lam"]}, 50,
                               np.random.default_rng(2))
    for lam, val in zip(d["lam"], d["pump"]):
        assert val == pytest.approx(mef.periodic_test(lam, 4e-4, 4020, 4740, 8760), rel=1e-12)
    assert mef.periodic_test(7e-4, 1e300, 120, 4740, 8760) == pytest.approx(
        mef.periodic_test(7e-4, 120, 4740, 8760), abs=1e-5)
    with pytest.raises(mef.MefError, match="takes 4, 5 or 11"):
        mef.parse("<opsa-mef><define-parameter name='p'><periodic-test><float value='1'/>"
                  "<float value='1'/></periodic-test></define-parameter></opsa-mef>")


@pytest.mark.parametrize("body,want", [
    ("<abs><float value='-0.25'/></abs>", 0.25),
    ("<sqrt><float value='0.09'/></sqrt>", 0.3),
    ("<log10><float value='1e-3'/></log10>", -3.0),
    ("<exp><log><float value='0.2'/></log></exp>", 0.2),
    ("<pow><float value='0.5'/><int value='3'/></pow>", 0.125),
    ("<mod><int value='-7'/><int value='3'/></mod>", -1.0),  # truncated, as C++ % on ints
    ("<mean><float value='0.1'/><float value='0.3'/><float value='0.5'/></mean>", 0.3),
    ("<max><float value='0.1'/><float value='0.3'/></max>", 0.3),
    ("<floor><float value='2.7'/></floor>", 2.0),
    ("<atan><tan><float value='0.4'/></tan></atan>", 0.4),
    ("<switch><case><bool value='false'/><float value='0.1'/></case><case><bool value='true'/><float value='0.2'/>"
     "</case><case><bool value='true'/><float value='0.3'/></case><float value='0.4'/></switch>", 0.2),
    ("<switch><case><bool value='false'/><float value='0.1'/></case><float value='0.4'/></switch>", 0.4),
])
def test_numeric_expressions(body, want):
    """The MEF's numeric built-ins and switch, as point values and as the
    vectorised form the uncertainty draws use."""
    m = mef.parse(f"<opsa-mef><define-parameter name='p'>{body}</define-parameter></opsa-mef>")
    assert m.parameters["p"].value(m.mission_time, m.parameters) == pytest.approx(want, rel=1e-12, abs=1e-15)
    d = mef.sample_expressions(m, {"p": m.parameters["p"]}, 3, np.random.default_rng(0))
    np.testing.assert_allclose(d["p"], want, rtol=1e-12, atol=1e-15)


@pytest.mark.parametrize("body", ["<log><float value='0'/></log>", "<sqrt><float value='-1'/></sqrt>",
                                  "<acos><float value='2'/></acos>", "<mod><int value='3'/><int value='0'/></mod>",
                                  "<div><float value='1'/><float value='0'/></div>"])
def test_numeric_domain_errors(body):
    with pytest.raises(mef.MefError, match="outside its domain"):
        mef.parse(f"<opsa-mef><define-parameter name='p'>{body}</define-parameter></opsa-mef>")


SUB_FIX = Path(__file__).parent / "golden" / "mef" / "substitution.xml"


def _substitution_fixture_exact() -> float:
    """P(top AND the declarative substitutions' implications) of the
    substitution fixture by enumeration, from its formulas written out here:
    top = atleast 2 of the pumps or the heat exchanger; no two of pump a,
    pump b and maintenance; pumps b and c imply the operator's failure; the
    heat exchanger implies the backup's; pump a or the heat exchanger imply
    the alarm's.  The non-declarative exchange event changes nothing."""
    q = lambda p: math.floor(p * TWO32) / TWO32  # the sampler's quantised probability
    p = {"a": 0.3, "b": 0.25, "c": 0.2, "hx": 0.05, "maint": 0.1, "op": 0.4, "backup": 0.6, "alarm": 0.9}
    names = list(p)
    total = 0.0
    for bits in itertools.product([False, True], repeat=len(names)):
        x = dict(zip(names, bits))
        w = math.prod(q(p[n]) if b else 1 - q(p[n]) for n, b in zip(names, bits))
        top = (x["a"] + x["b"] + x["c"] >= 2) or x["hx"]
        ok = (x["a"] + x["b"] + x["maint"] < 2) and (not (x["b"] and x["c"]) or x["op"]) and \
            (not x["hx"] or x["backup"]) and (not (x["a"] or x["hx"]) or x["alarm"])
        total += w * (top and ok)
    return total


def test_substitution_fixture_exact(oracle_mod):
    m = mef.parse(SUB_FIX)
    assert [mef.substitution_type(s) for s in m.substitutions.values()] == [
        "delete-terms", "recovery-rule", None, None, "exchange-event"]
    pdag, root, var_index, gate_index = m.build("top")
    assert gate_index["top"] != root  # the analysed root is AND(implications..., top)
    # the top's events first, then the substitutions' in definition order (GatherVariables)
    assert list(var_index)[:9] == ["pump_a", "pump_b", "pump_c", "heat_exchanger", "maintenance",
                                   "operator_fails", "backup_fails", "alarm_fails", "valve_x"]
    g = mef.load(SUB_FIX)
    assert g.n_be == 8  # the non-declarative substitution's events are not in the graph
    assert oracle_mod.bdd_probability(g) == pytest.approx(_substitution_fixture_exact(), rel=1e-9)


def test_substitution_errors():
    model = ("<opsa-mef><define-substitution name='s'{attr}><hypothesis>{hyp}</hypothesis>{src}<target>{tgt}"
             "</target></define-substitution><model-data>" +
             "".join(f"<define-basic-event name='{n}'><float value='0.1'/></define-basic-event>" for n in "abcd") +
             "</model-data></opsa-mef>")
    ab = "<and><basic-event name='a'/><basic-event name='b'/></and>"
    d = "<basic-event name='d'/>"
    cases = [("", "<xor><basic-event name='a'/><basic-event name='b'/></xor>", "", d, "must be coherent"),
             ("", ab, "", "<constant value='true'/>", "no effect"),
             ("", ab, "<source><basic-event name='c'/></source>", "<constant value='false'/>", "irrelevant"),
             ("", "<atleast min='2'><basic-event name='a'/><basic-event name='b'/><basic-event name='c'/></atleast>",
              "<source><basic-event name='c'/></source>", d, "AND/OR/NULL"),
             (" type='exchange-event'", ab, "", d, "does not match"),
             ("", "<and><basic-event name='a'/><gate name='b'/></and>", "", d, "unknown gate"),
             ("", ab, "<source><basic-event name='c'/><basic-event name='c'/></source>", d, "listed twice")]
    for attr, hyp, src, tgt, msg in cases:
        with pytest.raises(mef.MefError, match=msg):
            mef.parse(model.format(attr=attr, hyp=hyp, src=src, tgt=tgt))


TWO_TRAIN = reference_path("input", "TwoTrain")


@pytest.mark.skipif(not TWO_TRAIN.exists(), reason="the reference's TwoTrain model is not on this machine")
def test_reference_two_train_substitutions(oracle_mod):
    """The exact probabilities the reference's tests expect of its two-train
    model, plain and with declarative substitutions (tests/bench_two_train_tests.cc:
    24-72); its non-declarative substitutions leave the Monte Carlo graph as
    the plain model's."""
    assert oracle_mod.bdd_probability(mef.load(TWO_TRAIN / "two_train.xml")) == pytest.approx(0.7225, rel=1e-9)
    assert oracle_mod.bdd_probability(mef.load(TWO_TRAIN / "substitutions.xml")) == pytest.approx(0.329175, rel=1e-9)
    assert oracle_mod.bdd_probability(mef.load(TWO_TRAIN / "nondeclarative_substitutions.xml")) == \
        pytest.approx(0.7225, rel=1e-9)


MODEL_IN = reference_path("tests", "input", "model")
MODEL_CORRECT = ["extern_library.xml", "extern_function.xml", "extern_expression.xml", "valid_alignment.xml",
                 "valid_sum_alignment.xml", "private_phases.xml", "substitution.xml",
                 "substitution_optional_source.xml", "substitution_types.xml",
                 "substitution_declarative_target_is_another_source.xml", "substitution_target_is_hypothesis.xml",
                 "substitution_declarative_ccf.xml"]
MODEL_INCORRECT = [
    "duplicate_extern_libraries.xml", "duplicate_extern_functions.xml", "undefined_extern_library.xml",
    "invalid_num_param_extern_function.xml", "undefined_extern_function.xml",
    "invalid_num_args_extern_expression.xml", "extern_library_invalid_path_format.xml", "duplicate_phases.xml",
    "invalid_phase_fraction.xml", "zero_phase_fraction.xml", "negative_phase_fraction.xml",
    "undefined_target_set_house_event.xml", "duplicate_alignment.xml", "excess_alignment.xml",
    "incomplete_alignment.xml", "duplicate_substitution.xml", "substitution_undefined_hypothesis_event.xml",
    "substitution_undefined_source_event.xml", "substitution_undefined_target_event.xml",
    "substitution_duplicate_source_event.xml", "substitution_duplicate_hypothesis_event.xml",
    "substitution_nested_formula.xml", "substitution_non_basic_event_formula.xml", "substitution_type_mismatch.xml",
    "substitution_no_effect.xml", "substitution_nondeclarative_complex.xml", "substitution_source_equal_target.xml",
    "substitution_target_is_another_source.xml", "substitution_target_is_another_hypothesis.xml",
    "substitution_source_is_another_hypothesis.xml", "substitution_source_false_target.xml",
    "substitution_declarative_noncoherent.xml", "substitution_nondeclarative_ccf_hypothesis.xml",
    "substitution_nondeclarative_ccf_source.xml", "substitution_nondeclarative_ccf_target.xml",
    "empty_extern_function.xml", "empty_alignment.xml", "extern_library_ioerror.xml",
    "undefined_symbol_extern_function.xml"]

# a stand-in for the reference's test library: the symbols its model inputs name
_DUMMY_EXTERN = "int foo(void) { return 42; }\ndouble bar(void) { return 42; }\ndouble identity(double x) { return x; }\n"


def _shared_library(source: str, out: Path):
    import shutil
    import subprocess
    if shutil.which("gcc") is None:
        pytest.skip("no C compiler for the extern-function library")
    out.parent.mkdir(parents=True, exist_ok=True)
    src = out.with_suffix(".c")
    src.write_text(source)
    subprocess.run(["gcc", "-shared", "-fPIC", "-O1", "-o", str(out), str(src)], check=True)


@pytest.mark.skipif(not MODEL_IN.exists(), reason="the reference's model inputs are not on this machine")
def test_reference_model_inputs_accepted_and_rejected(tmp_path):
    """The reference's initializer lists of correct and incorrect model
    inputs (tests/initializer_tests.cc:332-414), read with extern libraries
    allowed; the inputs are copied beside a library of the symbols they name,
    at the relative path they load it from."""
    _shared_library(_DUMMY_EXTERN, tmp_path / "build" / "lib" / "scram" / "libscram_dummy_extern.so")
    d = tmp_path / "tests" / "input" / "model"
    d.mkdir(parents=True)
    for f in MODEL_IN.glob("*.xml"):
        (d / f.name).write_text(f.read_text())
    for name in MODEL_CORRECT:
        mef.parse(d / name, allow_extern=True)
    m = mef.parse(d / "extern_expression.xml", allow_extern=True)
    assert {k: e.value(0.0, m.parameters) for k, e in m.parameters.items()} == {
        "param1": 1.0, "param2": 42.0, "param": 42.0}
    for name in MODEL_INCORRECT:
        with pytest.raises(mef.MefError):
            mef.parse(d / name, allow_extern=True)
    with pytest.raises(mef.MefError, match="disallowed"):  # DefaultExternDisable
        mef.parse(d / "extern_library.xml")
    g = mef.load(d / "extern_full_check.xml", allow_extern=True)
    assert float(g.quantised_probabilities()[0]) == pytest.approx(0.1, abs=1e-9)


_SCALE_EXTERN = "double scale(double p, int n) { return p / n; }\nint twice(int x) { return 2 * x; }\n"


def test_extern_functions_in_a_model(oracle_mod, tmp_path):
    """Extern functions with int and double parameters: arguments convert as
    C++ converts them (2.9 -> 2, 3.7 -> 3), values feed basic events, and
    the uncertainty draws call them once per trial."""
    _shared_library(_SCALE_EXTERN, tmp_path / "lib" / "libscale.so")
    xml = tmp_path / "m.xml"
    xml.write_text(
        "<opsa-mef><define-extern-library name='l' path='lib/scale' decorate='true'/>"
        "<define-extern-function name='scale' symbol='scale' library='l'><double/><double/><int/>"
        "</define-extern-function><define-extern-function name='twice' symbol='twice' library='l'><int/><int/>"
        "</define-extern-function><define-fault-tree name='f'><define-gate name='top'><or>"
        "<basic-event name='e1'/><basic-event name='e2'/></or></define-gate>"
        "<define-basic-event name='e1'><extern-function name='scale'><float value='0.9'/><float value='3.7'/>"
        "</extern-function></define-basic-event>"
        "<define-basic-event name='e2'><div><float value='1'/><extern-function name='twice'>"
        "<float value='2.9'/></extern-function></div></define-basic-event>"
        "<define-basic-event name='e3'><extern-function name='scale'><uniform-deviate><float value='0.2'/>"
        "<float value='0.4'/></uniform-deviate><int value='2'/></extern-function></define-basic-event>"
        "</define-fault-tree></opsa-mef>")
    m = mef.parse(xml, allow_extern=True)
    assert m.probability("e1") == pytest.approx(0.3, rel=1e-15)
    assert m.probability("e2") == pytest.approx(0.25, rel=1e-15)
    assert m.probability("e3") == pytest.approx(0.15, rel=1e-15)  # the deviate's mean
    g = mef.load(xml, allow_extern=True)
    q = lambda p: math.floor(p * TWO32) / TWO32
    assert oracle_mod.bdd_probability(g) == pytest.approx(1 - (1 - q(0.3)) * (1 - q(0.25)), rel=1e-9)
    d = mef.sample_expressions(m, {"e3": m.basic_events["e3"]}, 2000, np.random.default_rng(3))["e3"]
    assert d.min() >= 0.1 and d.max() <= 0.2 and abs(d.mean() - 0.15) < 0.005
    with pytest.raises(mef.MefError, match="disallowed"):
        mef.parse(xml)
    for path, msg in [("", "invalid library path"), ("lib/", "invalid library path"), ("lib:", "invalid library path"),
                      ("..", "invalid library path"), ("lib/none", "cannot open")]:
        with pytest.raises(mef.MefError, match=msg):
            mef.parse(f"<opsa-mef><define-extern-library name='l' path='{path}'/></opsa-mef>", allow_extern=True)


@pytest.mark.gpu
def test_substitution_model_through_the_engine(oracle_mod, gpu):
    from mcscram_b200 import _capi
    g = mef.load(SUB_FIX)
    with _capi.Engine(g, mode=_capi.MODE_STRIP) as e:
        e.run(2, 1, 0, 1 << 14)
        ones, total = e.tallies()
    assert int(ones[0]) == int(oracle_mod.tallies(g, 2, 1, 0, 1 << 14)[0])
    p = int(ones[0]) / total
    assert abs(p - _substitution_fixture_exact()) <= 5 * math.sqrt(p * (1 - p) / total)


INPUT_DIR = reference_path("tests", "input")


@pytest.mark.skipif(not INPUT_DIR.exists(), reason="the reference's test inputs are not on this machine")
def test_reference_document_level_inputs():
    """The reference's document-level initializer cases
    (tests/initializer_tests.cc:28-103, 174-180, 213-247, 306-330): malformed
    XML, foreign namespaces, what its schema rejects (nested formulas, blank
    labels and attribute values, ints beyond 32 bits), XIncludes, the same
    file twice; and the inputs it reads."""
    rejected = ["xml_formatting_error.xml", "undefined_xmlns.xml", "custom_xmlns.xml", "schema_fail.xml",
                "fta/nested_formula.xml", "fta/nested_not_not.xml", "fta/nested_not_constant.xml",
                "unsupported_feature.xml", "unsupported_gate.xml", "unsupported_expression.xml",
                "empty_element.xml", "empty_attribute.xml", "xinclude_no_file.xml", "xinclude_cycle.xml",
                "fta/int_overflow.xml"]
    for name in rejected:
        with pytest.raises(mef.MefError):
            mef.parse(INPUT_DIR / name)
    with pytest.raises(OSError):
        mef.parse(INPUT_DIR / "nonexistent_file.xml")
    with pytest.raises(mef.MefError, match="twice"):
        mef.parse([INPUT_DIR / "fta" / "correct_tree_input.xml",
                   INPUT_DIR / ".." / "input" / "fta" / "correct_tree_input.xml"])
    for name in ["fta/labels_and_attributes.xml", "xinclude.xml", "xinclude_transitive.xml",
                 "fta/missing_bool_constant.xml", "fta/correct_tree_input_with_probs.xml", "fta/trailing_spaces.xml",
                 "fta/correct_expressions.xml", "fta/flavored_types.xml"]:
        mef.parse(INPUT_DIR / name)
    # an XInclude brings the included document's elements: the same model as the file itself
    a = mef.parse(INPUT_DIR / "xinclude_transitive.xml")
    b = mef.parse(INPUT_DIR / "fta" / "correct_tree_input.xml")
    assert a.gates == b.gates and a.basic_events.keys() == b.basic_events.keys()
    mef.parse([INPUT_DIR / "fta" / "correct_tree_input.xml", INPUT_DIR / "fta" / "second_fault_tree.xml"])
    with pytest.raises(mef.MefError, match="no probability expression"):  # missing_expression.xml
        mef.load(INPUT_DIR / "fta" / "missing_expression.xml")


def test_formula_arguments_follow_the_schema():
    base = "<opsa-mef><define-gate name='t'>{}</define-gate><define-basic-event name='a'><float value='0.1'/>" \
           "</define-basic-event><define-basic-event name='b'><float value='0.2'/></define-basic-event></opsa-mef>"
    for body in ["<and><or><basic-event name='a'/><basic-event name='b'/></or><basic-event name='a'/></and>",
                 "<not><not><basic-event name='a'/></not></not>", "<or><not><constant value='true'/></not>"
                 "<basic-event name='b'/></or>"]:
        with pytest.raises(mef.MefError):
            mef.parse(base.format(body))
    m = mef.parse(base.format("<or><not><basic-event name='a'/></not><basic-event name='b'/>"
                              "<constant value='false'/></or>"))
    assert m.gates["t"].args[0] == (True, "basic-event", "a")
    with pytest.raises(mef.MefError, match="32-bit"):
        mef.parse("<opsa-mef><define-parameter name='p'><int value='2147483648'/></define-parameter></opsa-mef>")
    mef.parse("<opsa-mef><define-parameter name='p'><int value='-2147483647'/></define-parameter></opsa-mef>")


REF_INPUT = reference_path("input")

# (files, the reference's exact-probability expectation, its tolerance): the
# non-rare-event branches of tests/bench_*_tests.cc
_BENCH_MODELS = [
    (["Autogenerated/200_event.xml"], 0.55985, 1e-5),
    (["Baobab/baobab1.xml", "Baobab/baobab1-basic-events.xml"], 1.2823e-6, 1e-8),
    (["BSCU/BSCU.xml"], 0.1124087, 1e-4),
    (["Chinese/chinese.xml", "Chinese/chinese-basic-events.xml"], 0.0045691, 1e-5),
    (["HIPPS/HIPPS.xml"], 0.0016209, 1e-5),
    (["Lift/lift.xml"], 1.19999e-5, 1e-5),
    (["ne574/ne574.xml"], 0.662208, 1e-6),
    (["SmallTree/SmallTree.xml"], 0.02678, 1e-5),
    (["ThreeMotor/three_motor.xml"], 0.0211538, 1e-5),
    (["TwoTrain/two_train.xml"], 0.7225, 1e-9),
]


@pytest.mark.skipif(not REF_INPUT.exists(), reason="the reference's models are not on this machine")
@pytest.mark.parametrize("files,want,tol", _BENCH_MODELS, ids=[f[0].split("/")[0] for f, _, _ in _BENCH_MODELS])
def test_reference_benchmark_models(oracle_mod, files, want, tol):
    """Exact probability (BDD) of the graph the loader builds against the
    value the reference's tests expect of its exact algorithm."""
    g = mef.parse([REF_INPUT / f for f in files]).flat()
    assert oracle_mod.bdd_probability(g) == pytest.approx(want, abs=tol)


@pytest.mark.skipif(not REF_INPUT.exists(), reason="the reference's models are not on this machine")
def test_reference_theatre_listed_value_is_not_the_files(oracle_mod):
    """tests/bench_theatre_tests.cc expects 0.00207 of input/Theatre/theatre.xml,
    but the file holds M & (G | R) with P(M) = 1, P(G) = 0, P(R) = 0.5: the
    file's value is 0.5, which the loaded graph gives."""
    g = mef.parse(REF_INPUT / "Theatre" / "theatre.xml").flat()
    assert oracle_mod.bdd_probability(g) == pytest.approx(0.5, abs=1e-9)


@pytest.mark.skipif(not REF_INPUT.exists(), reason="the reference's models are not on this machine")
@pytest.mark.parametrize("files,want", [
    (["ThreeMotor/three_motor.xml", "ThreeMotor/event_tree.xml"],  # tests/bench_three_motor_tests.cc:77-90
     {"S1": 0.02115, "S2": 0.00272, "S3": 0.00309, "S4": 0.00272, "S5": 0.00272, "S6": 0.00272, "S7": 0.00272,
      "S8": 0.00272}),
    (["EventTrees/gas_leak/gas_leak_reactive.xml"],  # tests/bench_gas_leak.cc:22-37
     {"S1": 0.81044, "S2": 0.04479, "S3": 0.04265, "S4": 2.36e-3, "S5": 0.04265, "S6": 2.36e-3, "S7": 4.5e-3,
      "S8": 0.05025}),
], ids=["ThreeMotor", "GasLeakReactive"])
def test_reference_event_tree_benchmarks(oracle_mod, files, want):
    from mcscram_b200 import eta
    m = mef.parse([REF_INPUT / f for f in files])
    (ie,) = m.initiating_events
    c = eta.combined_pdag(m, ie)
    g = c.flat()
    got = {s.sequence: oracle_mod.bdd_probability(g, root=int(g.tally_nodes[1 + k]))
           for k, (s, _) in enumerate(c.sequences)}
    assert set(got) == set(want)
    for s, v in want.items():
        assert got[s] == pytest.approx(v, abs=1e-5), s


def _bscu_trials(m, trials, seed):
    _, _, var_index, _ = m.build()
    return mef.sample_expressions(m, {n: m.basic_events[n] for n in var_index}, trials,
                                  np.random.default_rng(seed)), var_index


@pytest.mark.skipif(not REF_INPUT.exists(), reason="the reference's models are not on this machine")
def test_reference_bscu_uncertainty(oracle_mod):
    """tests/bench_bscu_tests.cc:22-54 (exact branch): over 10,000 trials of
    the model's lognormal deviates a mean of 0.117 and a sigma of 0.183
    (both to 5e-3), here from exact per-trial probabilities."""
    m = mef.parse(REF_INPUT / "BSCU" / "BSCU.xml")
    g = m.flat()
    d, var_index = _bscu_trials(m, 10_000, 5)
    name_of = {i: n for n, i in var_index.items()}
    cols = np.stack([np.clip(d[name_of[int(x)]], 0, 1) for x in g.be_pdag_idx], axis=1)
    top = np.array([oracle_mod.bdd_probability(g, row) for row in cols])
    assert top.mean() == pytest.approx(0.117, abs=5e-3)
    assert top.std(ddof=1) == pytest.approx(0.183, abs=5e-3)



def _exact_curve(oracle_mod, m, step, mission_time):
    """(P(top), t) at the reference's time grid, each point exact (BDD)."""
    times, k = [], 0
    while k * step < mission_time:
        times.append(k * step)
        k += 1
    times.append(mission_time)
    _, _, var_index, _ = m.build()
    g = m.flat()
    name_of = {i: n for n, i in var_index.items()}
    return [(oracle_mod.bdd_probability(g, np.array([m.probability(name_of[int(x)], t) for x in g.be_pdag_idx])), t)
            for t in times]


SINGLE_EXP = reference_path("tests", "input", "core", "single_exponential.xml")


@pytest.mark.skipif(not SINGLE_EXP.exists(), reason="the reference's test models are not on this machine")
def test_reference_probability_curve_and_sil(oracle_mod):
    """tests/risk_analysis_tests.cc:355-408: the curve of a single exponential
    event (rate 1e-5) at steps of 24 h up to 120 h, and its SIL metrics over
    the default 8760 h (PFD 0.04255, PFH 9.77e-6 and the band fractions),
    all to the reference's 1e-3."""
    m = mef.parse(SINGLE_EXP)
    curve = _exact_curve(oracle_mod, m, 24.0, 120.0)
    assert [t for _, t in curve] == [0, 24, 48, 72, 96, 120]
    for (p, _), want in zip(curve, [0, 2.399e-4, 4.7989e-4, 7.197e-4, 9.595e-4, 1.199e-3]):
        assert p == pytest.approx(want, rel=1e-3, abs=1e-12)
    sil = mef.safety_integrity_levels(_exact_curve(oracle_mod, m, 24.0, 8760.0))
    assert sil["pfd_avg"] == pytest.approx(0.04255, rel=1e-3)
    assert sil["pfh_avg"] == pytest.approx(9.77e-6, rel=1e-3)
    for (_, got), want in zip(sil["pfd_fractions"], [1.142e-4, 1.0275e-3, 1.02796e-2, 0.1033, 0.88527, 0]):
        assert got == pytest.approx(want, rel=1e-3, abs=1e-12)
    for (_, got), want in zip(sil["pfh_fractions"], [2.74e-7, 2.466e-6, 2.466e-5, 2.466e-4, 0.999726, 0]):
        assert got == pytest.approx(want, rel=1e-3, abs=1e-12)


def test_sil_of_simple_curves():
    """Hand-checkable curves: a constant curve puts all the time in its band;
    a straight line from 0 to 2e-5 spends half its time below 1e-5; one point
    counts whole."""
    flat = mef.safety_integrity_levels([(0.05, 0.0), (0.05, 100.0)])
    assert flat["pfd_avg"] == pytest.approx(0.05)
    assert [f for _, f in flat["pfd_fractions"]] == [0, 0, 0, 0, 1.0, 0]
    line = mef.safety_integrity_levels([(0.0, 0.0), (2e-5, 10.0)])
    assert line["pfd_avg"] == pytest.approx(1e-5)
    assert [f for _, f in line["pfd_fractions"]][:2] == [pytest.approx(0.5), pytest.approx(0.5)]
    one = mef.safety_integrity_levels([(3e-3, 10.0)])
    assert one["pfd_avg"] == 3e-3 and [f for _, f in one["pfd_fractions"]] == [0, 0, 0, 1.0, 0, 0]


@pytest.mark.gpu
def test_sil_from_the_gpu_curve(oracle_mod, gpu):
    """SIL metrics of the batched GPU curve of the timed fixture against those
    of the exact curve: averages within 1 % (2^20 samples a point, p from 1e-3
    to 0.3), band fractions within 0.02 of the mission time."""
    m = mef.parse(TIMED, mission_time=2000.0)
    got = mef.safety_integrity_levels(mef.probability_over_time(m, time_step=50.0, words=1 << 14, iteration=5))
    want = mef.safety_integrity_levels(_exact_curve(oracle_mod, m, 50.0, 2000.0))
    assert got["pfd_avg"] == pytest.approx(want["pfd_avg"], rel=1e-2)
    assert got["pfh_avg"] == pytest.approx(want["pfh_avg"], rel=1e-2)
    for key in ("pfd_fractions", "pfh_fractions"):
        for (b, f), (_, w) in zip(got[key], want[key]):
            assert abs(f - w) <= 0.02, (key, b)


CORE_EXACT = {  # tests/bench_core_tests.cc: the exact branch of each model's p_total expectation
    "abc": 0.496, "ab_bc": 0.074, "ab_or_not_ac": 0.29, "atleast": 0.098, "a_or_not_a": 1.0, "a_or_not_b": 0.82,
    "a_and_not_a": 0.0, "a_and_not_b": 0.08, "a_or_not_ab": 0.28, "multiple_parent_negative_gate": 0.9,
    "nand_or_equality": 1.0, "not_and_or_equality": 1.0, "unity": 1.0, "null": 0.0, "xor": 0.404, "iff": 0.404,
    "imply": 0.986, "cardinality": 0.49, "subtle_unity": 1.0, "subtle_null": 0.0, "zero_prob": 0.0, "one_prob": 1.0,
    "beta_factor_ccf": 0.04308, "phi_factor_ccf": 0.04104, "mgl_ccf": 0.01630, "alpha_factor_ccf": 0.05298,
}


@pytest.mark.skipif(not CORE_IN.exists(), reason="the reference's core inputs are not on this machine")
@pytest.mark.parametrize("name", list(CORE_EXACT))
def test_reference_core_models(oracle_mod, name):
    """Negations, constants, house events, the complex connectives and the
    CCF models of the reference's core tests: exact probability of the
    loaded graph (the sampler's quantised probabilities) against its
    expectation (CCF ones to its 1e-5)."""
    g = mef.parse(CORE_IN / f"{name}.xml", ccf_analysis="ccf" in name).flat()
    tol = 1e-5 if "ccf" in name else 1e-8
    assert oracle_mod.bdd_probability(g) == pytest.approx(CORE_EXACT[name], abs=tol)


@pytest.mark.parametrize("body,want", [
    # tests/expression_tests.cc:152-215, 419-448, 517-546 at the arguments' means
    ("<exponential><float value='10'/><float value='5'/></exponential>", 1 - math.exp(-50)),
    ("<GLM><float value='0.1'/><float value='10'/><float value='100'/><float value='5'/></GLM>",
     (10 - (10 - 0.10 * 110) * math.exp(-110 * 5)) / 110),
    ("<Weibull><float value='0.1'/><float value='10'/><float value='10'/><float value='500'/></Weibull>", 1.0),
    ("<lognormal-deviate><float value='10'/><float value='5'/></lognormal-deviate>", 5.9105e9),
    ("<histogram><float value='0'/><bin><float value='1'/><float value='2'/></bin>"
     "<bin><float value='3'/><float value='4'/></bin></histogram>", 1.5),
])
def test_reference_expression_values(body, want):
    m = mef.parse(f"<opsa-mef><define-parameter name='p'>{body}</define-parameter></opsa-mef>")
    got = m.parameters["p"].value(m.mission_time, m.parameters)
    assert got == pytest.approx(want, rel=1e-12) if want != 5.9105e9 else abs(got - want) <= 1e6


@pytest.mark.gpu
def test_command_line_curve_and_sil(oracle_mod, gpu, capsys):
    import json
    assert mef.main([str(TIMED), "--samples", str(2 ** 20), "--time-step", "1000", "--sil"]) == 0
    out = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    assert [t for _, t in out["p_time"]] == [1000.0 * k for k in range(9)] + [8760.0]
    ps = [p for p, _ in out["p_time"]]
    assert all(b >= a for a, b in zip(ps, ps[1:]))
    want = mef.safety_integrity_levels(_exact_curve(oracle_mod, mef.parse(TIMED), 1000.0, 8760.0))
    assert out["sil"]["pfd_avg"] == pytest.approx(want["pfd_avg"], rel=2e-2)


def test_command_line_refuses_a_curve_with_too_many_points(capsys):
    """A time step that would make more than MAX_TIME_POINTS curve points is
    refused before any point is built (8760 h / 1e-3 h = 8.76e6 points)."""
    assert mef.time_points(8760.0, 1000.0) == 10
    with pytest.raises(SystemExit) as exc:
        mef.main([str(TIMED), "--time-step", "1e-3"])
    assert exc.value.code == 2
    assert "points" in capsys.readouterr().err
    with pytest.raises(ValueError):
        mef.probability_over_time(mef.parse(TIMED), time_step=1e-3)
