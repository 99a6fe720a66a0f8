"""Importance-factor relations of the library (mcg_importance_from_conditionals,
the code mcg_importance_factors applies to its tallies) fed with exact BDD
conditionals P(top | x=1), P(top | x=0) of the reference's own test models,
against the factors its tests expect (tests/risk_analysis_tests.cc:263-310,
tests/bench_chinese_tree_tests.cc:54-81; relative 1e-3, its epsilon),
including the zeros it keeps where a factor is undefined.  Host only: no
device is needed."""
from pathlib import Path

import numpy as np
import pytest

from mcscram_b200 import mef
from tests.conftest import reference_path

REF = reference_path()
needs_ref = pytest.mark.skipif(not REF.exists(), reason="the reference's test models are not on this machine")


def _exact_factors(oracle_mod, files):
    from mcscram_b200.factors import factors_from_conditionals
    m = mef.parse([REF / f for f in files])
    _, _, var_index, _ = m.build()
    g = m.flat()
    name_of = {i: n for n, i in var_index.items()}
    # the model's own probabilities (not the sampler's quantised ones), house events as 0 / 1
    p = np.array([m.probability(name_of[int(x)]) if int(x) in name_of else float(q)
                  for x, q in zip(g.be_pdag_idx, g.quantised_probabilities())])
    top = oracle_mod.bdd_probability(g, p)
    out = {}
    for e, x in enumerate(g.be_pdag_idx):
        if int(x) not in name_of:
            continue
        p1, p0 = p.copy(), p.copy()
        p1[e], p0[e] = 1.0, 0.0
        out[name_of[int(x)]] = factors_from_conditionals(float(p[e]), top, oracle_mod.bdd_probability(g, p1),
                                                         oracle_mod.bdd_probability(g, p0))
    return top, out


# (mif, cif, dif, raw, rrw) per event, as the reference's tests list them
_CASES = {
    "default": (["tests/input/fta/correct_tree_input_with_probs.xml"], 0.646, {
        "PumpOne": (0.51, 0.4737, 0.7895, 1.316, 1.9), "PumpTwo": (0.38, 0.4118, 0.8235, 1.176, 1.7),
        "ValveOne": (0.34, 0.2105, 0.5263, 1.316, 1.267), "ValveTwo": (0.228, 0.1765, 0.5882, 1.176, 1.214)}),
    "negation": (["tests/input/fta/importance_neg_test.xml"], 0.04459, {
        "PumpOne": (0.0765, 0.1029, 0.1568, 2.613, 1.115), "PumpTwo": (0.057, 0.08948, 0.1532, 2.189, 1.098),
        "ValveOne": (0.94, 0.8432, 0.8495, 21.237, 6.379), "ValveTwo": (0.0558, 0.06257, 0.1094, 2.189, 1.067)}),
    "single": (["tests/input/core/null_a.xml"], None, {"OnlyChild": (1, 1, 1, 2, 0)}),
    "zero": (["tests/input/core/zero_prob.xml"], 0.0, {"A": (1, 0, 0, 0, 0)}),
    "one": (["tests/input/core/one_prob.xml"], 1.0, {"A": (1, 1, 1, 1, 0)}),
    "chinese": (["input/Chinese/chinese.xml", "input/Chinese/chinese-basic-events.xml"], 0.0045691, {
        **{e: (0.0745557, 0.326332, 0.339805, 16.9902, 1.48441) for e in ("e1", "e2", "e3")},
        **{e: (5.89643e-05, 0.000258088, 0.0202529, 1.01265, 1.00026) for e in ("e9", "e10", "e11")},
        **{e: (5.64596e-06, 2.47125e-05, 0.0200242, 1.00121, 1.00002) for e in ("e17", "e18")},
        **{e: (4.60982e-06, 2.01773e-05, 0.0200198, 1.00099, 1.00002) for e in ("e19", "e20")},
        "e21": (2.3919e-06, 1.04694e-05, 0.0200103, 1.00051, 1.00001),
        **{e: (9.51481e-05, 0.000416465, 0.0204081, 1.02041, 1.00042) for e in ("e12", "e13")},
        **{e: (0.0553923, 0.242453, 0.257604, 12.8802, 1.32005) for e in ("e4", "e5", "e6", "e7")},
        **{e: (5.1467e-06, 2.25272e-05, 0.0200221, 1.0011, 1.00002) for e in ("e14", "e15", "e16")},
        **{e: (1.03582e-05, 4.5338e-05, 0.0200444, 1.00222, 1.00005) for e in ("e22", "e23", "e24", "e25")},
        "e8": (0.000181647, 0.000795073, 0.0207792, 1.03896, 1.0008)}),
}


@needs_ref
@pytest.mark.parametrize("case", list(_CASES))
def test_reference_importance_factors(oracle_mod, case):
    files, p_top, want = _CASES[case]
    top, got = _exact_factors(oracle_mod, files)
    if p_top is not None:
        assert top == pytest.approx(p_top, rel=1e-4, abs=1e-12)
    assert set(want) <= set(got)
    for name, factors in want.items():
        for key, v in zip(("mif", "cif", "dif", "raw", "rrw"), factors):
            assert got[name][key] == pytest.approx(v, rel=1e-3, abs=1e-12), (name, key)


def test_relations_and_their_zeros():
    """The relations on hand-picked conditionals: P(top) = 0 leaves cif, raw,
    dif and rrw at 0; P(top) = p * mif leaves rrw at 0; invalid input fails."""
    from mcscram_b200 import _capi
    from mcscram_b200.factors import factors_from_conditionals
    p, g1, g0 = 0.2, 0.9, 0.4
    top = p * g1 + (1 - p) * g0
    f = factors_from_conditionals(p, top, g1, g0)
    mif = g1 - g0
    assert f["mif"] == pytest.approx(mif) and f["p_joint"] == pytest.approx(p * g1)
    assert f["cif"] == pytest.approx(p * mif / top) and f["raw"] == pytest.approx(g1 / top)
    assert f["dif"] == pytest.approx(p * g1 / top) and f["rrw"] == pytest.approx(top / g0)
    z = factors_from_conditionals(0.3, 0.0, 0.0, 0.0)
    assert (z["cif"], z["raw"], z["dif"], z["rrw"]) == (0.0, 0.0, 0.0, 0.0)
    assert factors_from_conditionals(0.5, 0.5, 1.0, 0.0)["rrw"] == 0.0
    with pytest.raises(_capi.McgError):
        factors_from_conditionals(1.5, 0.5, 1.0, 0.0)
