"""The C-ABI library without a GPU: it loads, exports every declared entry
point, and rejects malformed graphs with MCG_ERR_INVALID and a message (the
reference logs and exits instead, src/mc/queue/kernel_builder.h:340-342)."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

from mcscram_b200 import synth
from mcscram_b200.graph import AND, OR, FlatGraph
from tests.conftest import HAS_GPU

ROOT = Path(__file__).resolve().parent.parent


def declared_functions():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        names |= set(re.findall(r"\b(mcg_[a-z0-9_]+)\s*\(", text))
    return sorted(names)


def test_exports_every_declared_function(capi):
    lib = capi.load()
    names = declared_functions()
    assert len(names) >= 10
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_version_and_error_strings(capi):
    assert "sm_100a" in capi.version()
    assert capi.load().mcg_last_error() is not None


def _graph(**kw):
    base = dict(be_pdag_idx=[2, 3], be_event_idx=[0, 1], be_threshold=[1 << 30, 1 << 31], gate_op=[AND],
                gate_k=[0], gate_in_begin=[0], gate_in_count=[2], gate_neg_count=[0], inputs=[0, 1],
                tally_nodes=[2])
    base.update(kw)
    g = FlatGraph(**base)
    return g


def test_rejects_malformed_graphs(capi):
    lib = capi.load()
    # bypass FlatGraph.validate to reach the C validation
    for kw, msg in [
        (dict(inputs=[0, 2]), "not an earlier node"),
        (dict(gate_neg_count=[3]), "neg_count"),
        (dict(be_threshold=[(1 << 32) + 1, 5]), "threshold above 2^32"),
        (dict(tally_nodes=[7]), "out of range"),
        (dict(gate_op=[9]), "unknown connective"),
        (dict(gate_in_count=[5]), "inputs out of range"),
    ]:
        g = _graph(**kw)
        # build the descriptor without python-side validation
        p = lambda a, t: a.ctypes.data_as(C.POINTER(t))
        keep = [g.be_pdag_idx, g.be_event_idx, g.be_threshold, g.gate_pdag_idx, g.gate_op, g.gate_k,
                g.gate_in_begin, g.gate_in_count, g.gate_neg_count, g.inputs, g.tally_nodes]
        desc = capi.GraphDesc(g.n_be, g.n_gates, p(g.be_pdag_idx, C.c_int32), p(g.be_event_idx, C.c_uint32),
                              p(g.be_threshold, C.c_uint64), p(g.gate_pdag_idx, C.c_int32), p(g.gate_op, C.c_uint8),
                              p(g.gate_k, C.c_uint32), p(g.gate_in_begin, C.c_uint32),
                              p(g.gate_in_count, C.c_uint32), p(g.gate_neg_count, C.c_uint32),
                              p(g.inputs, C.c_uint32), g.inputs.size, g.tally_nodes.size,
                              p(g.tally_nodes, C.c_uint32))
        h = C.c_void_p()
        rc = lib.mcg_create(C.byref(desc), None, C.byref(h))
        assert rc == capi.MCG_ERR_INVALID, (kw, rc)
        assert msg in lib.mcg_last_error().decode(), (kw, lib.mcg_last_error())
        info = capi.ProgramInfo()
        assert lib.mcg_compile(C.byref(desc), 8, 0, C.byref(info), None, 0) == capi.MCG_ERR_INVALID
        del keep


def test_null_arguments(capi):
    lib = capi.load()
    assert lib.mcg_create(None, None, None) == capi.MCG_ERR_INVALID
    assert lib.mcg_run(None, 1, 1, 0, 1) == capi.MCG_ERR_INVALID
    assert lib.mcg_read_tallies(None, None, None) == capi.MCG_ERR_INVALID
    assert lib.mcg_destroy(None) == capi.MCG_OK


@pytest.mark.skipif(HAS_GPU, reason="checks the no-device path")
def test_no_device_reported(capi):
    with pytest.raises(capi.McgError) as ei:
        capi.Engine(synth.config1())
    assert ei.value.code == capi.MCG_ERR_NO_DEVICE


def test_product_package_does_not_import_oracle():
    pkg = ROOT / "mcscram_b200"
    for f in list(pkg.rglob("*.py")) + list(pkg.rglob("*.cu")) + list(pkg.rglob("*.cpp")) + list(pkg.rglob("*.h*")):
        text = f.read_text(errors="ignore")
        assert "import oracle" not in text and "from oracle" not in text and "liboracle" not in text, f
