"""Shared pytest setup: markers, import paths, library builds."""
import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


# Root of an mcSCRAM source tree, from the environment variable MCSCRAM_REF.
# The tests that read the reference's own input models, benchmark table and
# test-input lists skip when it is not set.
_REFERENCE_ROOT = os.environ.get("MCSCRAM_REF") or None


def reference_path(*parts) -> Path:
    """A path inside the reference tree; when MCSCRAM_REF is not set, a path
    under this directory that does not exist, so that `.exists()` guards skip."""
    base = Path(_REFERENCE_ROOT) if _REFERENCE_ROOT else Path(__file__).resolve().parent / "_reference_not_given"
    return base.joinpath(*parts)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long-running CPU test")


def _has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


HAS_GPU = _has_gpu()


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import oracle
    oracle.build()
    return oracle


@pytest.fixture(scope="session")
def capi():
    from mcscram_b200 import _capi
    _capi.load()
    return _capi


@pytest.fixture(scope="session")
def gpu():
    if not HAS_GPU:
        pytest.skip("no CUDA device")
    return 0
