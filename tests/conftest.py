"""Shared fixtures.  GPU tests are marked ``gpu``; everything else runs on CPU."""
import pathlib
import sys

import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "oracle"))

import importlib.util  # noqa: E402

_spec = importlib.util.spec_from_file_location(
    "abacus_public_b200", ROOT / "abacus-public_b200" / "__init__.py",
    submodule_search_locations=[str(ROOT / "abacus-public_b200")])
if "abacus_public_b200" not in sys.modules:
    _mod = importlib.util.module_from_spec(_spec)
    sys.modules["abacus_public_b200"] = _mod
    _spec.loader.exec_module(_mod)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def synth():
    from abacus_public_b200 import synth as s
    return s


@pytest.fixture(scope="session")
def capi():
    from abacus_public_b200 import capi as c
    return c


@pytest.fixture(scope="session")
def oracle():
    import oracle as o
    return o
