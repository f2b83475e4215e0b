"""abacus-public_b200: the abacus near-field direct-force path on B200 (sm_100a).

Python side of the package: the ctypes binding of the C ABI (capi), the
seeded synthetic boxes (synth).  The product is the CUDA library
lib/libnfb200.so built from csrc/ by build.py.

The directory name contains a dash, so it is loaded by path; load() does that
and registers it as ``abacus_public_b200``.
"""
from __future__ import annotations

import importlib.util
import pathlib
import sys

PKG_DIR = pathlib.Path(__file__).resolve().parent


def load(root: str | pathlib.Path | None = None):
    """Import the package directory as module ``abacus_public_b200``."""
    if "abacus_public_b200" in sys.modules:
        return sys.modules["abacus_public_b200"]
    d = pathlib.Path(root) / "abacus-public_b200" if root else PKG_DIR
    spec = importlib.util.spec_from_file_location(
        "abacus_public_b200", d / "__init__.py", submodule_search_locations=[str(d)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["abacus_public_b200"] = mod
    spec.loader.exec_module(mod)
    return mod
