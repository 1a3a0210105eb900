"""Test configuration: registers the ``gpu`` marker and makes the package importable as ``qsv_b200``
(its directory name contains dashes, so it is loaded from its path)."""
import importlib.util
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG_DIR = os.path.join(ROOT, "u55c-statevector-30q_b200")


def _load_package():
    if "qsv_b200" in sys.modules:
        return sys.modules["qsv_b200"]
    spec = importlib.util.spec_from_file_location("qsv_b200", os.path.join(PKG_DIR, "__init__.py"),
                                                  submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["qsv_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


_load_package()
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
