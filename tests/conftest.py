"""Shared fixtures.  GPU tests are marked ``gpu``; everything else runs on CPU.

The product package lives in ``adaptive-pf-flip_b200/`` and is imported under
the name ``adaptive_pf_flip_b200``; the CPU checkers live in ``oracle/``.
"""
import importlib.util
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

PKG_NAME = "adaptive_pf_flip_b200"
PKG_DIR = os.path.join(ROOT, "adaptive-pf-flip_b200")


def load_package():
    if PKG_NAME in sys.modules:
        return sys.modules[PKG_NAME]
    spec = importlib.util.spec_from_file_location(PKG_NAME, os.path.join(PKG_DIR, "__init__.py"),
                                                  submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[PKG_NAME] = mod
    spec.loader.exec_module(mod)
    return mod


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 GPU and libpfgpu.so")
    config.addinivalue_line("markers", "slow: larger CPU oracle runs")


@pytest.fixture(scope="session")
def pf():
    return load_package()


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle
    return oracle
