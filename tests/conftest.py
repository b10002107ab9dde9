"""Shared fixtures: the product package (mini-castro_b200/), the CPU oracle
(checker only) and the generated Helmholtz table."""
from __future__ import annotations

import importlib.util
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG_DIR = os.path.join(ROOT, "mini-castro_b200")
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))


def load_package():
    if "mini_castro_b200" in sys.modules:
        return sys.modules["mini_castro_b200"]
    spec = importlib.util.spec_from_file_location("mini_castro_b200", os.path.join(PKG_DIR, "__init__.py"),
                                                  submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["mini_castro_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); parity tests through the C-ABI")


@pytest.fixture(scope="session")
def pkg():
    return load_package()


@pytest.fixture(scope="session")
def table(pkg):
    return pkg.helm_table.ensure_table()


@pytest.fixture(scope="session")
def oracle():
    import oracle as O

    O.build()
    return O


def cuda_available() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False
