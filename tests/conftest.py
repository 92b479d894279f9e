"""Shared test set-up.

* registers the `gpu` marker (tests that need a B200; the rest run on CPU);
* puts the repository root on sys.path so `oracle` (the checker) imports;
* loads the product package from its directory `getting-air_b200/` under the
  module name `getting_air_b200`.
"""
from __future__ import annotations

import importlib.util
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def load_package():
    if "getting_air_b200" in sys.modules:
        return sys.modules["getting_air_b200"]
    pkg_dir = ROOT / "getting-air_b200"
    spec = importlib.util.spec_from_file_location(
        "getting_air_b200", pkg_dir / "__init__.py", submodule_search_locations=[str(pkg_dir)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["getting_air_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def lbm():
    return load_package()


@pytest.fixture(scope="session")
def oracle():
    import oracle as o
    return o
