"""Shared test set-up: markers, paths and loaders.

The package directory is `daphne-benchmark_b200/` (not an importable name);
it is loaded under the module name `daphne_benchmark_b200`.
"""
import importlib.util
import pathlib
import sys

import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
PKG_DIR = ROOT / "daphne-benchmark_b200"
sys.path.insert(0, str(ROOT / "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA (sm_100) device")
    config.addinivalue_line("markers", "slow: longer CPU cases")


def load_package():
    name = "daphne_benchmark_b200"
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(name, PKG_DIR / "__init__.py",
                                                  submodule_search_locations=[str(PKG_DIR)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


@pytest.fixture(scope="session")
def pkg():
    return load_package()


@pytest.fixture(scope="session")
def oracle():
    import binding
    return binding.Oracle()


@pytest.fixture(scope="session")
def reference():
    import binding
    if not binding.Reference.available("serial"):
        pytest.skip("compiled reference (oracle/_ref) not built here")
    return binding.Reference("serial")


@pytest.fixture(scope="session")
def binding_mod():
    import binding
    return binding
