"""Shared test setup: the `gpu` marker and loaders for the package and the oracle."""
import importlib.util
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a) GPU")


def load_package():
    """Import beyond-rpa_b200/ (a hyphenated directory) as `beyond_rpa_b200`."""
    name = "beyond_rpa_b200"
    if name in sys.modules:
        return sys.modules[name]
    pkg_dir = ROOT / "beyond-rpa_b200"
    spec = importlib.util.spec_from_file_location(name, pkg_dir / "__init__.py",
                                                  submodule_search_locations=[str(pkg_dir)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


@pytest.fixture(scope="session")
def pkg():
    return load_package()


@pytest.fixture(scope="session")
def oracle():
    from oracle import rpa_oracle
    return rpa_oracle


@pytest.fixture(scope="session")
def handle(pkg):
    h = pkg.Handle(0)
    yield h
    h.close()
