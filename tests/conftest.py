"""Test set-up: registers the package directory `heterogeneous-solvers_b200`
as the importable module `hs_b200`, loads the CPU oracle for the checkers and
declares the `gpu` marker."""
import importlib.util
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT / "tests") not in sys.path:
    sys.path.insert(0, str(ROOT / "tests"))


def load_package():
    if "hs_b200" in sys.modules:
        return sys.modules["hs_b200"]
    pkg_dir = ROOT / "heterogeneous-solvers_b200"
    spec = importlib.util.spec_from_file_location("hs_b200", pkg_dir / "__init__.py",
                                                  submodule_search_locations=[str(pkg_dir)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["hs_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a) and libhs_b200.so")


@pytest.fixture(scope="session")
def hs():
    return load_package()


@pytest.fixture(scope="session")
def ctx(hs):
    c = hs.Context(device=0)
    yield c
    c.close()
