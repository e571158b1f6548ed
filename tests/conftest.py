import importlib.util
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def _load_package():
    if "atum_b200" in sys.modules:
        return sys.modules["atum_b200"]
    pkg_dir = os.path.join(ROOT, "atum.jl_b200")
    spec = importlib.util.spec_from_file_location("atum_b200", os.path.join(pkg_dir, "__init__.py"),
                                                  submodule_search_locations=[pkg_dir])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["atum_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


_load_package()
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (runs through the CUDA C ABI)")
    config.addinivalue_line("markers", "slow: long CPU oracle runs")


@pytest.fixture(scope="session")
def atb():
    return sys.modules["atum_b200"]


@pytest.fixture(scope="session")
def orc():
    import pyoracle
    pyoracle.build()
    # element loops only: results do not depend on the thread count
    pyoracle.set_threads(min(os.cpu_count() or 1, 32))
    return pyoracle
