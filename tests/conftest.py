import importlib.util
import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def load_package():
    """Imports msbg-rs_b200/ under the module name msbg_rs_b200."""
    if "msbg_rs_b200" in sys.modules:
        return sys.modules["msbg_rs_b200"]
    pkg_dir = os.path.join(ROOT, "msbg-rs_b200")
    spec = importlib.util.spec_from_file_location("msbg_rs_b200", os.path.join(pkg_dir, "__init__.py"),
                                                  submodule_search_locations=[pkg_dir])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["msbg_rs_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


@pytest.fixture(scope="session")
def msbg():
    return load_package()


@pytest.fixture(scope="session")
def oracle():
    import oracle as o
    o.lib()
    return o


@pytest.fixture(scope="session")
def goldens():
    with open(os.path.join(ROOT, "tests", "golden", "reference_goldens.json")) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def ctx(msbg):
    c = msbg.Context(0)
    yield c
    c.synchronize()


def rng(seed):
    return np.random.default_rng(seed)
