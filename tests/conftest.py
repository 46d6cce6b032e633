"""Shared fixtures.  The `gpu` marker selects tests that need a B200; the rest
run on CPU (oracle pinning, ABI surface, generators, host logic)."""
import importlib.util
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))


def load_b2s():
    """Import the package in cpp-fem-solver_b200/ under the module name `b2s`."""
    if "b2s" in sys.modules:
        return sys.modules["b2s"]
    path = os.path.join(ROOT, "cpp-fem-solver_b200", "__init__.py")
    spec = importlib.util.spec_from_file_location("b2s", path,
                                                  submodule_search_locations=[os.path.dirname(path)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["b2s"] = mod
    spec.loader.exec_module(mod)
    return mod


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA B200 (run with -m gpu)")


@pytest.fixture(scope="session")
def b2s():
    return load_b2s()


@pytest.fixture(scope="session")
def orc():
    import oracle
    if not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "liborc.so")):
        oracle.build()
    return oracle.Orc()


@pytest.fixture(scope="session")
def ref():
    import oracle
    path = os.path.join(ROOT, "oracle", "_ref", "libref.so")
    if not os.path.exists(path):
        try:
            oracle.build()
        except Exception:
            pass
    if not os.path.exists(path):
        pytest.skip("reference library not built (reference sources absent)")
    r = oracle.Ref()
    r.set_threads(1)
    return r


@pytest.fixture(scope="session")
def ctx(b2s):
    c = b2s.Context(0)
    yield c
    c.close()


@pytest.fixture
def rng():
    return np.random.default_rng(12345)
