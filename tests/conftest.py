"""Shared test setup.

* registers the ``gpu`` marker (tests that need a B200; run with -m gpu),
* imports the package directory ``tapas-reduce_b200`` as ``tapas_reduce_b200``,
* imports the test oracle (oracle/oracle.py) as ``oracle``.
"""
import importlib.util
import pathlib
import sys

import pytest

ROOT = pathlib.Path(__file__).resolve().parent.parent


def _load_package():
    if "tapas_reduce_b200" in sys.modules:
        return sys.modules["tapas_reduce_b200"]
    pkg_dir = ROOT / "tapas-reduce_b200"
    spec = importlib.util.spec_from_file_location(
        "tapas_reduce_b200", pkg_dir / "__init__.py", submodule_search_locations=[str(pkg_dir)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["tapas_reduce_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


sys.path.insert(0, str(ROOT / "oracle"))
_load_package()


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 GPU (sm_100a)")


@pytest.fixture(scope="session")
def tb():
    return sys.modules["tapas_reduce_b200"]


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle
    oracle.build()
    return oracle


@pytest.fixture(scope="session")
def ctx(tb):
    c = tb.Context(0)
    yield c
    c.close()
