import importlib.util
import os
import sys

import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def _load(name, path):
    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


ENGINE = _load("sankhya_b200", os.path.join(ROOT, "the-solver_b200", "__init__.py"))
INSTANCES = _load("sankhya_b200_instances", os.path.join(ROOT, "the-solver_b200", "instances.py"))
LEARNED = _load("sankhya_b200_learned", os.path.join(ROOT, "the-solver_b200", "learned.py"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def engine():
    return ENGINE


@pytest.fixture(scope="session")
def instances():
    return INSTANCES


@pytest.fixture(scope="session")
def learned():
    return LEARNED


@pytest.fixture(scope="session")
def oracle():
    import oracle as O
    return O


@pytest.fixture(scope="session")
def golden_dir():
    return os.path.join(ROOT, "tests", "golden")
