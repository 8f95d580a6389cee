"""Shared fixtures. `-m "not gpu"` runs on any host (oracle KATs, the C ABI's
exports and host logic); `-m gpu` runs the CUDA parity tests on an sm_100 GPU
through the C ABI."""
import importlib.util
import json
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
# enough hardware work queues for the serving loop's streams (before any CUDA call)
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")
sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 (B200) GPU")


def _load(name, path):
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


@pytest.fixture(scope="session")
def sb():
    """The product package (sequoia-boost_b200/), importable as sequoia_boost_b200."""
    ge = _load("__graft_entry__", os.path.join(ROOT, "__graft_entry__.py"))
    return ge.load_package()


@pytest.fixture(scope="session")
def orc():
    """The CPU oracle (test infrastructure: the checker)."""
    lib = os.path.join(ROOT, "oracle", "liboracle.so")
    if not os.path.exists(lib):
        ge = _load("__graft_entry__", os.path.join(ROOT, "__graft_entry__.py"))
        ge.build_oracle()
    return _load("sb_pyoracle", os.path.join(ROOT, "oracle", "pyoracle.py")).Oracle()


@pytest.fixture(scope="session")
def kats():
    with open(os.path.join(ROOT, "tests", "golden", "reference_kats.json")) as fh:
        data = json.load(fh)
    return {c["name"]: c for c in data["cases"]}


@pytest.fixture(scope="session")
def ctx(sb):
    return sb.Context(0)


@pytest.fixture(scope="session")
def datagen(sb):
    return sys.modules["sequoia_boost_b200.datagen"] if "sequoia_boost_b200.datagen" in sys.modules \
        else __import__("sequoia_boost_b200.datagen", fromlist=["datagen"])
