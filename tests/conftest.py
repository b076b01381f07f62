"""Shared test setup: the `gpu` marker, the engine package and the oracle.

The engine package lives in ``quasistrided.jl_b200/`` (a directory name that
is not a Python identifier); it is loaded here under the module name
``quasistrided_b200``.
"""
import importlib.util
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
PKG_DIR = os.path.join(ROOT, "quasistrided.jl_b200")


def load_engine():
    if "quasistrided_b200" in sys.modules:
        return sys.modules["quasistrided_b200"]
    spec = importlib.util.spec_from_file_location(
        "quasistrided_b200", os.path.join(PKG_DIR, "__init__.py"),
        submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["quasistrided_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    lib = os.path.join(PKG_DIR, "lib", "libqsgpu.so")
    if not os.path.exists(lib):
        spec = importlib.util.spec_from_file_location("qs_build", os.path.join(PKG_DIR, "build.py"))
        b = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(b)
        b.build()


@pytest.fixture(scope="session")
def qs():
    return load_engine()


@pytest.fixture(scope="session")
def orc():
    from oracle import oracle
    oracle.lib()
    return oracle
