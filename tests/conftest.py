"""Shared fixtures.

GPU tests (marker ``gpu``) call the CUDA engine through its C ABI and compare it with the
golden fixtures in tests/golden/ (made by the reference's own lysh) and with the C
restatement in oracle/.  CPU tests check the oracle, the host logic and that the C-ABI
library loads and exports what include/witchgpu.h declares.
"""
from __future__ import annotations

import importlib.util
import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (runs on the B200 box)")


def load_package():
    name = "low_witch_finder_b200"
    if name in sys.modules:
        return sys.modules[name]
    path = os.path.join(ROOT, "low-witch-finder_b200", "__init__.py")
    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


@pytest.fixture(scope="session")
def wg():
    return load_package()


@pytest.fixture(scope="session")
def bind_mod():
    import bind
    return bind


@pytest.fixture(scope="session")
def port(bind_mod):
    return bind_mod.Port()


@pytest.fixture(scope="session")
def ref(bind_mod):
    if not os.path.exists(bind_mod.REF_LIB):
        pytest.skip("oracle/_ref not built (needs the reference sources)")
    return bind_mod.Ref()


def _has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def engine(wg):
    if not _has_gpu():
        pytest.skip("no CUDA device")
    eng = wg.Engine(0)
    yield eng
    eng.close()


@pytest.fixture(scope="session")
def golden():
    def load(name):
        p = os.path.join(GOLDEN, name)
        if name.endswith(".json"):
            with open(p) as f:
                return json.load(f)
        return np.load(p)
    return load
