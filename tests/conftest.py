"""Shared fixtures: the product binding (vbvs--vixen_b200) and the CPU oracle.

The package directory name is not a Python identifier, so it is loaded by path
under the module name `vx_b200`.
"""
import importlib.util
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG_DIR = os.path.join(ROOT, "vbvs--vixen_b200")
ORACLE_DIR = os.path.join(ROOT, "oracle")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def load_vx():
    if "vx_b200" in sys.modules:
        return sys.modules["vx_b200"]
    spec = importlib.util.spec_from_file_location("vx_b200", os.path.join(PKG_DIR, "__init__.py"),
                                                  submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["vx_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def load_oracle():
    if ORACLE_DIR not in sys.path:
        sys.path.insert(0, ORACLE_DIR)
    import vx_oracle
    return vx_oracle


@pytest.fixture(scope="session")
def vx():
    return load_vx()


@pytest.fixture(scope="session")
def vo():
    return load_oracle()


def has_cuda():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def cuda():
    if not has_cuda():
        pytest.fail("a CUDA device is required for -m gpu tests")
    import torch
    return torch.device("cuda:0")


def unit(v):
    v = np.asarray(v, np.float32)
    return v / np.float32(np.sqrt(np.float32((v[0] * v[0] + v[1] * v[1]) + v[2] * v[2])))
