"""Shared fixtures.  GPU tests are marked ``gpu``; everything else runs on
CPU.  The package directory is ``ib.cu_b200/`` (not an importable name), so
it is loaded by path as module ``ib_cu_b200``."""
import importlib.util
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def load_package():
    if "ib_cu_b200" in sys.modules:
        return sys.modules["ib_cu_b200"]
    pkg_dir = os.path.join(ROOT, "ib.cu_b200")
    spec = importlib.util.spec_from_file_location(
        "ib_cu_b200", os.path.join(pkg_dir, "__init__.py"), submodule_search_locations=[pkg_dir])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["ib_cu_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def ibk():
    return load_package()


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.build()
    return O


@pytest.fixture(scope="session")
def cuda(ibk):
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test run without a CUDA device")
    ibk.build()
    ibk.lib()
    return torch.device("cuda:0")
