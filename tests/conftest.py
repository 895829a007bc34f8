"""Shared fixtures.  The package directory is ceemdan-gpu_b200/ (not an importable name), so
it is loaded by path under the module name ceemdan_gpu_b200."""
import importlib.util
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def load_package():
    if "ceemdan_gpu_b200" in sys.modules:
        return sys.modules["ceemdan_gpu_b200"]
    pkg_dir = os.path.join(ROOT, "ceemdan-gpu_b200")
    spec = importlib.util.spec_from_file_location(
        "ceemdan_gpu_b200", os.path.join(pkg_dir, "__init__.py"),
        submodule_search_locations=[pkg_dir])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["ceemdan_gpu_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


@pytest.fixture(scope="session")
def pkg():
    return load_package()


@pytest.fixture(scope="session")
def orc():
    import oracle
    oracle.build()
    return oracle


@pytest.fixture(scope="session")
def wl(pkg):
    import ceemdan_gpu_b200.workloads as w  # noqa: F401  (loaded through the package path)
    return w


@pytest.fixture(scope="session")
def built_lib(pkg):
    """libceemdan_b200.so, compiled here when absent (nvcc cross-compiles without a GPU)."""
    if not os.path.exists(pkg.LIB_PATH):
        pkg.build()
    return pkg.LIB_PATH


@pytest.fixture(scope="session")
def cuda(pkg, built_lib):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")
