import importlib.util
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG_DIR = os.path.join(ROOT, "gpu-louvain_b200")
ORACLE_DIR = os.path.join(ROOT, "oracle")
GOLDEN_DIR = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def load_pkg():
    if "gpu_louvain_b200" in sys.modules:
        return sys.modules["gpu_louvain_b200"]
    if not os.path.exists(os.path.join(PKG_DIR, "lib", "liblouvain_b200.so")):
        subprocess.run(["make", "-C", PKG_DIR, "-j8"], check=True, capture_output=True)
    spec = importlib.util.spec_from_file_location(
        "gpu_louvain_b200", os.path.join(PKG_DIR, "__init__.py"), submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["gpu_louvain_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def load_oracle():
    if ORACLE_DIR not in sys.path:
        sys.path.insert(0, ORACLE_DIR)
    import oracle  # noqa: E402
    return oracle


@pytest.fixture(scope="session")
def lvb():
    return load_pkg()


@pytest.fixture(scope="session")
def orc():
    return load_oracle()


@pytest.fixture(scope="session")
def gnp():
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import graphs_np  # noqa: E402
    return graphs_np
