import importlib.util
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: longer CPU test")


def load_package():
    """Import the product package (its directory name is not an identifier)."""
    name = "spectral_bslpm_b200"
    if name in sys.modules:
        return sys.modules[name]
    pkg_dir = os.path.join(ROOT, "spectral-bslpm_b200")
    spec = importlib.util.spec_from_file_location(name, os.path.join(pkg_dir, "__init__.py"),
                                                  submodule_search_locations=[pkg_dir])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


@pytest.fixture(scope="session")
def sb():
    return load_package()


@pytest.fixture(scope="session")
def port():
    from oracle.pyoracle import Port

    return Port()


def _ensure_port_oracle():
    """Build the C restatement oracle (the checker) when it is missing."""
    so = os.path.join(ROOT, "oracle", "liboracle_port.so")
    if not os.path.exists(so):
        import subprocess

        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "port"], check=True)


_ensure_port_oracle()
