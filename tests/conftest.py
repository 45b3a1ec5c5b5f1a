import importlib.util
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG_DIR = os.path.join(ROOT, "vlite-frb_b200")
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))


def load_pkg():
    """Import the hyphen-named package directory as `vlite_frb_b200`."""
    if "vlite_frb_b200" in sys.modules:
        return sys.modules["vlite_frb_b200"]
    spec = importlib.util.spec_from_file_location("vlite_frb_b200", os.path.join(PKG_DIR, "__init__.py"),
                                                  submodule_search_locations=[PKG_DIR])
    m = importlib.util.module_from_spec(spec)
    sys.modules["vlite_frb_b200"] = m
    spec.loader.exec_module(m)
    return m


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA (B200) device")


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _has_gpu():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def vf():
    return load_pkg()


@pytest.fixture(scope="session")
def O():
    import vfrb_oracle
    return vfrb_oracle
