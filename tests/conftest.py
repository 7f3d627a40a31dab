"""Test configuration: registers the `gpu` marker and makes the engine package
(directory hmat-oss_b200, imported as `hmat_oss_b200`) and the oracle importable."""
import importlib.util
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
sys.path.insert(0, ROOT)


def load_engine_package():
    if "hmat_oss_b200" in sys.modules:
        return sys.modules["hmat_oss_b200"]
    pkg_dir = os.path.join(ROOT, "hmat-oss_b200")
    spec = importlib.util.spec_from_file_location("hmat_oss_b200", os.path.join(pkg_dir, "__init__.py"),
                                                  submodule_search_locations=[pkg_dir])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["hmat_oss_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")


@pytest.fixture(scope="session")
def hb():
    return load_engine_package()


@pytest.fixture(scope="session")
def oracle():
    import oracle as o  # noqa: E402  (oracle/oracle.py)
    return o


def has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


GOLDEN = os.path.join(ROOT, "tests", "golden")


def golden(name):
    import numpy as np
    return dict(np.load(os.path.join(GOLDEN, name + ".npz")))


def rel(a, b):
    import numpy as np
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))
