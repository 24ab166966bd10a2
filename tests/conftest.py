import importlib.util
import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
PKG_DIR = os.path.join(ROOT, "bnmf-algs_b200")
GOLDEN = os.path.join(ROOT, "tests", "golden")
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs libbldm.so kernels")


def load_package():
    """Import bnmf-algs_b200/ (a directory name with a hyphen) as bnmf_algs_b200."""
    if "bnmf_algs_b200" in sys.modules:
        return sys.modules["bnmf_algs_b200"]
    spec = importlib.util.spec_from_file_location(
        "bnmf_algs_b200", os.path.join(PKG_DIR, "__init__.py"),
        submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["bnmf_algs_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


@pytest.fixture(scope="session")
def bldm():
    pkg = load_package()
    if not os.path.exists(pkg.LIB_PATH):
        pkg.build()
    return pkg


@pytest.fixture(scope="session")
def workloads():
    load_package()
    import bnmf_algs_b200.workloads as W
    return W


@pytest.fixture(scope="session")
def oracle():
    import oracle as O
    O.lib()
    return O


@pytest.fixture(scope="session")
def kat():
    with open(os.path.join(GOLDEN, "kat_8x10.json")) as f:
        d = json.load(f)
    d["X"] = np.array(d["X"])
    return d


@pytest.fixture(scope="session")
def psi_points():
    with open(os.path.join(GOLDEN, "psi_points.json")) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def plain_small_golden():
    return dict(np.load(os.path.join(GOLDEN, "plain_small.npz")))


def eigen_is_approx(a, b, prec):
    """Eigen's isApprox: ||a - b|| <= prec * min(||a||, ||b||) (Frobenius)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return np.linalg.norm(a - b) <= prec * min(np.linalg.norm(a), np.linalg.norm(b))


@pytest.fixture(scope="session")
def is_approx():
    return eigen_is_approx
