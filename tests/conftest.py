import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import __graft_entry__ as entry  # noqa: E402


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


HAS_GPU = _has_gpu()


@pytest.fixture(scope="session")
def rv():
    return entry.load_package()


@pytest.fixture(scope="session")
def orc():
    return entry.load_oracle()


@pytest.fixture(scope="session")
def mlp_oracle():
    """The float64 oracle of the precision selector's network (checker only)."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("rvg_mlp_oracle", os.path.join(ROOT, "oracle", "mlp_oracle.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


@pytest.fixture(scope="session")
def golden():
    import json
    with open(os.path.join(ROOT, "tests", "golden", "hand_constructed.json")) as f:
        return json.load(f)


def golden_system(rv, name, g):
    import scipy.sparse as sp
    e = np.array(g["entries"], dtype=float).reshape(-1, 3)
    n = g["n"]
    r, c, v = e[:, 0].astype(int), e[:, 1].astype(int), e[:, 2]
    off = r != c
    a = sp.csc_matrix((np.concatenate([v, v[off]]), (np.concatenate([r, c[off]]), np.concatenate([c, r[off]]))),
                      shape=(n, n))
    return rv.problems.from_scipy(name, a, inertia=tuple(g["inertia"]))


def pytest_collection_modifyitems(config, items):
    if HAS_GPU:
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)
