import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (runs the CUDA path)")


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
def oracle():
    from oracle import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def reference():
    from oracle import Reference
    if not Reference.available():
        pytest.skip("compiled reference (oracle/_ref) not built here")
    return Reference()


@pytest.fixture(scope="session")
def g12():
    import g12kba_b200
    g12kba_b200.lib()
    return g12kba_b200


def rel_err(a, b, floor=1e-300):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(float(np.max(np.abs(b))), floor)) if b.size else 0.0


def dipole_err(p, p_ref, traj_ref):
    """max |p - p_ref| over the larger of max |p_ref| and the G1 scale of the
    trajectory: a dipole that is pure round-off (quench off, symmetric chain)
    has no relative error of its own."""
    scale = max(float(np.max(np.abs(p_ref))) if np.size(p_ref) else 0.0, float(np.max(np.abs(traj_ref))))
    return float(np.max(np.abs(np.asarray(p) - np.asarray(p_ref)))) / scale


def rand_c(rng, *shape, scale=1.0):
    return scale * (rng.standard_normal(shape) + 1j * rng.standard_normal(shape))


def load_golden(name):
    return np.load(os.path.join(GOLDEN, name), allow_pickle=False)
