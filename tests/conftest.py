import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden", "golden_l4.npz")
PITCH = 0.205  # resting pitch of the reference's fixtures (scripts/engine_metrics.py:55)
DIMS = (0.3, 0.3, 0.2)
DT = 1 / 240


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the sm_100a library")


def stack(K):
    """scripts/colored_vs_jacobi.py:100-101"""
    return [[0, 0, 0.101 + k * PITCH] for k in range(K)]


def lattice(n_target, layers=2):
    """scripts/colored_vs_jacobi.py:104-112"""
    side = int(np.ceil(np.sqrt(n_target / layers)))
    out = []
    for lz in range(layers):
        for iy in range(side):
            for ix in range(side):
                out.append([ix * 0.35, iy * 0.35, 0.101 + lz * PITCH])
    return out[:n_target]


SCENES = {"stack8": (lambda: stack(8), 120), "lattice1000": (lambda: lattice(1000), 40)}


@pytest.fixture(scope="session")
def golden():
    return np.load(GOLDEN)


@pytest.fixture(scope="session")
def me():
    import __graft_entry__ as ge
    return ge.load_package()


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import oracle as O
    return O


def cuda_ok():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
