import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def _ensure_built():
    from fve_dg_b200 import build as B
    lib = os.path.join(ROOT, "fve_dg_b200", "libfvedg_b200.so")
    orc = os.path.join(ROOT, "oracle", "liboracle.so")
    if not os.path.exists(lib):
        B.build()
    if not os.path.exists(orc):
        B.build_oracle(with_ref=False)


_ensure_built()


def gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def rng():
    return np.random.default_rng(20261203)


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


# (order, tet rule, tri rule) cases: the configurations' rules and the reference's Auto rules
CASES = [(1, 0, 1), (1, 0, 0), (1, 2, 2), (2, 1, 2), (2, 2, 3), (3, 3, 3), (3, 4, 3), (4, 5, 3), (4, 6, 3)]
