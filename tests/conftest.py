"""Shared fixtures. GPU tests carry @pytest.mark.gpu; everything else runs on CPU."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "gpu-conjugate-gradient-solver_b200")
for p in (PKG, ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def cuda_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def gs():
    import gpusolver_b200
    gpusolver_b200.lib()
    return gpusolver_b200


@pytest.fixture(scope="session")
def orc():
    from oracle import oracle
    oracle.orc()
    return oracle


@pytest.fixture(scope="session")
def ref(orc):
    if not orc.ref_available():
        pytest.skip("reference oracle (oracle/_ref) not built")
    orc.ref()
    orc.ref_set_threads(1)  # sequential reductions: the FP32 pin is bit-exact
    return orc


@pytest.fixture(scope="session")
def device():
    if not cuda_available():
        pytest.skip("no CUDA device")
    return 0


def golden(name):
    return np.load(os.path.join(GOLDEN, name), allow_pickle=False)
