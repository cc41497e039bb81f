import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an NVIDIA B200 (sm_100a) GPU")


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


HAS_GPU = _has_gpu()


@pytest.fixture(scope="session")
def gpu():
    if not HAS_GPU:
        pytest.skip("no CUDA device")
    import torch
    return torch.device("cuda:0")


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import oracle as O
    O.oracle_lib()
    return O


@pytest.fixture(scope="session")
def ref_mod(oracle_mod):
    if not oracle_mod.ref_available():
        pytest.skip("reference oracle library oracle/_ref/libccmref.so not built")
    return oracle_mod
