import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
for p in (ROOT, ROOT / "vt-physics_b200", ROOT / "tests"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built sm_100a library")


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def oracle_lib():
    from oracle import build as ob
    ob.build()
    from oracle import oracle
    return oracle


@pytest.fixture(scope="session")
def vtp_gpu():
    if not gpu_available():
        pytest.skip("no CUDA device")
    import vtp
    vtp.lib()  # fails loudly when libvtp.so is missing
    return vtp
