import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.build()
    return O


@pytest.fixture(scope="session")
def emu():
    """Serial host emulation of the engine's warp algorithm (oracle/td_emu.cc, test only)."""
    import ctypes as C
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)
    return C.CDLL(os.path.join(ROOT, "oracle", "libtdemu.so"))


@pytest.fixture(scope="session")
def td():
    from td16_b200 import build
    build.build()
    import td16_b200
    return td16_b200


def has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
