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
    """Serial host emulation of the engine's warp algorithm (test only)."""
    import ctypes as C
    src = os.path.join(ROOT, "tests", "emu", "td_emu.cc")
    lib = os.path.join(ROOT, "tests", "emu", "libtdemu.so")
    if not os.path.exists(lib) or os.path.getmtime(lib) < max(
            os.path.getmtime(src), os.path.getmtime(os.path.join(ROOT, "td16_b200", "csrc", "td_core.cuh"))):
        subprocess.run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-fno-fast-math", "-ffp-contract=off",
                        "-o", lib, src], check=True)
    return C.CDLL(lib)


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
