import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TESTS = os.path.dirname(os.path.abspath(__file__))
for p in (ROOT, TESTS):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 GPU and the CUDA engine library")
    config.addinivalue_line("markers", "slow: long-running CPU test")


@pytest.fixture(scope="session")
def emu_engine():
    """The host-emulation build of the engine kernels (test harness, CPU only)."""
    from profess_b200 import build, native
    path = build.build_emu()
    eng = native.Engine(path)
    yield eng
    eng.close()


@pytest.fixture(scope="session")
def gpu_engine():
    """The CUDA engine library on the first GPU.  Fails loudly if it is missing."""
    import torch
    assert torch.cuda.is_available(), "GPU test needs a CUDA device"
    from profess_b200 import native
    eng = native.Engine()
    yield eng
    eng.close()
