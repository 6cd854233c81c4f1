import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built library")


def pytest_sessionstart(session):
    """The library is a build artefact (not in the repository): build it when a fresh checkout
    runs the tests before the build step."""
    import subprocess

    lib = os.path.join(ROOT, "staccato_b200", "libstaccato_rom.so")
    if not os.path.exists(lib):
        subprocess.run([sys.executable, os.path.join(ROOT, "staccato_b200", "build.py")], check=True)


@pytest.fixture(scope="session")
def cuda_device():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for gpu-marked tests")
    return torch.device("cuda:0")


@pytest.fixture(scope="session")
def handle(cuda_device):
    from staccato_b200 import _capi

    h = _capi.Handle(0)
    yield h
    h.close()
