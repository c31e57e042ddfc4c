"""Shared test setup: import paths, the `gpu` marker, and built libraries."""
import subprocess
import sys
from pathlib import Path

import pytest

REPO = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(REPO / "vocalsim-2p5d-fdtd_b200" / "python"))
sys.path.insert(0, str(REPO / "oracle"))
sys.path.insert(0, str(REPO))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); parity tests through the C ABI")


@pytest.fixture(scope="session", autouse=True)
def built_libraries():
    """Build the oracle and the solver library if they are missing (no-op when prebuilt)."""
    import oracle
    oracle.build()
    lib = REPO / "vocalsim-2p5d-fdtd_b200" / "lib" / "libvocalsim_b200.so"
    if not lib.exists():
        subprocess.run([sys.executable, str(REPO / "vocalsim-2p5d-fdtd_b200" / "build.py")], check=True)
    yield


@pytest.fixture(scope="session")
def cuda_ok():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("gpu test without a CUDA device")
    torch.cuda.init()
    return True
