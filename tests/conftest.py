"""Shared test setup.

Markers: ``gpu`` tests need a B200 and call the CUDA path through the C ABI;
everything else runs on the CPU.  The CPU checker (``oracle``) is built on
first use; the native library is expected to be built (``__graft_entry__.build()``).
"""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


def gpu_present() -> bool:
    if shutil.which("nvidia-smi") is None:
        return False
    try:
        out = subprocess.run(["nvidia-smi", "-L"], capture_output=True, text=True, timeout=30)
    except Exception:
        return False
    return out.returncode == 0 and "GPU" in out.stdout


@pytest.fixture(scope="session")
def has_gpu():
    return gpu_present()


@pytest.fixture(scope="session")
def culbm():
    """The product package with its native library (fails loudly if unbuilt)."""
    import culbm_b200
    from culbm_b200 import _capi
    _capi.lib()
    return culbm_b200


@pytest.fixture(scope="session")
def orc():
    import oracle
    oracle.lib()
    return oracle
