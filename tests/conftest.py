"""Shared test setup.

Markers:
  gpu  -- needs a CUDA device (an sm_100 B200); run with `pytest -m gpu`.
CPU tests (`-m "not gpu"`) cover the oracle against the reference's golden
vectors, the host logic through the CPU emulator build (tests/emu), and the
C ABI export surface of the built libraries.
"""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "notorious-fft_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: requires a CUDA GPU (sm_100a)")


@pytest.fixture(scope="session")
def oracle_d():
    from oracle import Oracle
    return Oracle(single=False)


@pytest.fixture(scope="session")
def oracle_f():
    from oracle import Oracle
    return Oracle(single=True)


def _gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def lib_d():
    if not _gpu_available():
        pytest.skip("no CUDA device")
    from notorious_fft import load
    return load(single=False)


@pytest.fixture(scope="session")
def lib_f():
    if not _gpu_available():
        pytest.skip("no CUDA device")
    from notorious_fft import load
    return load(single=True)


@pytest.fixture(scope="session")
def emu_d():
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "tests", "emu")], check=True)
    from notorious_fft import Library
    return Library(os.path.join(ROOT, "tests", "emu", "_build", "libnfft_emu_d.so"))


@pytest.fixture(scope="session")
def emu_f():
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "tests", "emu")], check=True)
    from notorious_fft import Library
    return Library(os.path.join(ROOT, "tests", "emu", "_build", "libnfft_emu_f.so"))
