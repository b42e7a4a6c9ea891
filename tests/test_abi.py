"""The C-ABI libraries load and export every symbol include/notorious_fft.h
declares (CPU only; no compute calls without a GPU)."""
import ctypes
import os
import re
import subprocess

import pytest

from notorious_fft import EXTENSION_SYMBOLS, REFERENCE_SYMBOLS, default_path

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "notorious_fft.h")


def declared_symbols():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(notorious_fft_[a-z0-9_]+)\s*\(", text)))


@pytest.fixture(scope="module", params=[False, True], ids=["double", "float"])
def libpath(request):
    p = default_path(single=request.param)
    if not os.path.exists(p):
        pytest.skip("library not built")
    return p, request.param


def exported(path):
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True, check=True).stdout
    return {line.split()[-1] for line in out.splitlines() if " T " in line}


def test_header_declares_reference_api():
    decl = set(declared_symbols())
    assert set(REFERENCE_SYMBOLS) <= decl
    assert len(REFERENCE_SYMBOLS) == 27


def test_exports_every_declared_symbol(libpath):
    path, _ = libpath
    exp = exported(path)
    missing = [s for s in declared_symbols() if s not in exp]
    assert not missing, missing
    assert set(EXTENSION_SYMBOLS) <= exp


def test_no_unresolved_internal_symbols(libpath):
    path, _ = libpath
    out = subprocess.run(["nm", "-D", "--undefined-only", path], capture_output=True, text=True, check=True).stdout
    assert "nfft" not in out


def test_loads_and_reports_precision(libpath):
    path, single = libpath
    lib = ctypes.CDLL(path, mode=os.RTLD_LOCAL)
    lib.notorious_fft_real_size.restype = ctypes.c_int
    lib.notorious_fft_version.restype = ctypes.c_char_p
    assert lib.notorious_fft_real_size() == (4 if single else 8)
    assert b"sm_100a" in lib.notorious_fft_version()


def test_no_gpu_mkaux_returns_null():
    """Without a CUDA device every mkaux_* returns NULL with an error code
    (there is no CPU fallback)."""
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except Exception:
        pass
    lib = ctypes.CDLL(default_path(False), mode=os.RTLD_LOCAL)
    lib.notorious_fft_mkaux_dft_1d.restype = ctypes.c_void_p
    lib.notorious_fft_last_error.restype = ctypes.c_int
    assert not lib.notorious_fft_mkaux_dft_1d(16)
    assert lib.notorious_fft_last_error() != 0
