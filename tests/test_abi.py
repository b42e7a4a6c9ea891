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


from oracle import reference_dir  # noqa: E402

_REF = reference_dir()
REF_HPP = os.path.join(_REF, "include", "notorious_fft.hpp") if _REF else ""


@pytest.mark.skipif(not _REF, reason="reference sources not present (set NOTORIOUS_FFT_REF_DIR)")
@pytest.mark.parametrize("single", [False, True], ids=["double", "float"])
def test_reference_cpp_wrapper_compiles_against_this_header(tmp_path, single):
    """The reference's C++17 wrapper (include/notorious_fft.hpp) builds
    unchanged on top of include/notorious_fft.h and links against the library.
    The wrapper is copied to a temporary directory at test time so that its
    #include "notorious_fft.h" resolves to this repository's header."""
    import shutil
    shutil.copy(REF_HPP, tmp_path / "notorious_fft.hpp")
    src = tmp_path / "app.cpp"
    src.write_text(
        '#include "notorious_fft.hpp"\n'
        "int main() {\n"
        "  auto a = notorious_fft::mkaux_dft_1d(64);\n"
        "  std::vector<notorious_fft_cmpl> x(64), y(64);\n"
        "  notorious_fft::dft(x.data(), y.data(), a);\n"
        "  std::vector<notorious_fft::complex_t> v(64);\n"
        "  auto w = notorious_fft::dft(v);\n"
        "  std::vector<notorious_fft::real_t> r(64);\n"
        "  auto z = notorious_fft::realdft(r);\n"
        "  return (int)(w.size() + z.size()) == 0;\n"
        "}\n")
    lib = default_path(single)
    if not os.path.exists(lib):
        pytest.skip("library not built")
    cmd = ["g++", "-std=c++17", "-c", "-I", str(tmp_path), "-I",
           os.path.join(ROOT, "include"), str(src), "-o", str(tmp_path / "app.o")]
    if single:
        cmd.insert(2, "-DNOTORIOUS_FFT_SINGLE")
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
    r = subprocess.run(["g++", str(tmp_path / "app.o"), "-o", str(tmp_path / "app"), lib,
                        "-Wl,-rpath," + os.path.dirname(lib)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
