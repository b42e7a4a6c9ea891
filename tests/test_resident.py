"""Resident two-pass kernels (both Stockham passes of a batched complex DFT in
one persistent launch, the inter-pass scratch kept in L2), forced on for every
two-pass size in a child process (the switches are read once per process):
plain (NOTORIOUS_FFT_RESIDENT=1), software-pipelined
(NOTORIOUS_FFT_RESIDENT_PREFETCH=1) and fed by tensor copies through a stage
ring (NOTORIOUS_FFT_RESIDENT=2).  The child writes inputs and outputs; the
oracle checks them here.  The CPU variant runs the emulator build, which also
checks the work-order decode, the pass-1-before-pass-2 order of every
transform, each prefetched address against line_setup, and for the
tensor-copy form the box geometry, the 16-byte rule of the inner coordinate,
every copied element's address, the discarded scratch lines and the in-place
exchanges within the stage buffer.
"""
import os
import subprocess
import sys

import numpy as np
import pytest

from oracle import rel_l2

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r'''
import sys, numpy as np
sys.path.insert(0, sys.argv[1])
from notorious_fft import Library, load
path, out, single = sys.argv[2], sys.argv[3], sys.argv[4] == "f"
lib = Library(path) if path != "-" else load(single)
rng = np.random.default_rng(7)
res = {}
for n, B in [(int(a), int(b)) for a, b in (s.split("x") for s in sys.argv[5:])]:
    x = (rng.uniform(-1, 1, (B, n)) + 1j * rng.uniform(-1, 1, (B, n))).astype(lib.cdt)
    y = np.zeros_like(x); z = np.zeros_like(x)
    with lib.mkaux("dft", [n]) as a:
        a.batched("dft", x, y, B, n, n)
        a.batched("invdft", x, z, B, n, n)
    res[f"x{n}"], res[f"y{n}"], res[f"z{n}"] = x, y, z
f = getattr(lib.lib, "nfft_emu_resident_tma_launches", None)
if f is not None:
    import ctypes
    f.restype = ctypes.c_longlong
    res["tma_launches"] = np.array(f())
np.savez(out, **res)
'''


FORMS = {"plain": ("1", "0"), "prefetch": ("1", "1"), "tma": ("2", "0")}


def _run(tmp_path, path, prec, cases, form):
    out = str(tmp_path / "res.npz")
    mode, prefetch = FORMS[form]
    env = dict(os.environ, NOTORIOUS_FFT_RESIDENT=mode, NOTORIOUS_FFT_RESIDENT_PREFETCH=prefetch)
    r = subprocess.run([sys.executable, "-c", CHILD, os.path.join(ROOT, "notorious-fft_b200"), path, out, prec] + cases,
                       env=env, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-2000:]
    return np.load(out)


def _check(data, oracle, cases, tol):
    for c in cases:
        n = int(c.split("x")[0])
        x, y, z = data[f"x{n}"], data[f"y{n}"], data[f"z{n}"]
        for b in (0, x.shape[0] - 1):
            assert rel_l2(y[b], oracle.transform("dft", x[b])) <= tol * np.log2(n), (n, b, "dft")
            assert rel_l2(z[b], oracle.transform("invdft", x[b])) <= tol * np.log2(n), (n, b, "invdft")


@pytest.mark.parametrize("form", ["plain", "tma"])
@pytest.mark.parametrize("prec", ["d", "f"])
def test_resident_emulated(tmp_path, emu_d, oracle_d, prec, form):
    path = os.path.join(ROOT, "tests", "emu", "_build", "libnfft_emu_%s.so" % prec)
    cases = ["16384x3", "32768x1"] if form == "plain" else ["16384x3", "32768x2", "65536x1"]
    data = _run(tmp_path, path, prec, cases, form)
    _check(data, oracle_d, cases, 3e-15 if prec == "d" else 3e-6)
    if form == "tma":
        # two launches (dft, invdft) per case went through the tensor-copy form
        assert int(data["tma_launches"]) == 2 * len(cases)


@pytest.mark.gpu
@pytest.mark.parametrize("form", ["plain", "prefetch", "tma"])
@pytest.mark.parametrize("prec", ["d", "f"])
def test_resident_gpu(tmp_path, lib_d, oracle_d, prec, form):
    cases = ["8192x3", "16384x37", "65536x300", "131072x5", "524288x3", "1048576x2"]
    if form == "tma":
        cases += ["8192x1", "32768x1000", "262144x9"]
    _check(_run(tmp_path, "-", prec, cases, form), oracle_d, cases, 3e-15 if prec == "d" else 3e-6)
