"""Oracle loader -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and the CPU-baseline leg of bench.py
import this module, and only as the checker.  The CUDA library never calls it.

Two back ends:

* ``Oracle`` -- the C restatement in oracle/nfft_oracle.c (long double inside),
  built into oracle/_build/liboracle_{d,f}.so.  Travels to the GPU box.
* ``Reference`` -- the reference itself, compiled from its own sources by
  oracle/Makefile into oracle/_ref/libref_*.so, called through its public C
  API (include/notorious_fft.h of the reference: notorious_fft_mkaux_*,
  notorious_fft_dft ... notorious_fft_free_aux).

Arrays are numpy; complex data is numpy complex (interleaved re/im in memory,
the reference's notorious_fft_cmpl layout).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
REFDIR = os.path.join(HERE, "_ref")

R2R_KINDS = {"dct2": 2, "dst2": 3, "dct3": 4, "dst3": 5, "dct4": 6, "dst4": 7}
KINDS = ("dft", "invdft", "realdft", "invrealdft") + tuple(R2R_KINDS)


# Where the reference project's sources are read from (its include/ and
# tests/ directories).  Only the recipes that compile them (oracle/Makefile,
# tests/refsuite/Makefile) and the compile check of its C++ wrapper read
# there; every other test uses what they built.  Set NOTORIOUS_FFT_REF_DIR to
# point elsewhere; without it the conventional read-only mount is used when
# present.
_DEFAULT_REF_DIR = "/root/reference"


def reference_dir():
    """The reference sources' directory, or None when they are not present."""
    d = os.environ.get("NOTORIOUS_FFT_REF_DIR") or _DEFAULT_REF_DIR
    return d if os.path.exists(os.path.join(d, "include", "notorious_fft.h")) else None


def build():
    """Build the C restatement (and the reference, when its sources exist)."""
    ref = reference_dir()
    subprocess.run(["make", "-s", "-C", HERE] + ([f"REF={ref}"] if ref else []), check=True)


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


class Oracle:
    """The C restatement, double (``single=False``) or float I/O."""

    def __init__(self, single: bool = False):
        self.single = single
        name = "liboracle_f.so" if single else "liboracle_d.so"
        path = os.path.join(BUILD, name)
        if not os.path.exists(path):
            build()
        self.lib = ctypes.CDLL(path, mode=os.RTLD_LOCAL)
        p = "oracle_f_" if single else "oracle_d_"
        self.rdt = np.float32 if single else np.float64
        self.cdt = np.complex64 if single else np.complex128
        L, I, V = ctypes.c_long, ctypes.c_int, ctypes.c_void_p
        self._dft = getattr(self.lib, p + "dft"); self._dft.argtypes = [V, V, L, I]
        self._rdft = getattr(self.lib, p + "realdft"); self._rdft.argtypes = [V, V, L]
        self._irdft = getattr(self.lib, p + "invrealdft"); self._irdft.argtypes = [V, V, L]
        self._r2r = getattr(self.lib, p + "r2r"); self._r2r.argtypes = [I, V, V, L]
        self._dftnd = getattr(self.lib, p + "dft_nd"); self._dftnd.argtypes = [I, V, V, V, I]
        self._r2rnd = getattr(self.lib, p + "r2r_nd"); self._r2rnd.argtypes = [I, I, V, V, V]
        self._rnd = getattr(self.lib, p + "realdft_nd"); self._rnd.argtypes = [I, V, V, V]
        self._irnd = getattr(self.lib, p + "invrealdft_nd"); self._irnd.argtypes = [I, V, V, V]
        for f in (self._dft, self._rdft, self._irdft, self._r2r, self._dftnd, self._r2rnd, self._rnd, self._irnd):
            f.restype = None

    # -- 1-D, applied over the last axis of a batched array ----------------
    def transform(self, kind: str, x: np.ndarray) -> np.ndarray:
        """Apply a 1-D transform along the last axis (batched over the rest)."""
        if kind in ("dft", "invdft"):
            x = np.ascontiguousarray(x, self.cdt)
            n = x.shape[-1]
            y = np.empty_like(x)
            xf, yf = x.reshape(-1, n), y.reshape(-1, n)
            for b in range(xf.shape[0]):
                self._dft(_ptr(xf[b]), _ptr(yf[b]), n, 1 if kind == "invdft" else 0)
            return y
        if kind == "realdft":
            x = np.ascontiguousarray(x, self.rdt)
            n = x.shape[-1]
            y = np.empty(x.shape[:-1] + (n // 2 + 1,), self.cdt)
            xf, yf = x.reshape(-1, n), y.reshape(-1, n // 2 + 1)
            for b in range(xf.shape[0]):
                self._rdft(_ptr(xf[b]), _ptr(yf[b]), n)
            return y
        if kind == "invrealdft":
            raise ValueError("use invrealdft(z, n)")
        code = R2R_KINDS[kind]
        x = np.ascontiguousarray(x, self.rdt)
        n = x.shape[-1]
        y = np.empty_like(x)
        xf, yf = x.reshape(-1, n), y.reshape(-1, n)
        for b in range(xf.shape[0]):
            self._r2r(code, _ptr(xf[b]), _ptr(yf[b]), n)
        return y

    def invrealdft(self, z: np.ndarray, n: int) -> np.ndarray:
        z = np.ascontiguousarray(z, self.cdt)
        y = np.empty(z.shape[:-1] + (n,), self.rdt)
        zf, yf = z.reshape(-1, n // 2 + 1), y.reshape(-1, n)
        for b in range(zf.shape[0]):
            self._irdft(_ptr(zf[b]), _ptr(yf[b]), n)
        return y

    # -- N-D ----------------------------------------------------------------
    def nd(self, kind: str, x: np.ndarray, dims=None) -> np.ndarray:
        """N-D transform of one array with shape ``dims`` (row-major)."""
        dims = tuple(x.shape) if dims is None else tuple(dims)
        Ns = (ctypes.c_int * len(dims))(*dims)
        d = len(dims)
        if kind in ("dft", "invdft"):
            x = np.ascontiguousarray(x, self.cdt)
            y = np.empty_like(x)
            self._dftnd(d, Ns, _ptr(x), _ptr(y), 1 if kind == "invdft" else 0)
            return y
        if kind == "realdft":
            x = np.ascontiguousarray(x, self.rdt)
            y = np.empty(dims[:-1] + (dims[-1] // 2 + 1,), self.cdt)
            self._rnd(d, Ns, _ptr(x), _ptr(y))
            return y
        if kind == "invrealdft":
            z = np.ascontiguousarray(x, self.cdt)
            y = np.empty(dims, self.rdt)
            self._irnd(d, Ns, _ptr(z), _ptr(y))
            return y
        x = np.ascontiguousarray(x, self.rdt)
        y = np.empty_like(x)
        self._r2rnd(R2R_KINDS[kind], d, Ns, _ptr(x), _ptr(y))
        return y


class Reference:
    """The reference library itself (compiled here from its own sources)."""

    VARIANTS = ("d_avx2", "d_scalar", "s_scalar", "s_avx2")

    def __init__(self, variant: str = "d_avx2"):
        path = os.path.join(REFDIR, f"libref_{variant}.so")
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.lib = ctypes.CDLL(path, mode=os.RTLD_LOCAL)
        self.single = variant.startswith("s_")
        self.rdt = np.float32 if self.single else np.float64
        self.cdt = np.complex64 if self.single else np.complex128
        V, I = ctypes.c_void_p, ctypes.c_int
        for fam in ("dft", "realdft", "t2t3", "t4"):
            f = getattr(self.lib, f"notorious_fft_mkaux_{fam}")
            f.argtypes = [I, V]
            f.restype = V
        for k in KINDS:
            f = getattr(self.lib, f"notorious_fft_{k}")
            f.argtypes = [V, V, V]
            f.restype = None
        self.lib.notorious_fft_free_aux.argtypes = [V]
        self.lib.notorious_fft_free_aux.restype = None

    @staticmethod
    def family(kind: str) -> str:
        if kind in ("dft", "invdft"):
            return "dft"
        if kind in ("realdft", "invrealdft"):
            return "realdft"
        if kind in ("dct4", "dst4"):
            return "t4"
        return "t2t3"

    def mkaux(self, kind, dims):
        dims = tuple(dims)
        Ns = (ctypes.c_int * len(dims))(*dims)
        a = getattr(self.lib, f"notorious_fft_mkaux_{self.family(kind)}")(len(dims), Ns)
        return a

    def run(self, kind: str, x: np.ndarray, dims, out_shape=None):
        """One call of notorious_fft_<kind> on an aux made for ``dims``."""
        a = self.mkaux(kind, dims)
        if not a:
            return None
        try:
            if kind in ("dft", "invdft"):
                x = np.ascontiguousarray(x, self.cdt)
                y = np.empty_like(x)
            elif kind == "realdft":
                x = np.ascontiguousarray(x, self.rdt)
                y = np.empty(tuple(dims[:-1]) + (dims[-1] // 2 + 1,), self.cdt)
            elif kind == "invrealdft":
                x = np.ascontiguousarray(x, self.cdt)
                y = np.empty(tuple(dims), self.rdt)
            else:
                x = np.ascontiguousarray(x, self.rdt)
                y = np.empty_like(x)
            getattr(self.lib, f"notorious_fft_{kind}")(_ptr(x), _ptr(y), a)
            return y
        finally:
            self.lib.notorious_fft_free_aux(a)


def ref_fill(n: int) -> np.ndarray:
    """Deterministic fixture of the reference tests: sin(1.23456789 i + 0.1 i^2)
    (tests/test_notoriousfft.c:45-48)."""
    i = np.arange(n, dtype=np.float64)
    return np.sin(i * 1.23456789 + 0.1 * i * i)


def rel_l2(a, b) -> float:
    a = np.asarray(a, dtype=np.complex128 if np.iscomplexobj(a) or np.iscomplexobj(b) else np.float64)
    b = np.asarray(b, dtype=a.dtype)
    nb = np.linalg.norm(b.ravel())
    d = np.linalg.norm((a - b).ravel())
    if nb == 0:
        return float(d)
    return float(d / nb)
