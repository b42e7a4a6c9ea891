"""Python binding of the B200 Notorious-FFT libraries (ctypes over the C ABI).

The functions mirror the reference C API (include/notorious_fft.h of
NotoriousLOB/Notorious-FFT): ``mkaux_*`` builds a plan, ``dft`` ... ``dst4``
run it, ``free_aux`` releases it.  Arrays may be numpy arrays (host memory;
the call stages them through the GPU and returns when the result is in
place) or CUDA torch tensors (device memory; the call is enqueued on the
library stream).  The libraries are loaded from ``notorious-fft_b200/lib``;
there is no CPU implementation behind this module -- if the shared library is
missing, loading raises.
"""
from __future__ import annotations

import ctypes
import os
from typing import Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
LIBDIR = os.path.join(PKG, "lib")

KINDS = ("dft", "invdft", "realdft", "invrealdft", "dct2", "dst2", "dct3", "dst3", "dct4", "dst4")
KIND_CODE = {k: i for i, k in enumerate(KINDS)}
FAMILY = {"dft": "dft", "invdft": "dft", "realdft": "realdft", "invrealdft": "realdft",
          "dct2": "t2t3", "dst2": "t2t3", "dct3": "t2t3", "dst3": "t2t3", "dct4": "t4", "dst4": "t4"}
FORM_PLAIN, FORM_SPLIT_TC = 0, 1

# Symbols of include/notorious_fft.h, for the export checks.
REFERENCE_SYMBOLS = (
    [f"notorious_fft_{k}" for k in KINDS]
    + [f"notorious_fft_mkaux_{f}{s}" for f in ("dft", "realdft", "t2t3", "t4") for s in ("_1d", "_2d", "_3d", "")]
    + ["notorious_fft_free_aux"]
)
EXTENSION_SYMBOLS = (
    [f"notorious_fft_{k}_batched" for k in KINDS]
    + [f"notorious_fft_{k}_vjp" for k in KINDS]
    + ["notorious_fft_vjp_batched", "notorious_fft_execute_batched", "notorious_fft_last_error",
       "notorious_fft_last_error_string", "notorious_fft_clear_error", "notorious_fft_set_stream",
       "notorious_fft_get_stream", "notorious_fft_synchronize", "notorious_fft_set_form", "notorious_fft_get_form",
       "notorious_fft_real_size", "notorious_fft_version", "notorious_fft_launch_count",
       "notorious_fft_dft_noalloc", "notorious_fft_mkbatch", "notorious_fft_batch_in_size",
       "notorious_fft_batch_out_size", "notorious_fft_batch_execute", "notorious_fft_batch_status",
       "notorious_fft_batch_set_graph", "notorious_fft_batch_info", "notorious_fft_free_batch",
       "notorious_fft_batch_debug_withhold", "notorious_fft_autotune", "notorious_fft_tune_lookup",
       "notorious_fft_tune_lookup_plan", "notorious_fft_aux_schedule"]
)


class NotoriousFFTError(RuntimeError):
    pass


def default_path(single: bool = False) -> str:
    return os.path.join(LIBDIR, "libnotorious_fftf.so" if single else "libnotorious_fft.so")


def _is_torch(a) -> bool:
    return type(a).__module__.startswith("torch")


class Library:
    """One loaded precision of the library (or a test build with the same ABI)."""

    def __init__(self, path: str | None = None, single: bool = False):
        path = path or default_path(single)
        if not os.path.exists(path):
            raise NotoriousFFTError(f"CUDA library not built: {path} (run notorious-fft_b200/build.py)")
        self.path = path
        self.lib = ctypes.CDLL(path, mode=os.RTLD_LOCAL)
        V, I, P = ctypes.c_void_p, ctypes.c_int, ctypes.c_ssize_t
        L = self.lib
        for f in ("dft", "realdft", "t2t3", "t4"):
            fn = getattr(L, f"notorious_fft_mkaux_{f}")
            fn.argtypes, fn.restype = [I, V], V
        for k in KINDS:
            for suffix, args in (("", [V, V, V]), ("_vjp", [V, V, V]), ("_batched", [V, V, V, I, P, P])):
                fn = getattr(L, f"notorious_fft_{k}{suffix}")
                fn.argtypes, fn.restype = args, None
        L.notorious_fft_free_aux.argtypes, L.notorious_fft_free_aux.restype = [V], None
        L.notorious_fft_execute_batched.argtypes = [I, V, V, V, I, P, P]
        L.notorious_fft_execute_batched.restype = None
        L.notorious_fft_vjp_batched.argtypes = [I, V, V, V, I, P, P]
        L.notorious_fft_vjp_batched.restype = None
        L.notorious_fft_last_error.restype = I
        L.notorious_fft_last_error_string.restype = ctypes.c_char_p
        L.notorious_fft_set_stream.argtypes = [V]
        L.notorious_fft_get_stream.restype = V
        L.notorious_fft_synchronize.restype = I
        L.notorious_fft_set_form.argtypes, L.notorious_fft_set_form.restype = [V, I], I
        L.notorious_fft_get_form.argtypes, L.notorious_fft_get_form.restype = [V], I
        L.notorious_fft_real_size.restype = I
        L.notorious_fft_version.restype = ctypes.c_char_p
        L.notorious_fft_launch_count.restype = ctypes.c_longlong
        LL = ctypes.c_longlong
        PLL = ctypes.POINTER(LL)
        L.notorious_fft_mkbatch.argtypes = [I, V, V, V, V]
        L.notorious_fft_mkbatch.restype = V
        L.notorious_fft_batch_in_size.argtypes = [V]
        L.notorious_fft_batch_in_size.restype = LL
        L.notorious_fft_batch_out_size.argtypes = [V]
        L.notorious_fft_batch_out_size.restype = LL
        L.notorious_fft_batch_execute.argtypes, L.notorious_fft_batch_execute.restype = [V, V, V], I
        L.notorious_fft_batch_status.argtypes, L.notorious_fft_batch_status.restype = [V], I
        L.notorious_fft_batch_set_graph.argtypes, L.notorious_fft_batch_set_graph.restype = [V, I], I
        L.notorious_fft_batch_info.argtypes = [V, PLL, PLL, PLL, ctypes.POINTER(I)]
        L.notorious_fft_batch_info.restype = I
        L.notorious_fft_free_batch.argtypes, L.notorious_fft_free_batch.restype = [V], None
        L.notorious_fft_batch_debug_withhold.argtypes = [V, LL]
        L.notorious_fft_batch_debug_withhold.restype = I
        L.notorious_fft_autotune.argtypes, L.notorious_fft_autotune.restype = [I, I], I
        L.notorious_fft_tune_lookup.argtypes, L.notorious_fft_tune_lookup.restype = [I, I, ctypes.POINTER(I), I], I
        PI = ctypes.POINTER(I)
        L.notorious_fft_tune_lookup_plan.argtypes = [I, I, PI, I, PI]
        L.notorious_fft_tune_lookup_plan.restype = I
        L.notorious_fft_aux_schedule.argtypes = [V, I, PI, I, PI]
        L.notorious_fft_aux_schedule.restype = I
        self.real_size = L.notorious_fft_real_size()
        self.single = self.real_size == 4
        self.rdt = np.float32 if self.single else np.float64
        self.cdt = np.complex64 if self.single else np.complex128
        # test builds (the CPU emulator) expose host-buffer registration hooks
        self._register = getattr(L, "nfft_emu_register_host", None)
        if self._register is not None:
            self._register.argtypes = [V, ctypes.c_size_t]
            self._unregister = L.nfft_emu_unregister_host
            self._unregister.argtypes = [V]

    # -- errors ---------------------------------------------------------------
    def last_error(self) -> tuple[int, str]:
        return self.lib.notorious_fft_last_error(), self.lib.notorious_fft_last_error_string().decode()

    def check(self):
        code, msg = self.last_error()
        if code:
            raise NotoriousFFTError(f"notorious_fft error {code}: {msg}")

    # -- plans ------------------------------------------------------------------
    def mkaux(self, family_or_kind: str, dims: Sequence[int]) -> "Aux":
        fam = FAMILY.get(family_or_kind, family_or_kind)
        dims = [int(d) for d in dims]
        arr = (ctypes.c_int * len(dims))(*dims)
        ptr = getattr(self.lib, f"notorious_fft_mkaux_{fam}")(len(dims), arr)
        if not ptr:
            code, msg = self.last_error()
            raise NotoriousFFTError(f"mkaux_{fam}{tuple(dims)} failed ({code}: {msg})")
        return Aux(self, ptr, fam, tuple(dims))

    def mkbatch(self, kinds: Sequence[str], Ns: Sequence[int], in_offsets=None, out_offsets=None) -> "Batch":
        """A ragged batch (one persistent launch for all transforms)."""
        return Batch(self, kinds, Ns, in_offsets, out_offsets)

    def autotune(self, kind: str, n: int) -> None:
        if self.lib.notorious_fft_autotune(KIND_CODE[kind], int(n)):
            self.check()

    def tune_lookup(self, kind: str, n: int) -> list:
        buf = (ctypes.c_int * 4)()
        k = self.lib.notorious_fft_tune_lookup(KIND_CODE[kind], int(n), buf, 4)
        return [buf[i] for i in range(min(k, 4))]

    def tune_lookup_plan(self, kind: str, n: int):
        """(split, logt) cached for standalone plans of kind's family and n, or None."""
        buf = (ctypes.c_int * 4)()
        lt = ctypes.c_int(0)
        k = self.lib.notorious_fft_tune_lookup_plan(KIND_CODE[kind], int(n), buf, 4, ctypes.byref(lt))
        if k < 0:
            return None
        return [buf[i] for i in range(min(k, 4))], lt.value

    def mkaux_raw(self, fam: str, dims: Sequence[int]):
        """The raw pointer (or None) -- mirrors the C convention of returning NULL."""
        arr = (ctypes.c_int * len(dims))(*[int(d) for d in dims])
        return getattr(self.lib, f"notorious_fft_mkaux_{fam}")(len(dims), arr)

    def mkaux_1d_raw(self, fam: str, n: int):
        fn = getattr(self.lib, f"notorious_fft_mkaux_{fam}_1d")
        fn.argtypes, fn.restype = [ctypes.c_int], ctypes.c_void_p
        return fn(int(n))

    def free_raw(self, ptr):
        self.lib.notorious_fft_free_aux(ptr)

    # -- streams ----------------------------------------------------------------
    def set_stream(self, stream) -> None:
        handle = getattr(stream, "cuda_stream", stream)
        self.lib.notorious_fft_set_stream(ctypes.c_void_p(int(handle) if handle else 0))

    def launch_count(self) -> int:
        return self.lib.notorious_fft_launch_count()

    def synchronize(self) -> None:
        if self.lib.notorious_fft_synchronize():
            self.check()

    # -- calls ------------------------------------------------------------------
    def _ptr(self, a):
        if a is None:
            return None
        if isinstance(a, int):
            return a
        if _is_torch(a):
            return a.data_ptr()
        return a.ctypes.data

    def _call(self, fn, x, y, aux, *extra, regs=()):
        hooks = []
        if self._register is not None:
            for a in (x, y):
                if isinstance(a, np.ndarray):
                    self._register(a.ctypes.data, a.nbytes)
                    hooks.append(a.ctypes.data)
        try:
            fn(self._ptr(x), self._ptr(y), aux.ptr, *extra)
        finally:
            for h in hooks:
                self._unregister(h)
        self.check()


class Aux:
    """A plan handle (notorious_fft_aux*).  Use as a context manager or free()."""

    def __init__(self, lib: Library, ptr: int, family: str, dims: tuple):
        self.L, self.ptr, self.family, self.dims = lib, ptr, family, dims

    def free(self):
        if self.ptr:
            self.L.lib.notorious_fft_free_aux(self.ptr)
            self.ptr = None

    __del__ = free

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.free()

    def set_form(self, form: int) -> None:
        if self.L.lib.notorious_fft_set_form(self.ptr, form):
            self.L.check()

    @property
    def form(self) -> int:
        return self.L.lib.notorious_fft_get_form(self.ptr)

    def schedule(self, axis: int = -1):
        """(pass radices log2, threads log2 or 0) of an axis's inner power-of-two FFT."""
        buf = (ctypes.c_int * 4)()
        lt = ctypes.c_int(0)
        k = self.L.lib.notorious_fft_aux_schedule(self.ptr, int(axis), buf, 4, ctypes.byref(lt))
        if k < 0:
            self.L.check()
        return [buf[i] for i in range(min(k, 4))], lt.value

    # shapes of one transform
    def in_shape(self, kind: str) -> tuple:
        if kind == "invrealdft":
            return self.dims[:-1] + (self.dims[-1] // 2 + 1,)
        return self.dims

    def out_shape(self, kind: str) -> tuple:
        if kind == "realdft":
            return self.dims[:-1] + (self.dims[-1] // 2 + 1,)
        return self.dims

    def _dtype(self, kind: str, side: str):
        cplx = {"in": kind in ("dft", "invdft", "invrealdft"), "out": kind in ("dft", "invdft", "realdft")}[side]
        return self.L.cdt if cplx else self.L.rdt

    def __call__(self, kind: str, x, y=None):
        """One transform (numpy in -> numpy out, or device tensors)."""
        if y is None:
            if _is_torch(x):
                raise ValueError("pass an output tensor for device calls")
            y = np.empty(self.out_shape(kind), self._dtype(kind, "out"))
        if not _is_torch(x):
            x = np.ascontiguousarray(x, self._dtype(kind, "in"))
        self.L._call(getattr(self.L.lib, f"notorious_fft_{kind}"), x, y, self)
        return y

    def batched(self, kind: str, x, y, howmany: int, idist: int, odist: int):
        self.L._call(getattr(self.L.lib, f"notorious_fft_{kind}_batched"), x, y, self, int(howmany), int(idist),
                     int(odist))
        return y

    def vjp(self, kind: str, g, gx=None):
        """Adjoint of `kind`: g has the output's shape, the result the input's."""
        if gx is None:
            if _is_torch(g):
                raise ValueError("pass an output tensor for device calls")
            gx = np.empty(self.in_shape(kind), self._dtype(kind, "in"))
        if not _is_torch(g):
            g = np.ascontiguousarray(g, self._dtype(kind, "out"))
        self.L._call(getattr(self.L.lib, f"notorious_fft_{kind}_vjp"), g, gx, self)
        return gx

    def vjp_batched(self, kind: str, g, gx, howmany: int, idist: int, odist: int):
        self.L._call_vjp_batched(kind, g, gx, self, howmany, idist, odist)
        return gx


def _call_vjp_batched(self, kind, g, gx, aux, howmany, idist, odist):
    hooks = []
    if self._register is not None:
        for a in (g, gx):
            if isinstance(a, np.ndarray):
                self._register(a.ctypes.data, a.nbytes)
                hooks.append(a.ctypes.data)
    try:
        self.lib.notorious_fft_vjp_batched(KIND_CODE[kind], self._ptr(g), self._ptr(gx), aux.ptr, int(howmany),
                                           int(idist), int(odist))
    finally:
        for h in hooks:
            self._unregister(h)
    self.check()


Library._call_vjp_batched = _call_vjp_batched


class Batch:
    """A ragged batch: transform i is kinds[i] of length Ns[i], reading
    in[in_offsets[i]:] and writing out[out_offsets[i]:] (offsets in reals;
    None: packed layout).  Buffers are flat real arrays (numpy or CUDA torch)
    of at least in_size / out_size reals."""

    def __init__(self, lib: Library, kinds, Ns, in_offsets=None, out_offsets=None):
        self.L = lib
        self.kinds = [KIND_CODE[k] if isinstance(k, str) else int(k) for k in kinds]
        self.Ns = [int(n) for n in Ns]
        count = len(self.kinds)
        ka = np.ascontiguousarray(self.kinds, dtype=np.int32)
        na = np.ascontiguousarray(self.Ns, dtype=np.int32)
        ia = None if in_offsets is None else np.ascontiguousarray(in_offsets, dtype=np.int64)
        oa = None if out_offsets is None else np.ascontiguousarray(out_offsets, dtype=np.int64)
        self.ptr = lib.lib.notorious_fft_mkbatch(count, ka.ctypes.data, na.ctypes.data,
                                                 None if ia is None else ia.ctypes.data,
                                                 None if oa is None else oa.ctypes.data)
        if not self.ptr:
            code, msg = lib.last_error()
            raise NotoriousFFTError(f"mkbatch failed ({code}: {msg})")
        self.in_size = lib.lib.notorious_fft_batch_in_size(self.ptr)
        self.out_size = lib.lib.notorious_fft_batch_out_size(self.ptr)

    def free(self):
        if getattr(self, "ptr", None):
            self.L.lib.notorious_fft_free_batch(self.ptr)
            self.ptr = None

    __del__ = free

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.free()

    def execute(self, x, y):
        """Run the batch; host arrays return when done, device tensors are asynchronous."""
        L = self.L
        hooks = []
        if L._register is not None:
            for a in (x, y):
                if isinstance(a, np.ndarray):
                    L._register(a.ctypes.data, a.nbytes)
                    hooks.append(a.ctypes.data)
        try:
            rc = L.lib.notorious_fft_batch_execute(self.ptr, L._ptr(x), L._ptr(y))
        finally:
            for h in hooks:
                L._unregister(h)
        if rc:
            L.check()
            raise NotoriousFFTError(f"batch execute returned {rc}")
        return y

    def status(self) -> int:
        return self.L.lib.notorious_fft_batch_status(self.ptr)

    def set_graph(self, on: bool) -> None:
        self.L.lib.notorious_fft_batch_set_graph(self.ptr, 1 if on else 0)

    def withhold(self, spin_limit: int) -> None:
        self.L.lib.notorious_fft_batch_debug_withhold(self.ptr, int(spin_limit))

    def info(self) -> dict:
        it, tl, sc = ctypes.c_longlong(), ctypes.c_longlong(), ctypes.c_longlong()
        ctas = ctypes.c_int()
        self.L.lib.notorious_fft_batch_info(self.ptr, ctypes.byref(it), ctypes.byref(tl), ctypes.byref(sc),
                                            ctypes.byref(ctas))
        return {"items": it.value, "tiles": tl.value, "scratch_bytes": sc.value, "ctas": ctas.value}


_LIBS: dict = {}


def load(single: bool = False) -> Library:
    """The product library of the given precision (cached)."""
    key = bool(single)
    if key not in _LIBS:
        _LIBS[key] = Library(single=single)
    return _LIBS[key]
